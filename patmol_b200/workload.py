"""Quartet-class bookkeeping and the algorithmic FP64 work of the Fock build.

Counts follow the kernels' enumeration: unique shell pairs (i >= j, both
with components), the larger l first, pairs ordered by class; unique
quartets are pairs-of-pairs (u >= v), i.e. the 8-fold symmetric set the
reference enumerates in twoints.c:228-295.

Algorithmic flops of one primitive shell quartet of class (la lb|lc ld) with
n = (la+lb+lc+ld)/2 + 1 Rys roots, in the canonical Rys scheme the kernels
implement (counts of FP64 operations, an FMA counted as two):
  roots/weights  2n Chebyshev series of degree 11 (Clenshaw, 2 FMA a term)
  recursion      3n (L12+1)(L34+1) table entries, 4 flops each
  transfer       3n sum_{a,b,c,d} (b+1)(d+1) FMA
  assembly       n FMA + n MUL per component integral (3n flops)
  digestion      six dot-product terms per integral (12 flops, RHF)
"""
from __future__ import annotations

from collections import Counter

from .basis import ncart

RYS_DEG = 11


def pair_class_counts(basis):
    c = Counter()
    shells = [s for s in basis.shells if s.nst > 0]
    for i in range(len(shells)):
        for j in range(i + 1):
            la, lb = shells[i].l, shells[j].l
            if la < lb:
                la, lb = lb, la
            c[(la, lb)] += 1
    return c


def class_key(p):
    la, lb = p
    return la * (la + 1) // 2 + lb


def quartet_class_counts(basis):
    """Unscreened unique shell quartets per class (la, lb, lc, ld)."""
    pc = pair_class_counts(basis)
    keys = sorted(pc, key=class_key)
    out = {}
    for iu, u in enumerate(keys):
        for v in keys[:iu + 1]:
            n = pc[u] * pc[v] if u != v else pc[u] * (pc[u] + 1) // 2
            out[u + v] = n
    return out


def nroots(cls):
    return sum(cls) // 2 + 1


def roots_histogram(counts):
    h = Counter()
    for cls, n in counts.items():
        h[nroots(cls)] += n
    return dict(sorted(h.items()))


def flops_per_quartet(cls, mode="rhf"):
    la, lb, lc, ld = cls
    n = nroots(cls)
    ncart_q = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    roots = 2 * n * 2 * (RYS_DEG + 1)
    vrr = 3 * n * (la + lb + 1) * (lc + ld + 1) * 4
    hrr = 3 * n * sum((b + 1) * (d + 1) * 2 for a in range(la + 1) for b in range(lb + 1)
                      for c in range(lc + 1) for d in range(ld + 1))
    assembly = 3 * n * ncart_q
    digest = {"rhf": 12, "jk": 12, "uhf": 20}[mode] * ncart_q
    return roots + vrr + hrr + assembly + digest


def fock_flops(class_counts, mode="rhf", nprim_quartets=None):
    """class_counts: iterable of ((la,lb,lc,ld), count)."""
    tot = 0
    for cls, cnt in class_counts:
        tot += cnt * flops_per_quartet(tuple(cls), mode)
    return tot


def shell_pairs(basis):
    """Shell pairs in the library's order: both shells with components, the
    larger l first, stable-sorted by pair class."""
    out = []
    for i, si in enumerate(basis.shells):
        if not si.nst:
            continue
        for j in range(i + 1):
            sj = basis.shells[j]
            if not sj.nst:
                continue
            a, b = (i, j) if si.l >= sj.l else (j, i)
            out.append((class_key((basis.shells[a].l, basis.shells[b].l)), a, b))
    out.sort(key=lambda t: t[0])        # Python's sort is stable
    return [(a, b) for _, a, b in out]


def enumerate_quartets(basis, rank=0, nranks=1, start_shell=0):
    """Unscreened quartets (bra pair, ket pair) owned by `rank`: per class
    pair (bra class >= ket class), bra-major order, every nranks-th one."""
    pairs = shell_pairs(basis)
    cls = [class_key((basis.shells[a].l, basis.shells[b].l)) for a, b in pairs]
    by = {}
    for u, c in enumerate(cls):
        by.setdefault(c, []).append(u)
    out = []
    for cu in sorted(by):
        for cv in sorted(by):
            if cv > cu:
                continue
            k = 0
            for u in by[cu]:
                for v in by[cv]:
                    if cu == cv and v > u:
                        break
                    if max(pairs[u] + pairs[v]) < start_shell:
                        continue
                    if k % nranks == rank:
                        out.append((u, v))
                    k += 1
    return pairs, out
