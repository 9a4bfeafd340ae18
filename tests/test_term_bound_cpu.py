"""The mixed-precision window of the library (library.cu, term_bound) sends a
quartet to FP32 when an estimate of the largest term of its Rys quadrature
is below tau_fp32, because FP32 rounding scales with those terms and not
with the integral (which the Schwarz bound limits).  This checks on the CPU
that the estimate is an upper bound: for sampled quartets of two bases with
diffuse and tight shells, every product Ix Iy Iz the quadrature sums (per
root and Cartesian component, with the weight and prefactor in the z
factor), computed in FP64 with the oracle's Rys roots, stays below it.

The estimate restated: per primitive pair, 2 pi^(5/2) |K_ab K_cd| /
sqrt(p+q) * S_bra^(la+lb) * S_ket^(lc+ld) with S_bra = 2|A-B| +
q/(p+q)|P-Q| + sqrt((la+lb+1)/2p) and S_ket likewise."""
import math

import numpy as np
import pytest

import patref
from patmol_b200 import configs

KSR = 2.0 * math.pi ** 2.5


def term_bound(la, lb, lc, ld, A, B, C, D, a, b, c, d, Kab, Kcd):
    p, q = a + b, c + d
    P, Q = (a * A + b * B) / p, (c * C + d * D) / q
    R = float(np.linalg.norm(P - Q))
    lab, lcd = la + lb, lc + ld
    sb = 2.0 * np.linalg.norm(A - B) + q / (p + q) * R + math.sqrt((lab + 1) / (2.0 * p))
    sk = 2.0 * np.linalg.norm(C - D) + p / (p + q) * R + math.sqrt((lcd + 1) / (2.0 * q))
    return KSR * abs(Kab * Kcd) / math.sqrt(p + q) * sb ** lab * sk ** lcd


def rys_tables(la, lb, lc, ld, g00, B00, B10, B01, C, Cp, ab, cd):
    """One root and direction: the 2-D recursion and the binomial transfer
    (the kernels' vrr_hrr), table[a, b, c, d]."""
    L12, L34 = la + lb, lc + ld
    G = np.zeros((L12 + 1, L34 + 1))
    G[0, 0] = g00
    if L12 > 0:
        G[1, 0] = C * g00
    for i in range(1, L12):
        G[i + 1, 0] = i * B10 * G[i - 1, 0] + C * G[i, 0]
    for j in range(L34):
        for i in range(L12 + 1):
            v = Cp * G[i, j]
            if j > 0:
                v += j * B01 * G[i, j - 1]
            if i > 0:
                v += i * B00 * G[i - 1, j]
            G[i, j + 1] = v
    T = np.zeros((la + 1, lb + 1, lc + 1, ld + 1))
    for c in range(lc + 1):
        for d in range(ld + 1):
            H = [sum(math.comb(d, k) * cd ** k * G[i, c + d - k] for k in range(d + 1)) for i in range(L12 + 1)]
            for a in range(la + 1):
                for b in range(lb + 1):
                    T[a, b, c, d] = sum(math.comb(b, k) * ab ** k * H[a + b - k] for k in range(b + 1))
    return T


def cart(l):
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1)]


def largest_term(la, lb, lc, ld, A, B, C, D, a, b, c, d, Kab, Kcd):
    p, q = a + b, c + d
    P, Q = (a * A + b * B) / p, (c * C + d * D) / q
    sr = KSR * Kab * Kcd / math.sqrt(p + q)
    n = (la + lb + lc + ld) // 2 + 1
    x, w = patref.Oracle.rys(n, p * q / (p + q) * float((P - Q) @ (P - Q)))
    big = 0.0
    for r in range(n):
        f = x[r] / (p + q)
        B00 = 0.5 * f
        B10, B01 = (0.5 - B00 * q) / p, (0.5 - B00 * p) / q
        tabs = [rys_tables(la, lb, lc, ld, w[r] * sr if dim == 2 else 1.0, B00, B10, B01,
                           (P - A)[dim] - q * (P - Q)[dim] * f, (Q - C)[dim] + p * (P - Q)[dim] * f,
                           (A - B)[dim], (C - D)[dim]) for dim in range(3)]
        for ea in cart(la):
            for eb in cart(lb):
                for ec in cart(lc):
                    for ed in cart(ld):
                        t = 1.0
                        for dim in range(3):
                            t *= tabs[dim][ea[dim], eb[dim], ec[dim], ed[dim]]
                        big = max(big, abs(t))
    return big


@pytest.mark.parametrize("which", ["organic4_spdf", "water_spdf_positron"])
def test_term_bound_covers_every_quadrature_term(which):
    b = configs.organic_basis(4, 11, with_f=True) if which == "organic4_spdf" else configs.water_spdf_positron()
    shells = [s for s in b.shells if s.nst > 0]
    rng = np.random.default_rng(5)
    tested = 0
    for _ in range(500):
        s = [shells[k] for k in rng.integers(0, len(shells), 4)]
        if s[0].l < s[1].l:
            s[0], s[1] = s[1], s[0]
        if s[2].l < s[3].l:
            s[2], s[3] = s[3], s[2]
        A, B, C, D = (b.coords[x.cen] for x in s)
        a, bb, c, d = (x.alpha[0] for x in s)
        Kab = s[0].coef[0] * s[1].coef[0] * math.exp(-a * bb / (a + bb) * float((A - B) @ (A - B))) / (a + bb)
        Kcd = s[2].coef[0] * s[3].coef[0] * math.exp(-c * d / (c + d) * float((C - D) @ (C - D))) / (c + d)
        args = (s[0].l, s[1].l, s[2].l, s[3].l, A, B, C, D, a, bb, c, d, Kab, Kcd)
        big, bound = largest_term(*args), term_bound(*args)
        assert big <= bound * (1.0 + 1e-12), (args[:4], big, bound)
        tested += 1
    assert tested == 500
