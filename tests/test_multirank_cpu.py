"""The multi-GPU Fock build's host logic on CPU ranks (gloo, world size 2):
every rank digests its class-strided share of the shell quartets into a
partial n x n accumulator with the degeneracy-factor rule the kernels use,
the partials are summed with one all-reduce, and G = A + A^T must equal the
reference-order digestion of the restatement."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from patmol_b200 import workload
from patmol_b200.basis import unpack, pack


def digest_partial(basis, oracle, P, rank, nranks):
    """Python statement of the kernels' digestion (eri.cu header)."""
    n = basis.norb
    D = unpack(P, n)
    A = np.zeros((n, n))
    pairs, quartets = workload.enumerate_quartets(basis, rank, nranks)
    sh = basis.shells
    for u, v in quartets:
        a, b = pairs[u]
        c, d = pairs[v]
        blk = oracle.eri_block(a, b, c, d)
        deg = (1 if a == b else 2) * (1 if c == d else 2) * (1 if u == v else 2)
        fa, fb, fc, fd = sh[a].off, sh[b].off, sh[c].off, sh[d].off
        ia, ib, ic, id_ = (np.arange(sh[s].nst) for s in (a, b, c, d))
        Dab, Dcd = D[np.ix_(fa + ia, fb + ib)], D[np.ix_(fc + ic, fd + id_)]
        Dbd, Dbc = D[np.ix_(fb + ib, fd + id_)], D[np.ix_(fb + ib, fc + ic)]
        Dad, Dac = D[np.ix_(fa + ia, fd + id_)], D[np.ix_(fa + ia, fc + ic)]
        sJ, sK = 0.5 * deg, 0.125 * deg
        A[np.ix_(fa + ia, fb + ib)] += sJ * np.einsum("ijkl,kl->ij", blk, Dcd)
        A[np.ix_(fc + ic, fd + id_)] += sJ * np.einsum("ijkl,ij->kl", blk, Dab)
        A[np.ix_(fa + ia, fc + ic)] -= sK * np.einsum("ijkl,jl->ik", blk, Dbd)
        A[np.ix_(fa + ia, fd + id_)] -= sK * np.einsum("ijkl,jk->il", blk, Dbc)
        A[np.ix_(fb + ib, fc + ic)] -= sK * np.einsum("ijkl,il->jk", blk, Dad)
        A[np.ix_(fb + ib, fd + id_)] -= sK * np.einsum("ijkl,ik->jl", blk, Dac)
    return A


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    import torch
    import patref
    from golden.make_golden import mini_basis, seeded_density
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = mini_basis()
    O = patref.Oracle(b)
    P = seeded_density(b.norb, 9)
    A = torch.from_numpy(digest_partial(b, O, P, rank, world))
    dist.all_reduce(A)
    G = pack((A + A.T).numpy())
    if rank == 0:
        ref = O.gmat(P)
        out.put(float(np.abs(G - ref).max()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_fock_build_matches_oracle():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    err = q.get(timeout=10)
    assert err < 1e-11, err


def test_partition_covers_every_quartet_once():
    from golden.make_golden import mini_basis
    b = mini_basis()
    _, whole = workload.enumerate_quartets(b, 0, 1)
    parts = []
    for r in range(3):
        parts += workload.enumerate_quartets(b, r, 3)[1]
    assert sorted(parts) == sorted(whole)
    assert len(whole) == sum(workload.quartet_class_counts(b).values())


# ---------------------------------------------------------------------------
# Fixed-point accumulation (the library's deterministic mode): the device
# conversion of one contribution (acc_add in eri.cuh) and the finishing sum
# (fix_sum), restated with numpy integers.
FIX_HI = 2.0 ** 28
FIX_LO = 2.0 ** 32
SHIFT = 1.5 * 2.0 ** 52


def _bits(x):
    return np.asarray(x, dtype=np.float64).view(np.int64)


def to_fixed(v):
    """Contributions (float64 array) -> (low word, high word) int64 arrays:
    the 1.5 * 2^52 shift rounds to the nearest integer."""
    sc = np.asarray(v, dtype=np.float64) * FIX_HI
    t = sc + SHIFT
    hi = _bits(t) - _bits(SHIFT)
    r = sc - (t - SHIFT)
    lo = _bits(r * FIX_LO + SHIFT) - _bits(SHIFT)   # r * 2^32 is exact, so fma = mul + add here
    return lo, hi


def fixed_value(lo, hi):
    h = hi + (lo >> 32)
    return h.astype(np.float64) / FIX_HI + (lo & 0xffffffff).astype(np.float64) / (FIX_HI * FIX_LO)


def test_fixed_point_sum_is_order_independent_and_exact():
    import math
    rng = np.random.default_rng(3)
    # contributions spanning many magnitudes and both signs, as J/K targets see
    v = rng.normal(size=20000) * 10.0 ** rng.uniform(-14, 1, size=20000)
    lo, hi = to_fixed(v)
    sums = set()
    for seed in range(5):
        perm = np.random.default_rng(seed).permutation(v.size)
        L = np.int64(0)
        H = np.int64(0)
        for k in perm[:2000]:            # a scalar walk in a random order
            L += lo[k]
            H += hi[k]
        L += lo[perm[2000:]].sum()
        H += hi[perm[2000:]].sum()
        sums.add(float(fixed_value(np.array([L]), np.array([H]))[0]).hex())
    assert len(sums) == 1
    exact = math.fsum(v)
    got = float.fromhex(sums.pop())
    assert abs(got - exact) < 1e-13 * max(1.0, abs(exact)) + v.size * 2.0 ** -60


def _fixed_worker(rank, world, port, out):
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(11)
    v = rng.normal(size=(4096, 16)) * 10.0 ** rng.uniform(-12, 1, size=(4096, 16))
    # rank r owns every world-th row (the class-strided split), summed in its own order
    lo, hi = to_fixed(v[rank::world])
    A = torch.from_numpy(np.stack([lo.sum(axis=0), hi.sum(axis=0)]))
    dist.all_reduce(A)
    if rank == 0:
        lo1, hi1 = to_fixed(v)
        whole = fixed_value(lo1.sum(axis=0), hi1.sum(axis=0))
        split = fixed_value(A[0].numpy(), A[1].numpy())
        out.put(whole.tobytes() == split.tobytes())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_fixed_point_reduce_matches_single_rank_bitwise():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + os.getpid() % 1000
    procs = [ctx.Process(target=_fixed_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    assert q.get(timeout=10) is True
