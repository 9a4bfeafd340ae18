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
