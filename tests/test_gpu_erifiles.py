"""The reference's ERI files written from the GPU integrals
(patgpu_write_eri_files), against the reference's own files.

Records are compared in stream order.  Values agree within 1e-12 except in
quartets that hit the reference's inexact Rys roots (test_oracle.rys_defect);
a record present on one side only must lie within 1e-13 of the 1e-14 record
threshold or come from such a quartet.  Also: the card-dealt split over MPI
ranks reproduces the single-rank records, and file rollover only cuts the
stream into files.
"""
import os

import numpy as np
import pytest

from conftest import golden
from patmol_b200 import configs
import patref

from golden.make_golden import mini_basis  # noqa: E402
from test_oracle import f2s_map, quartet_T, rys_defect  # noqa: E402

pytestmark = pytest.mark.gpu

gpu = pytest.importorskip("patmol_b200.gpu")


def keys(r):
    return (r["i"].astype(np.uint64) << 48) | (r["j"].astype(np.uint64) << 32) | \
        (r["k"].astype(np.uint64) << 16) | r["l"].astype(np.uint64)


def defect(basis, f2s, i, j, k, l):
    q = (f2s[i][0], f2s[j][0], f2s[k][0], f2s[l][0])
    n = sum(basis.shells[s].l for s in q) // 2 + 1
    return any(rys_defect(n, t) for t in quartet_T(basis, *q))


def compare_streams(basis, got, ref):
    f2s = f2s_map(basis)
    kg, kr = keys(got), keys(ref)
    only_g = ~np.isin(kg, kr)
    only_r = ~np.isin(kr, kg)
    for rec, mask in ((got, only_g), (ref, only_r)):
        for x in rec[mask]:
            assert abs(x["val"]) < 1e-13 or defect(basis, f2s, x["i"], x["j"], x["k"], x["l"]), x
    g, r = got[~only_g], ref[~only_r]
    assert np.array_equal(keys(g), keys(r))          # same records in the same order
    bad = np.nonzero(np.abs(g["val"] - r["val"]) > 1e-12)[0]
    for t in bad:
        assert defect(basis, f2s, g["i"][t], g["j"][t], g["k"][t], g["l"][t]), (g[t], r[t])
    return len(g), len(bad)


def write(basis, tmp_path, **kw):
    h = gpu.GpuBasis(basis)
    prefix = str(tmp_path) + os.sep
    numints = h.write_eri_files(prefix, "MINTS.DAT", **kw)
    rank = kw.get("rank", 0)
    recs = gpu.read_eri_files(prefix, "MINTS.DAT", rank, len(numints))
    assert len(recs) == sum(numints)
    h.close()
    return recs, numints


def test_mini_basis_against_reference_records(tmp_path):
    b = mini_basis()
    g = golden("mini_ints.npz")
    ref = np.zeros(len(g["val"]), dtype=gpu.ERINT_DTYPE)
    for f in ("val", "i", "j", "k", "l"):
        ref[f] = g[f]
    got, _ = write(b, tmp_path)
    n, nbad = compare_streams(b, got, ref)
    assert n > 0.99 * len(ref)


def test_water_spd_against_reference_files(tmp_path):
    b = configs.water_spd()
    _, outs = patref.run_ref(b, ["ints"], outputs=["eri.bin"])
    ref = outs["eri.bin"]
    got, numints = write(b, tmp_path)
    n, nbad = compare_streams(b, got, ref)
    assert n > 0.999 * len(ref) and len(ref) > 1.7e7


def test_rank_split_and_file_rollover(tmp_path):
    b = mini_basis()
    d = tmp_path / "one"
    d.mkdir()
    one, _ = write(b, d)
    parts = []
    for r in range(3):
        d = tmp_path / f"r{r}"
        d.mkdir()
        recs, _ = write(b, d, rank=r, nproc=3)
        parts.append(recs)
    merged = np.concatenate(parts)
    assert len(merged) == len(one)
    assert np.array_equal(np.sort(keys(merged)), np.sort(keys(one)))
    d = tmp_path / "small"
    d.mkdir()
    small, numints = write(b, d, max_records=500)
    assert len(numints) > 3
    assert all(c > 500 for c in numints[:-1])
    assert np.array_equal(keys(small), keys(one)) and np.array_equal(small["val"], one["val"])
