"""Mixed precision: quartets whose Rys-term bound is below 1e-8 run in FP32
arithmetic with FP64 accumulation.  Checked against the all-FP64 build at a
physical density (the core-Hamiltonian guess): the first-order energy error
tr(P dG) must stay below 1e-6 Eh and G below 1e-9 elementwise (the
term bound keeps each FP32 integral's error near 1e-7 of 1e-8)."""
import numpy as np
import pytest

from patmol_b200 import configs
from patmol_b200.basis import unpack, pack

pytestmark = pytest.mark.gpu

gpu = pytest.importorskip("patmol_b200.gpu")


def core_guess_density(G, nocc):
    """P = C_occ C_occ^T of the core Hamiltonian in the orthogonalised basis
    (rhfscf.c:433-471), the reference's own starting density."""
    n = G.n
    S, T, H = G.one_electron_ints()
    Sf, Hf = unpack(S, n), unpack(H, n)
    e, U = np.linalg.eigh(Sf)
    X = U / np.sqrt(e)
    w, V = np.linalg.eigh(X.T @ Hf @ X)
    C = X @ V[:, :nocc]
    return pack(C @ C.T)


def mixed_vs_fp64(basis, tau_fp32=1e-8):
    G = gpu.GpuBasis(basis)
    P = core_guess_density(G, basis.nelec // 2)
    g64 = G.rhf_form_gmatrix(P)
    nfp32 = G.set_mixed_precision(tau_fp32)
    gmx = G.rhf_form_gmatrix(P)
    G.set_mixed_precision(0.0)
    n = basis.norb
    de = float(np.sum(unpack(P, n) * unpack(gmx - g64, n)))
    return nfp32, G.stats()["quartets"], float(np.abs(gmx - g64).max()), de


@pytest.mark.parametrize("variant32", [None, "smem"])
def test_mixed_water_spdf_positron(variant32, monkeypatch):
    """Tuned (the library may keep a small FP32 window on the class's FP64
    kernel, and then counts it as FP64) and with the FP32 kernel forced."""
    if variant32 is None:
        monkeypatch.delenv("PATGPU_VARIANT32", raising=False)
    else:
        monkeypatch.setenv("PATGPU_VARIANT32", variant32)
    nfp32, nq, dg, de = mixed_vs_fp64(configs.water_spdf_positron())
    assert nfp32 > 0 if variant32 else 0 <= nfp32 < nq
    assert dg < 1e-9 and abs(de) < 1e-6, (nfp32, nq, dg, de)


def test_mixed_organic_molecule():
    """A seeded 8-atom organic molecule of the random-walk family, with the
    s/p/d/f electron basis: many small bounds, so many FP32 quartets."""
    b = configs.organic_basis(8, seed=3)
    nfp32, nq, dg, de = mixed_vs_fp64(b)
    assert nfp32 > 0
    assert dg < 1e-9 and abs(de) < 1e-6, (nfp32, nq, dg, de)


@pytest.mark.parametrize("variant32", ["smem", "lane", "warp"])
def test_mixed_each_fp32_kernel(variant32, monkeypatch):
    """Each FP32 kernel (shared-memory, lane, warp), forced for every class."""
    monkeypatch.setenv("PATGPU_VARIANT32", variant32)
    b = configs.organic_basis(6, seed=4)
    nfp32, nq, dg, de = mixed_vs_fp64(b)
    assert nfp32 > 0.01 * nq
    assert dg < 1e-9 and abs(de) < 1e-6, (variant32, nfp32, nq, dg, de)
