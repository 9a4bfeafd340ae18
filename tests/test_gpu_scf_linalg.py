"""SCF linear algebra on the GPU (patgpu_scf_*: X^T F X, cuSOLVER syevd,
C = X V, P and W) against numpy on the host:
  * at a water s/p/d Fock matrix, orbital energies within 1e-10 Eh and the
    half density P and energy-weighted density W within 1e-10 of their
    largest entry (P reaches ~200 in this nearly dependent diffuse basis, so
    the bound is relative: two backward-stable eigensolvers differ by about
    the condition number times the rounding unit; eigenvector signs are
    free, P and W are not);
  * the SCF with the device step reaches the host SCF's energy within 1e-10 Eh.
"""
import numpy as np
import pytest

from patmol_b200 import configs
from patmol_b200.basis import pack, unpack

pytestmark = pytest.mark.gpu

gpu = pytest.importorskip("patmol_b200.gpu")
scf = pytest.importorskip("patmol_b200.scf")


def test_density_step_matches_numpy():
    b = configs.water_spd()
    g = gpu.GpuBasis(b)
    g.two_electron_ints()
    Sp, _, Hp = g.one_electron_ints()
    n, nocc = b.norb, b.nelec // 2
    X = scf.orthogonalizer(unpack(Sp, n))
    e0, V = np.linalg.eigh(X.T @ unpack(Hp, n) @ X)
    C0 = X @ V
    P0 = C0[:, :nocc] @ C0[:, :nocc].T
    F = unpack(Hp, n) + unpack(g.rhf_form_gmatrix(pack(P0)), n)
    e, V = np.linalg.eigh(X.T @ F @ X)
    C = X @ V
    P = C[:, :nocc] @ C[:, :nocc].T
    W = (C[:, :nocc] * e[:nocc]) @ C[:, :nocc].T
    la = gpu.GpuScfLinalg(X, nocc)
    eg, Cg, Pg, Wg = la.density(pack(F))
    assert np.abs(eg - e).max() < 1e-10
    assert np.abs(unpack(Pg, n) - P).max() < 1e-10 * np.abs(P).max()
    assert np.abs(unpack(Wg, n) - W).max() < 1e-10 * np.abs(W).max()
    assert np.abs(np.abs(Cg[:, :nocc]) - np.abs(C[:, :nocc])).max() < 1e-9 * np.abs(C[:, :nocc]).max()
    la.close()
    g.close()


def test_scf_with_device_step():
    b = configs.water_spd()
    host = scf.rhf(b)
    dev = scf.rhf(b, device_linalg=True)
    assert host.converged and dev.converged
    assert abs(host.energy - dev.energy) < 1e-10, (host.energy, dev.energy)
