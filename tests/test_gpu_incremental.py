"""Density-weighted screening and incremental Fock builds.

  * With tau_dens = 0 the host build is the full build; with tau_dens = 1e-14
    a build over a late-SCF-sized density difference (1e-10) computes fewer
    quartets, and what it drops stays below 1e-12 in every G element.
  * The incremental SCF (G from density differences, full rebuild every 8
    iterations, final energy from a full build) converges to the full SCF's
    energy within 1e-9 Eh on water s/p/d, and its late iterations compute
    fewer quartets than a full build.
"""
import numpy as np
import pytest

from patmol_b200 import configs

pytestmark = pytest.mark.gpu

gpu = pytest.importorskip("patmol_b200.gpu")
scf = pytest.importorskip("patmol_b200.scf")


def test_density_screened_difference_build():
    b = configs.water_spd()
    res = scf.rhf(b)
    g = gpu.GpuBasis(b)
    g.two_electron_ints()
    rng = np.random.default_rng(5)
    dP = 1e-10 * rng.normal(size=res.P.shape)
    full = g.rhf_form_gmatrix(dP)
    n_full = g.last_computed()
    g.set_density_screening(1e-14)
    part = g.rhf_form_gmatrix(dP)
    n_part = g.last_computed()
    g.set_density_screening(0.0)
    # water s/p/d is compact: most quartets have large Schwarz bounds, so the
    # screen drops about a tenth of them here (more in extended molecules)
    assert n_part < 0.95 * n_full, (n_part, n_full)
    assert np.abs(part - full).max() < 1e-12
    assert np.abs(g.rhf_form_gmatrix(dP) - full).max() < 1e-13
    g.close()


def test_incremental_scf_energy():
    b = configs.water_spd()
    ref = scf.rhf(b)
    inc = scf.rhf(b, incremental=True)
    assert ref.converged and inc.converged, (ref.iterations, inc.iterations)
    assert abs(ref.energy - inc.energy) < 1e-9, (ref.energy, inc.energy)
    q = inc.quartets_computed
    assert min(q[1:]) < q[0], q
