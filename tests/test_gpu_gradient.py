"""Nuclear gradient (patgpu_rhf_gradient) against finite differences.

The reference has no gradient, so parity is with derivatives of energies:
  * each part at a FIXED density (two-electron tr(P G[P]), one-electron
    2 tr(P H) - 2 tr(W S) with and without the DPM potential, nuclear
    repulsion) against Richardson-extrapolated central differences of the
    ORACLE's energies (steps 1e-3 and 5e-4 bohr; truncation error O(h^4)),
    tolerance 1e-8 relative to the gradient's largest entry plus 1e-9;
  * the converged SCF energy's full gradient against central differences
    with step 1e-4 bohr of SCF energies from the GPU driver, tolerance
    2e-6 Eh/bohr (SCF energies converged to 1e-12 Eh);
  * rotational and translational invariance of the converged gradient of
    water s/p/d (132 functions): sum_i g_i = 0 and sum_i R_i x g_i = 0.
"""
import numpy as np
import pytest

from patmol_b200 import configs
from patmol_b200.basis import Basis
import patref

from golden.make_golden import mini_basis, seeded_density  # noqa: E402

pytestmark = pytest.mark.gpu

gpu = pytest.importorskip("patmol_b200.gpu")
scf = pytest.importorskip("patmol_b200.scf")


def small_water(f_on_o: bool = True, nelec: int = 10) -> Basis:
    """Water with a few even-tempered shells per centre (f on O optional)."""
    specs = []
    for c in range(3):
        heavy = c == 0
        for a in configs.even_tempered(0.15, 3.0, 4 if heavy else 3):
            specs.append((0, c, [a], [1.0]))
        for a in configs.even_tempered(0.2, 3.0, 3 if heavy else 2):
            specs.append((1, c, [a], [1.0]))
        for a in configs.even_tempered(0.5, 3.0, 2 if heavy else 1):
            specs.append((2, c, [a], [1.0]))
        if heavy and f_on_o:
            specs.append((3, c, [0.8], [1.0]))
    return Basis.from_shell_list(configs.WATER_Q, configs.WATER_XYZ, specs, nelec=nelec, mult=1)


def packed_weights(n):
    w = np.full(n * (n + 1) // 2, 2.0)
    w[[i * (i + 1) // 2 + i for i in range(n)]] = 1.0
    return w


def richardson(f, basis, h=1e-3):
    """(4 D(h/2) - D(h)) / 3 of the central differences, every centre and axis."""
    g = np.zeros((basis.ncen, 3))
    for c in range(basis.ncen):
        for d in range(3):
            D = []
            for s in (h, h / 2):
                D.append((f(basis.displaced(c, d, s)) - f(basis.displaced(c, d, -s))) / (2 * s))
            g[c, d] = (4 * D[1] - D[0]) / 3
    return g


def close(g, ref, rel=1e-8, abs_=1e-9):
    err = float(np.abs(g - ref).max())
    assert err < rel * float(np.abs(ref).max()) + abs_, (err, g, ref)


@pytest.mark.parametrize("make", [mini_basis, small_water], ids=["mini", "water_spdf"])
def test_two_electron_part_vs_oracle(make):
    b = make()
    P = seeded_density(b.norb, 11)
    wts = packed_weights(b.norb)
    g = gpu.GpuBasis(b).rhf_gradient(P, parts=gpu.GpuBasis.GRAD_2E)

    def e2(bx):
        return float(np.sum(wts * P * patref.Oracle(bx).gmat(P)))

    close(g, richardson(e2, b))


@pytest.mark.parametrize("with_dpm", [False, True])
def test_one_electron_part_vs_oracle(with_dpm):
    b = small_water(f_on_o=True).dpm_augmented([0.3, -0.2, 2.4])
    P = seeded_density(b.norb, 12)
    W = seeded_density(b.norb, 13)
    wts = packed_weights(b.norb)
    g = gpu.GpuBasis(b).rhf_gradient(P, W, parts=gpu.GpuBasis.GRAD_1E, with_dpm=with_dpm)

    def e1(bx):
        O = patref.Oracle(bx)
        S, _, H = O.oneints()
        if with_dpm:
            H = O.dpm(H)
        return float(2.0 * np.sum(wts * P * H) - 2.0 * np.sum(wts * W * S))

    close(g, richardson(e1, b))
    if with_dpm:
        assert np.abs(g[b.skipcen]).max() > 1e-4   # the positron centre feels the DPM term


def test_nuclear_part_vs_oracle():
    b = small_water().dpm_augmented([0.3, -0.2, 2.4])
    P = seeded_density(b.norb, 14)
    g = gpu.GpuBasis(b).rhf_gradient(P, parts=gpu.GpuBasis.GRAD_NUC)
    close(g, richardson(lambda bx: patref.Oracle(bx).enuc(), b))


def scf_energy(bx, dpm):
    r = scf.rhf(bx, dpm=dpm)
    assert r.converged
    return r.energy


@pytest.mark.parametrize("dpm", [False, True], ids=["ground", "dpm"])
def test_scf_gradient_vs_energy_differences(dpm):
    b = small_water(f_on_o=False)
    if dpm:
        b = b.dpm_augmented([0.2, 0.4, 3.0])
    res = scf.rhf(b, dpm=dpm)
    assert res.converged
    g = scf.rhf_gradient(b, res, dpm=dpm)
    h = 1e-4
    coords = [(0, 2), (1, 1), (1, 2), (2, 0)] + ([(b.skipcen, 1), (b.skipcen, 2)] if dpm else [])
    for c, d in coords:
        fd = (scf_energy(b.displaced(c, d, h), dpm) - scf_energy(b.displaced(c, d, -h), dpm)) / (2 * h)
        assert abs(g[c, d] - fd) < 2e-6, (c, d, g[c, d], fd)


def alkane_dpm(ncarbon: int) -> Basis:
    """The alkane + DPM recipe at small size: s/p/d shells on every atom, a q=0
    ghost at the centroid with s/p/d shells, DPM on with the positron at the
    centroid.  The atom and ghost exponents are moderate (0.2*3^k) so that the
    overlap stays well conditioned and the SCF energy converges to 1e-12 Eh;
    the full-size recipe's 0.002*2.2^k ghost shells make S nearly singular."""
    sym, xyz = configs.alkane(ncarbon, 0)
    cen = xyz.mean(axis=0)
    specs = []
    for c in range(len(sym)):
        heavy = sym[c] != "H"
        for a in configs.even_tempered(0.2, 3.0, 4 if heavy else 3):
            specs.append((0, c, [a], [1.0]))
        for a in configs.even_tempered(0.3, 3.0, 2 if heavy else 1):
            specs.append((1, c, [a], [1.0]))
        if heavy:
            specs.append((2, c, [0.8], [1.0]))
    for l in (0, 1, 2):
        for a in configs.even_tempered(0.2, 3.0, 2):
            specs.append((l, len(sym), [a], [1.0]))
    mol = configs.molecule_basis(sym, xyz, with_f=False)
    q = np.concatenate([mol.charges, [0.0]])
    return Basis.from_shell_list(q, np.vstack([xyz, cen[None, :]]), specs, nelec=mol.nelec, mult=1,
                                 dpm=1).dpm_augmented(cen)


def test_alkane_dpm_gradient_vs_energy_differences():
    b = alkane_dpm(2)
    res = scf.rhf(b, dpm=True)
    assert res.converged
    g = scf.rhf_gradient(b, res, dpm=True)
    h = 1e-4
    for c, d in [(0, 0), (2, 2), (b.skipcen, 0)]:
        fd = (scf_energy(b.displaced(c, d, h), True) - scf_energy(b.displaced(c, d, -h), True)) / (2 * h)
        assert abs(g[c, d] - fd) < 2e-6, (c, d, g[c, d], fd)


def test_scf_gradient_invariances():
    b = configs.water_spd()
    res = scf.rhf(b)
    assert res.converged
    g = scf.rhf_gradient(b, res)
    assert np.abs(g.sum(axis=0)).max() < 1e-9
    torque = np.cross(b.coords, g).sum(axis=0)
    assert np.abs(torque).max() < 1e-7, torque
    assert np.abs(g).max() > 1e-3


def test_uhf_two_electron_part_vs_oracle():
    """Open shell: E2 = sum_s tr(P_s G_s)/2 with G_s = J[Pa+Pb] - K[P_s]."""
    b = small_water(f_on_o=True, nelec=9)
    PA = seeded_density(b.norb, 31)
    PB = seeded_density(b.norb, 32)
    wts = packed_weights(b.norb)
    g = gpu.GpuBasis(b).uhf_gradient(PA, PB, parts=gpu.GpuBasis.GRAD_2E)

    def e2(bx):
        GA, GB = patref.Oracle(bx).gmat(PA, PB)
        return float(0.5 * np.sum(wts * (PA * GA + PB * GB)))

    close(g, richardson(e2, b))


@pytest.mark.parametrize("dpm", [False, True], ids=["doublet", "doublet_dpm"])
def test_uhf_scf_gradient_vs_energy_differences(dpm):
    """The water cation doublet (9 electrons), with and without DPM."""
    b = small_water(f_on_o=False, nelec=9)
    b.mult = 2
    if dpm:
        b = b.dpm_augmented([0.2, 0.4, 3.0])
    res = scf.uhf(b, dpm=dpm)
    assert res.converged
    g = scf.uhf_gradient(b, res, dpm=dpm)
    h = 1e-4

    def energy(bx):
        r = scf.uhf(bx, dpm=dpm)
        assert r.converged
        return r.energy

    coords = [(0, 2), (1, 1), (2, 2)] + ([(b.skipcen, 2)] if dpm else [])
    for c, d in coords:
        fd = (energy(b.displaced(c, d, h)) - energy(b.displaced(c, d, -h))) / (2 * h)
        assert abs(g[c, d] - fd) < 2e-6, (c, d, g[c, d], fd)
