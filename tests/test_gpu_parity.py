"""Parity of the GPU library (through its C ABI) with the oracle and with the
reference's golden outputs.  Tolerances:
  * ERIs: 1e-12 absolute against the quad-precision restatement; against the
    reference's own records, 1e-12 outside the two windows where the
    reference's Rys roots are inexact (see test_oracle.rys_defect).
  * G, J, K at a fixed density: 1e-11 absolute against the restatement.
  * one-body S, T, H and the DPM potential: 1e-12 against the reference.
"""
import itertools

import numpy as np
import pytest

from conftest import golden
from patmol_b200 import configs
from patmol_b200.basis import unpack
import patref

from golden.make_golden import mini_basis, he_dpm_basis, seeded_density  # noqa: E402
from test_oracle import f2s_map, quartet_T, rys_defect  # noqa: E402

pytestmark = pytest.mark.gpu

gpu = pytest.importorskip("patmol_b200.gpu")


@pytest.fixture(scope="module")
def mini():
    b = mini_basis()
    return b, gpu.GpuBasis(b), patref.Oracle(b)


def test_eri_blocks_vs_oracle(mini):
    b, G, O = mini
    quartets = list(itertools.product(range(b.nshell), repeat=4))
    blocks = G.eri_quartets(quartets)
    worst = 0.0
    for q, blk in zip(quartets, blocks):
        worst = max(worst, float(np.abs(blk - O.eri_block(*q)).max()))
    assert worst < 1e-12, worst


def test_eri_records_vs_reference(mini):
    b, G, _ = mini
    g = golden("mini_ints.npz")
    f2s = f2s_map(b)
    keys = sorted({(f2s[i][0], f2s[j][0], f2s[k][0], f2s[l][0]) for i, j, k, l in zip(g["i"], g["j"], g["k"], g["l"])})
    blocks = dict(zip(keys, G.eri_quartets(keys)))
    worst, checked = 0.0, 0
    for i, j, k, l, v in zip(g["i"], g["j"], g["k"], g["l"], g["val"]):
        (a, ia), (bb, ib), (c, ic), (d, id_) = f2s[i], f2s[j], f2s[k], f2s[l]
        key = (a, bb, c, d)
        n = sum(b.shells[s].l for s in key) // 2 + 1
        if any(rys_defect(n, t) for t in quartet_T(b, *key)):
            continue
        worst = max(worst, abs(blocks[key][ia, ib, ic, id_] - v))
        checked += 1
    assert checked > 20000
    assert worst < 1e-12, worst


def test_water_counts_match_survey():
    b = configs.water_spd()
    G = gpu.GpuBasis(b)
    s = G.stats()
    assert s["n"] == 132 and s["pairs"] == 1326 and s["unscreened"] == 879801


def test_water_rhf_gmatrix_vs_oracle():
    b = configs.water_spd()
    P = seeded_density(b.norb, 11)
    G = gpu.GpuBasis(b).rhf_form_gmatrix(P)
    Go = patref.Oracle(b).gmat(P)
    assert np.abs(G - Go).max() < 1e-11, np.abs(G - Go).max()


def test_water_rhf_gmatrix_vs_reference():
    """Against the reference's own G: equal up to its root2 defect."""
    b = configs.water_spd()
    P = seeded_density(b.norb, 11)
    G = gpu.GpuBasis(b).rhf_form_gmatrix(P)
    assert np.abs(G - golden("water_spd.npz")["G"]).max() < 1e-4


def test_water_uhf_gmatrix_vs_oracle():
    b = configs.water_spd()
    PA, PB = seeded_density(b.norb, 11), seeded_density(b.norb, 12)
    GA, GB = gpu.GpuBasis(b).uhf_form_gmatrix(PA, PB)
    OA, OB = patref.Oracle(b).gmat(PA, PB)
    assert np.abs(GA - OA).max() < 1e-11
    assert np.abs(GB - OB).max() < 1e-11


def test_gmatrix_accumulates():
    b = configs.water_spd()
    P = seeded_density(b.norb, 3)
    Gb = gpu.GpuBasis(b)
    G1 = Gb.rhf_form_gmatrix(P)
    G2 = Gb.rhf_form_gmatrix(P, G1.copy())
    assert np.allclose(G2, 2 * G1, rtol=0, atol=1e-12)


def test_jk_consistent_with_g():
    b = configs.water_spd()
    P = seeded_density(b.norb, 5)
    Gb = gpu.GpuBasis(b)
    J, K = Gb.jk(P)
    G = Gb.rhf_form_gmatrix(P)
    assert np.abs(2 * J - K - G).max() < 1e-11


def test_water_oneints_vs_reference():
    b = configs.water_spd()
    g = golden("water_spd.npz")
    S, T, H = gpu.GpuBasis(b).one_electron_ints()
    assert np.abs(S - g["S"]).max() < 1e-13
    assert np.abs(T - g["T"]).max() < 1e-11
    assert np.abs(H - g["H"]).max() < 1e-11


def test_dpm_vs_reference():
    b = he_dpm_basis().dpm_augmented([0.0, 0.0, 3.0])
    g = golden("he_dpm.npz")
    S, T, H, Hd = gpu.onebody(b, True, None)
    assert np.abs(H - g["H0"]).max() < 1e-12
    _, _, _, Hd = gpu.onebody(b, False, H)
    assert np.abs(Hd - g["Hdpm"]).max() < 1e-12


def test_water_spdf_dpm_vs_reference():
    b = configs.water_spdf_positron().dpm_augmented(configs.water_centroid())
    g = golden("water_spdf_dpm.npz")
    _, _, H0, _ = gpu.onebody(b, True, None)
    assert np.abs(H0 - g["H0"]).max() < 1e-10
    _, _, _, Hd = gpu.onebody(b, False, H0)
    assert np.abs((H0 - Hd) - g["Vdpm"]).max() < 1e-12


def test_spdf_sampled_quartets_vs_oracle():
    """Water s/p/d/f + ghost positron shells: 400 seeded shell quartets of
    every class (f shells give 6-7 Rys roots) against the restatement."""
    b = configs.water_spdf_positron()
    rng = np.random.default_rng(7)
    qs = rng.integers(0, b.nshell, size=(400, 4))
    fsh = [i for i, s in enumerate(b.shells) if s.l == 3]
    qs[:40] = rng.choice(fsh, size=(40, 4))
    G = gpu.GpuBasis(b)
    O = patref.Oracle(b)
    worst = 0.0
    for q, blk in zip(qs, G.eri_quartets(qs)):
        worst = max(worst, float(np.abs(blk - O.eri_block(*q)).max()))
    assert worst < 1e-12, worst


def test_spdf_counts_match_survey():
    b = configs.water_spdf_positron()
    s = gpu.GpuBasis(b).stats()
    assert s["n"] == 292 and s["pairs"] == 3828 and s["unscreened"] == 7328706


def test_start_shell_restricts_quartets():
    """Quartets with largest shell index >= start (twoints.c:228) give the
    G of the reference's `start` argument."""
    b = configs.water_spd()
    P = seeded_density(b.norb, 2)
    Gb = gpu.GpuBasis(b)
    Gb.two_electron_ints(start=40)
    G = Gb.rhf_form_gmatrix(P)
    Go = patref.Oracle(b).gmat(P, start=40)
    assert np.abs(G - Go).max() < 1e-11


def test_partition_sums_to_whole():
    b = configs.water_spd()
    P = seeded_density(b.norb, 4)
    Gb = gpu.GpuBasis(b)
    full = Gb.rhf_form_gmatrix(P)
    parts = np.zeros_like(full)
    for r in range(3):
        Gb.two_electron_ints(0, r, 3)
        parts += Gb.rhf_form_gmatrix(P)
    assert np.abs(parts - full).max() < 1e-11


def test_energy_symmetry_property_spdf():
    """Size-independent check on the config with f shells and the ghost
    centre: E2(P1,P2) = tr(P1 G(P2)) is symmetric in P1, P2 for RHF G."""
    b = configs.water_spdf_positron()
    n = b.norb
    Gb = gpu.GpuBasis(b)
    P1, P2 = seeded_density(n, 21) * 0.1, seeded_density(n, 22) * 0.1
    G1, G2 = Gb.rhf_form_gmatrix(P1), Gb.rhf_form_gmatrix(P2)
    e12 = np.sum(unpack(P1, n) * unpack(G2, n))
    e21 = np.sum(unpack(P2, n) * unpack(G1, n))
    assert abs(e12 - e21) < 1e-9 * max(1.0, abs(e12))
    # linearity
    G12 = Gb.rhf_form_gmatrix(P1 + P2)
    assert np.abs(G12 - G1 - G2).max() < 1e-10


def test_no_gpu_fallback_message():
    assert gpu.LIB_PATH.endswith("libpatgpu.so")
