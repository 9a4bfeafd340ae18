"""Every kernel variant, forced for every class where it exists
(PATGPU_VARIANT=lane|reg|smem|smem_occ|warp), gives the oracle's G within 1e-11
on a 65-function water basis whose shells cover all 55 quartet classes up to
(ff|ff); the autotuner's own choice is checked the same way.  The FP32
kernels of the mixed-precision window (PATGPU_VARIANT32=smem|lane|warp), run
over every quartet (window bound 1e30), stay within 1e-6 of it."""

import numpy as np
import pytest

import patref

from golden.make_golden import seeded_density  # noqa: E402
from test_gpu_gradient import small_water  # noqa: E402

pytestmark = pytest.mark.gpu

gpu = pytest.importorskip("patmol_b200.gpu")


@pytest.fixture(scope="module")
def water_ref():
    b = small_water(f_on_o=True)
    P = seeded_density(b.norb, 21)
    return b, P, patref.Oracle(b).gmat(P)


@pytest.mark.parametrize("variant", ["lane", "reg", "smem", "smem_occ", "warp", None])
def test_variant_matches_oracle(water_ref, variant, monkeypatch):
    b, P, ref = water_ref
    if variant is None:
        monkeypatch.delenv("PATGPU_VARIANT", raising=False)
    else:
        monkeypatch.setenv("PATGPU_VARIANT", variant)
    g = gpu.GpuBasis(b)
    assert len(g.class_counts()) == 55
    G = g.rhf_form_gmatrix(P)
    assert np.abs(G - ref).max() < 1e-11
    g.close()


def test_implicit_enumeration_without_lists(water_ref, monkeypatch):
    """PATGPU_LISTS=0: the kernels screen the implicit quartet space on the
    fly; same G, and mixed precision stays off (FP32 runs over lists only)."""
    b, P, ref = water_ref
    monkeypatch.setenv("PATGPU_LISTS", "0")
    g = gpu.GpuBasis(b)
    assert np.abs(g.rhf_form_gmatrix(P) - ref).max() < 1e-11
    assert g.set_mixed_precision(1e-8) == 0
    assert np.abs(g.rhf_form_gmatrix(P) - ref).max() < 1e-11
    g.close()


@pytest.mark.parametrize("variant32", ["smem", "lane", "warp"])
def test_fp32_variant_close_to_oracle(water_ref, variant32, monkeypatch):
    b, P, ref = water_ref
    monkeypatch.setenv("PATGPU_VARIANT32", variant32)
    g = gpu.GpuBasis(b)
    nfp32 = g.set_mixed_precision(1e30)
    assert nfp32 == g.stats()["quartets"]
    G = g.rhf_form_gmatrix(P)
    assert np.abs(G - ref).max() < 1e-6 * max(1.0, float(np.abs(ref).max()))
    g.close()


def test_warp_kernel_jk_and_uhf_fallback(water_ref, monkeypatch):
    """J and K separately through the warp kernel (one density set), and the
    open-shell build, which the warp kernel leaves to the lane kernel."""
    b, P, _ = water_ref
    monkeypatch.setenv("PATGPU_VARIANT", "warp")
    g = gpu.GpuBasis(b)
    O = patref.Oracle(b)
    J, K = g.jk(P)
    G = g.rhf_form_gmatrix(P)
    assert np.abs((2.0 * J - K) - G).max() < 1e-11
    PB = seeded_density(b.norb, 22)
    GA, GB = g.uhf_form_gmatrix(P, PB)
    RA, RB = O.gmat(P, PB)
    assert np.abs(GA - RA).max() < 1e-11 and np.abs(GB - RB).max() < 1e-11
    g.close()
