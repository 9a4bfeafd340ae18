"""Moment integrals on the GPU (patgpu_moments and the drop-in momints)
against the reference's MOMINTS.DAT records (momints.c:88-188, written by
the compiled reference; tests/golden/make_pins.py moments): dipole and
quadrupole integrals about the origin within 1e-12, for a contracted s/p/d/f
basis and water s/p/d, and the drop-in program's own MOMINTS.DAT record for
record."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden
from patmol_b200 import configs
from patmol_b200.basis import packed_index

from golden.make_golden import mini_basis  # noqa: E402
from golden.make_pins import MOM_DTYPE  # noqa: E402

pytestmark = pytest.mark.gpu

gpu = pytest.importorskip("patmol_b200.gpu")

DROPIN = os.path.join(ROOT, "oracle", "_ref", "patmol_dropin")


@pytest.mark.parametrize("name", ["mini", "water_spd"])
def test_moments_vs_reference_records(name):
    b = mini_basis() if name == "mini" else configs.water_spd()
    g = golden("moments.npz")
    i, j, dip_ref, quad_ref = g[f"{name}_i"], g[f"{name}_j"], g[f"{name}_dip"], g[f"{name}_quad"]
    assert len(i) == b.norb * (b.norb + 1) // 2
    dip, quad = gpu.moments(b)
    ij = np.array([packed_index(int(a), int(c)) for a, c in zip(i, j)])
    assert np.abs(dip[:, ij].T - dip_ref).max() < 1e-12
    assert np.abs(quad[:, ij].T - quad_ref).max() < 1e-12


def test_dropin_writes_reference_momints(tmp_path):
    """rhf_init calls momints (rhfscf.c:156); in the drop-in program that is
    the GPU's, and its MOMINTS.DAT matches the reference's record stream."""
    if not os.path.exists(DROPIN):
        pytest.skip("oracle/_ref/patmol_dropin was not built (needs the reference tree)")
    configs.water_spd().write_patin(str(tmp_path / "patin.dat"))
    r = subprocess.run([DROPIN], cwd=tmp_path, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-3000:]
    rec = np.fromfile(tmp_path / "MOMINTS.DAT", dtype=MOM_DTYPE)
    g = golden("moments.npz")
    assert np.array_equal(rec["i"], g["water_spd_i"]) and np.array_equal(rec["j"], g["water_spd_j"])
    assert np.abs(rec["dip"] - g["water_spd_dip"]).max() < 1e-12
    assert np.abs(rec["quad"] - g["water_spd_quad"]).max() < 1e-12
