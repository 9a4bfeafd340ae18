"""The drop-in binding: the reference's own host program (SCF drivers, basis
module, linear algebra) linked against libpatgpu.so in place of twoints.c,
dpmints.c, oneints.c, rys.c and scfaux.c's two G builds (oracle/Makefile,
target `dropin`).  Converged energies against the reference's."""
import os
import re
import shutil
import subprocess

import pytest

from conftest import GOLDEN, ROOT
from patmol_b200 import configs

pytestmark = pytest.mark.gpu

DROPIN = os.path.join(ROOT, "oracle", "_ref", "patmol_dropin")


def run_dropin(tmp_path, basis=None, patin=None, env=None):
    if not os.path.exists(DROPIN):
        pytest.skip("oracle/_ref/patmol_dropin was not built (needs the reference tree)")
    if patin:
        shutil.copy(patin, tmp_path / "patin.dat")
    else:
        basis.write_patin(str(tmp_path / "patin.dat"))
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([DROPIN], cwd=tmp_path, capture_output=True, text=True, timeout=1200, env=e)
    assert r.returncode == 0, r.stderr[-3000:]
    vals = [float(x) for x in open(tmp_path / "short.gs.dat").read().split()]
    return vals, r.stderr


def test_dropin_water_energy(tmp_path, golden_meta):
    vals, err = run_dropin(tmp_path, configs.water_spd(), env={"PATGPU_VERBOSE": "1"})
    # the reference's own clean-up at exit (rhfscf.c:15-19) reaches the
    # library's clean_ERIFS, which frees the handle's device state
    assert "patgpu: clean_ERIFS released the handle's device state, 0 bound" in err, err[-2000:]
    g = golden_meta["water_spd"]
    # exact-integral energy (reference energy corrected for its root2 defect)
    assert abs(vals[1] - g["e_total_exact_integrals"]) < 5e-9
    # the reference's own energy, whose Rys roots are off by up to 3.5e-4 for 15 < T <= 31
    assert abs(vals[1] - g["scf"]["e_total"]) < 1e-6


def test_dropin_sf6_fixture(tmp_path, golden_meta):
    """The reference's shipped example (SF6, contracted s/p/d, 214 functions)."""
    vals, _ = run_dropin(tmp_path, patin=os.path.join(GOLDEN, "sf6_patin.dat"))
    g = golden_meta["sf6"]
    assert abs(vals[1] - g["e_total"]) < 1e-5, (vals[1], g["e_total"])


def test_dropin_writes_reference_eri_files(tmp_path, golden_meta):
    """PATGPU_ERI_FILES=1: two_electron_ints also writes the reference's ERI
    files through the host program's createERIFile and reports them in the
    ERIFS handle; the reference's own clean-up (clean_ERIFS, erifs.c:68-81)
    then finds and removes every one of them, and the SCF is unchanged.  The
    files' contents are checked in test_gpu_erifiles.py."""
    vals, err = run_dropin(tmp_path, configs.water_spd(), env={"PATGPU_ERI_FILES": "1"})
    assert abs(vals[1] - golden_meta["water_spd"]["e_total_exact_integrals"]) < 5e-9
    m = re.search(r"patgpu: wrote (\d+) ERI file\(s\), (\d+) records", err)
    assert m and int(m.group(1)) >= 1 and int(m.group(2)) > 1.7e7, err[-500:]
    # <rank><file number>MINTS.DAT (erifs.c:54-73); MOMINTS.DAT is the
    # reference's moment-integral file, not an ERI file
    left = [p for p in os.listdir(tmp_path) if re.fullmatch(r"\d+MINTS\.DAT", p)]
    assert not left, left
