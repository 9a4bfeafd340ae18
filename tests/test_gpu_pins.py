"""Parity pins at the tolerances the drop-in promises, on the inputs the bench
times and on the reference's own example, through the C ABI.

Fixtures (tests/golden/pins.json and the .npz files beside it) come from the
compiled reference and the CPU restatement (tests/golden/make_pins.py).  The
reference's Rys roots are inexact in two windows (two roots for
15 < T <= 31.2; six and seven roots), while the GPU evaluates exact
quadrature; each fixture therefore carries the reference's own number and
the root-defect term tr(P (G_exact - G_reference)) at the same density, and
the GPU is held to their sum at the tight bar and to the raw reference
number at the size of that term.

  * 292-function water + ghost-positron workload (the bench's): every packed
    element of G at two densities against the oracle, 1e-11 absolute; E[P] =
    tr(P G[P]) against the reference's own rhf_form_gmatrix plus the defect
    term, 1e-9 Eh.
  * SF6 (the reference's shipped example) through the drop-in program:
    converged energy within 1e-8 Eh of the reference's energy plus the defect
    term at its converged density.
  * He + DPM through the drop-in program: the reference's dpmvpol.dat value
    and ground-state energy, 1e-9 Eh.
  * Converged SCF energies of small molecules of the batched family: FP64
    within 1e-9 Eh and mixed precision within 1e-6 Eh of the oracle's
    converged energy; the reference's own energy plus its first-order defect
    term within 5e-5 Eh.
  * Analytic nuclear gradients of the converged SCF against central
    differences (h = 1e-4 bohr) of the reference's own SCF energies, with and
    without DPM: 1e-6 Eh/bohr.
"""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden
from patmol_b200 import configs
from patmol_b200.basis import Basis

from golden.make_pins import (GRAD_COORDS, GRAD_H, GRAD_POS, MOLS, gradfd_bases,  # noqa: E402
                              seeded_density, trace_pg)

pytestmark = pytest.mark.gpu

gpu = pytest.importorskip("patmol_b200.gpu")
scf = pytest.importorskip("patmol_b200.scf")

DROPIN = os.path.join(ROOT, "oracle", "_ref", "patmol_dropin")


@pytest.fixture(scope="module")
def pins():
    with open(os.path.join(GOLDEN, "pins.json")) as f:
        return json.load(f)


# ------------------------------------------------- the bench's workload, full G
@pytest.fixture(scope="module")
def c1_handle():
    b = configs.water_spdf_positron()
    g = gpu.GpuBasis(b)
    yield b, g
    g.close()


@pytest.mark.parametrize("which", ["seeded", "core_guess"])
def test_c1_full_gmatrix_and_energy(which, c1_handle, pins):
    b, g = c1_handle
    n = b.norb
    fx = golden("water_spdf_g.npz")
    meta = pins["c1"]
    if which == "seeded":
        P = seeded_density(n, meta["seeded_density"]["seed"], meta["seeded_density"]["scale"])
    else:
        P = fx["P_core_guess"]
    G = g.rhf_form_gmatrix(P)
    Go = fx[f"G_{which}"]
    assert G.shape == Go.shape == (n * (n + 1) // 2,)
    err = float(np.abs(G - Go).max())
    assert err < 1e-11, err
    m = meta[which]
    e_gpu = trace_pg(P, G, n)
    # exact-integral energy functional: the reference's own E[P] plus its root-defect term
    assert abs(e_gpu - (m["E_reference"] + m["de_root_defect"])) < 1e-9, (e_gpu, m)
    assert abs(e_gpu - m["E_oracle"]) < 1e-9
    # and the raw reference value differs by the defect term alone
    assert abs((e_gpu - m["E_reference"]) - m["de_root_defect"]) < 1e-9


# ------------------------------------------------------------- drop-in program
def run_dropin(tmp_path, patin_text=None, basis=None, posgrid=None):
    if not os.path.exists(DROPIN):
        pytest.skip("oracle/_ref/patmol_dropin was not built (needs the reference tree)")
    if basis is not None:
        basis.write_patin(str(tmp_path / "patin.dat"))
    else:
        (tmp_path / "patin.dat").write_text(patin_text)
    if posgrid is not None:
        (tmp_path / "posgrid.dat").write_text(f"{len(posgrid)}\n" +
                                              "".join("%.17g %.17g %.17g\n" % tuple(p) for p in posgrid))
    r = subprocess.run([DROPIN], cwd=tmp_path, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-3000:]
    return [float(x) for x in (tmp_path / "short.gs.dat").read_text().split()]


def test_sf6_dropin_energy_exact_integrals(tmp_path, pins):
    vals = run_dropin(tmp_path, patin_text=open(os.path.join(GOLDEN, "sf6_patin.dat")).read())
    s = pins["sf6"]
    assert abs(vals[1] - s["e_total_exact_integrals"]) < 1e-8, (vals[1], s)
    # the reference's own energy (this machine's build agrees with the
    # published short.gs.dat to 3e-11) differs by the defect term alone
    assert abs((vals[1] - s["e_total_reference_here"]) - s["de_root_defect"]) < 1e-8


def test_he_dpm_dropin_vpol(tmp_path, golden_meta):
    from golden.make_golden import he_dpm_basis
    g = golden_meta["he_dpm"]
    vals = run_dropin(tmp_path, basis=he_dpm_basis(), posgrid=[g["pos"]])
    assert abs(vals[1] - g["scf"]["e_total"]) < 1e-9, (vals[1], g["scf"]["e_total"])
    # rhf_dpm_calculation's output line (rhfscf.c:252-258): x y z vpol alfa vstat
    row = (tmp_path / "dpmvpol.dat").read_text().split()
    vpol = float(row[3])
    assert abs(vpol - g["scf"]["dpm"][0]["vpol"]) < 1e-9, (vpol, g["scf"]["dpm"][0]["vpol"])


# ----------------------------------------- converged SCF energies, FP64 and mixed
@pytest.mark.parametrize("natom,seed", MOLS)
def test_scf_energy_vs_reference(natom, seed, pins):
    """FP64 within 1e-9 Eh and mixed precision within 1e-6 Eh of the oracle's
    converged energy (exact quadrature).  The reference's own converged energy
    differs from it by the reference's root defect, up to 2.2e-4 Eh on these
    molecules; the first-order term tr(P dG) at the reference's density
    accounts for most of it and leaves up to 3.5e-5 Eh (second order: the
    defect also moves the converged density)."""
    rec = next(r for r in pins["mols"] if r["natom"] == natom and r["seed"] == seed)
    assert rec["oracle_scf"]["converged"]
    b = configs.organic_basis(natom, seed, with_f=False)
    g = gpu.GpuBasis(b)
    e64 = scf.rhf(b, gpu=g, conv=1e-11, maxit=200)
    emx = scf.rhf(b, gpu=g, tau_fp32=1e-8, conv=1e-11, maxit=200)
    g.close()
    assert e64.converged and emx.converged
    exact = rec["oracle_scf"]["e_total"]
    assert abs(e64.energy - exact) < 1e-9, (e64.energy, exact, rec)
    assert abs(emx.energy - exact) < 1e-6, (emx.energy, exact)
    ref = rec["scf"]["e_total"] + rec["de_root_defect_first_order"]
    assert abs(e64.energy - ref) < 5e-5, (e64.energy, ref)
    assert abs(e64.energy - rec["scf"]["e_total"]) < 5e-4


# --------------------------------------------- gradients vs the reference's FD
def test_gradient_vs_reference_fd(pins):
    fd = pins["gradfd"]
    assert fd["h"] == GRAD_H and tuple(fd["pos"]) == GRAD_POS
    b = gradfd_bases()
    res = scf.rhf(b)
    assert res.converged
    grad = scf.rhf_gradient(b, res)
    for rec, (c, d) in zip(fd["ground"], GRAD_COORDS):
        assert (rec["center"], rec["dim"]) == (c, d)
        assert abs(grad[c, d] - rec["fd"]) < 1e-6, (c, d, grad[c, d], rec["fd"])


def test_dpm_gradient_vs_reference_fd(pins):
    fd = pins["gradfd"]
    b0 = gradfd_bases()
    b0.dpm = 1
    b = b0.dpm_augmented(GRAD_POS)
    res = scf.rhf(b, dpm=True)
    assert res.converged
    grad = scf.rhf_gradient(b, res, dpm=True)
    for rec in fd["dpm"]:
        c = b.skipcen if rec["center"] == "positron" else rec["center"]
        assert abs(grad[c, rec["dim"]] - rec["fd"]) < 1e-6, (rec, grad[c, rec["dim"]])
