"""Generate the parity-pin fixtures of tests/golden from the compiled reference
and the CPU restatement (the oracle).

Run in the build container, where the reference tree exists (it is needed to
build oracle/_ref):

    PATMOL_REFERENCE=<reference tree> python tests/golden/make_pins.py <part> ...

Parts (each writes its own files and merges its entry into pins.json):

  c1       The 292-function water s/p/d/f + ghost-positron workload that the
           bench times.  At a seeded density and at the core-Hamiltonian
           guess density: the oracle's full G (every packed element, the
           elementwise pin of the GPU build), the reference's own
           rhf_form_gmatrix E[P] = tr(P G[P]) (scfaux.c:429-552 over its own
           ERI files) and the root-defect term tr(P (G_oracle - G_reference)).
  sf6      The reference's shipped SF6 example: the reference's own SCF
           energy on this machine, its converged density (PMATRIX.OUT,
           rhfscf.c:419-423) and the first-order energy of exact integrals
           at that density (the reference's Rys roots are inexact for
           15 < T <= 31.2 with two roots and for six and seven roots).
  mols     SCF energies of small molecules of the batched-SCF family
           (config-0 basis): the reference's (its integrals, G build and
           diagonaliser, driven to convergence by the harness's DIIS: the
           reference's own damping stalls on them), the first-order
           root-defect term at its converged density, and the restatement's
           converged energy (exact quadrature) started from that density.
  gradfd   Central differences (h = 1e-4 bohr) of the reference's own SCF
           energies for the gradient pins: closed-shell water and water with
           the DPM potential (positron displaced too).
  moments  The reference's MOMINTS.DAT records (momints.c:88-188) for the
           contracted s/p/d/f mini basis and water s/p/d.
  org      The oracle's converged SCF energy of an 8-atom molecule of the
           40-atom family (s/p/d/f on every atom): DIIS SCF on the CPU
           restatement's G builds (slow: hours on 8 cores).

The reference's own energies are used as they come; where its inexact roots
matter, the fixture also stores the exact-integral correction so that the
GPU's exact quadrature can be held to the tight bar.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from patmol_b200 import configs  # noqa: E402
from patmol_b200.basis import Basis, pack, unpack  # noqa: E402
import patref  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
PINS = os.path.join(OUT, "pins.json")


def reference_tree() -> str:
    ref = os.environ.get("PATMOL_REFERENCE")
    if not ref or not os.path.isdir(ref):
        raise SystemExit("set PATMOL_REFERENCE to the reference source tree")
    return ref


def packed_weights(n: int) -> np.ndarray:
    w = np.full(n * (n + 1) // 2, 2.0)
    w[[i * (i + 1) // 2 + i for i in range(n)]] = 1.0
    return w


def trace_pg(P, G, n) -> float:
    """tr(P G) of two packed symmetric matrices."""
    return float(np.sum(packed_weights(n) * P * G))


def seeded_density(n: int, seed: int, scale: float = 0.1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.normal(scale=scale, size=n * (n + 1) // 2)


def core_guess_density(basis: Basis, S, H) -> np.ndarray:
    """P = C_occ C_occ^T of the core Hamiltonian (rhfscf.c:455-471), canonical
    orthogonalisation over overlap eigenvalues above 1e-10."""
    n = basis.norb
    s, U = np.linalg.eigh(unpack(S, n))
    keep = s > 1e-10
    X = U[:, keep] / np.sqrt(s[keep])
    _, V = np.linalg.eigh(X.T @ unpack(H, n) @ X)
    C = X @ V[:, :basis.nelec // 2]
    return pack(C @ C.T)


def merge(key, value):
    d = {}
    if os.path.exists(PINS):
        with open(PINS) as f:
            d = json.load(f)
    d[key] = value
    with open(PINS, "w") as f:
        json.dump(d, f, indent=1)


def ref_gmat(basis, P):
    _, g = patref.run_ref(basis, ["gmat", "P.bin"], inputs={"P.bin": P}, outputs=["G.bin"], timeout=7200)
    return g["G.bin"]


def defect(basis, P):
    """tr(P G_oracle[P]), tr(P G_reference[P]) and G_oracle[P]."""
    n = basis.norb
    go = patref.Oracle(basis).gmat(P)
    gr = ref_gmat(basis, P)
    return trace_pg(P, go, n), trace_pg(P, gr, n), go


# ------------------------------------------------------------------ parts
def part_c1():
    b = configs.water_spdf_positron()
    n = b.norb
    S, _, H = patref.Oracle(b).oneints()
    dens = {"seeded": seeded_density(n, 21, 0.05), "core_guess": core_guess_density(b, S, H)}
    arrays, meta = {}, {"basis": "water s/p/d/f + ghost positron s/p/d (87 shells, 292 functions)",
                        "seeded_density": {"seed": 21, "scale": 0.05}}
    for name, P in dens.items():
        t = time.time()
        eo, er, go = defect(b, P)
        arrays[f"G_{name}"] = go
        if name != "seeded":
            arrays[f"P_{name}"] = P
        meta[name] = {"E_oracle": eo, "E_reference": er, "de_root_defect": eo - er,
                      "max_abs_G": float(np.abs(go).max())}
        print(name, meta[name], f"{time.time() - t:.0f}s", flush=True)
    np.savez_compressed(os.path.join(OUT, "water_spdf_g.npz"), **arrays)
    merge("c1", meta)


def run_patmol(patin_text: str, extra=None):
    """The reference's own serial program on a patin.dat; returns the work dir."""
    d = tempfile.mkdtemp(prefix="patmol_")
    with open(os.path.join(d, "patin.dat"), "w") as f:
        f.write(patin_text)
    for name, data in (extra or {}).items():
        with open(os.path.join(d, name), "w") as f:
            f.write(data)
    r = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "patmol")], cwd=d, capture_output=True, text=True,
                       timeout=7200)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    return d


def part_sf6():
    src = open(os.path.join(OUT, "sf6_patin.dat")).read().splitlines()
    # line 6 holds the three print flags (basis.c:256); the third writes the
    # converged density to PMATRIX.OUT (rhfscf.c:419-423)
    src[5] = "  0   0   1"
    d = run_patmol("\n".join(src) + "\n")
    vals = [float(x) for x in open(os.path.join(d, "short.gs.dat")).read().split()]
    b = Basis.read_patin(os.path.join(OUT, "sf6_patin.dat"))
    n = b.norb
    P = np.fromfile(os.path.join(d, "PMATRIX.OUT"), dtype=np.float64)
    assert P.size == n * (n + 1) // 2
    shutil.rmtree(d)
    eo, er, _ = defect(b, P)
    meta = {"e_total_reference_here": vals[1], "enrg0": vals[0], "ediff": vals[2],
            "E2_oracle_at_Pconv": eo, "E2_reference_at_Pconv": er,
            "de_root_defect": eo - er, "e_total_exact_integrals": vals[1] + (eo - er)}
    np.savez_compressed(os.path.join(OUT, "sf6_pconv.npz"), P=P)
    print(meta, flush=True)
    merge("sf6", meta)


MOLS = [(3, 11), (4, 12), (5, 13), (6, 14), (7, 15)]


def oracle_scf(basis, P0, conv=1e-11, maxit=60):
    """DIIS SCF on the restatement's G builds (exact Rys quadrature), started
    from the density P0 (packed)."""
    from patmol_b200.scf import _RHFState
    O = patref.Oracle(basis)
    S, _, H = O.oneints()
    st = _RHFState(basis, S, H, ndiis=8, conv=conv)
    st.P = unpack(np.asarray(P0, dtype=np.float64), basis.norb)
    while st.it < maxit and not st.converged:
        st.step(O.gmat(st.packed_density()))
    res = st.finish(O.gmat(st.packed_density()))
    return res


def part_mols():
    # the reference's damping (scfaux.c:64-95) stalls on these molecules; the
    # harness's DIIS driver keeps every reference computation but the damping
    os.environ["REF_HARNESS_DIIS"] = "1"
    out = []
    for natom, seed in MOLS:
        b = configs.organic_basis(natom, seed, with_f=False)
        t = time.time()
        o, c = patref.run_ref(b, ["scf"], outputs=["Pconv.bin"], timeout=7200)
        scf = json.loads(o.strip().splitlines()[-1])
        P = c["Pconv.bin"]
        eo, er, _ = defect(b, P)
        ores = oracle_scf(b, P)
        rec = {"natom": natom, "seed": seed, "n": b.norb, "scf": scf,
               "de_root_defect_first_order": eo - er,
               "oracle_scf": {"e_total": ores.energy, "iterations": ores.iterations,
                              "converged": bool(ores.converged)}}
        out.append(rec)
        print(rec, f"{time.time() - t:.0f}s", flush=True)
    merge("mols", out)


def gradfd_bases():
    """The closed-shell water basis of the gradient tests (no f), and the
    same with DPM on and the positron at (0.2, 0.4, 3.0) bohr."""
    specs = []
    for c in range(3):
        heavy = c == 0
        for a in configs.even_tempered(0.15, 3.0, 4 if heavy else 3):
            specs.append((0, c, [a], [1.0]))
        for a in configs.even_tempered(0.2, 3.0, 3 if heavy else 2):
            specs.append((1, c, [a], [1.0]))
        for a in configs.even_tempered(0.5, 3.0, 2 if heavy else 1):
            specs.append((2, c, [a], [1.0]))
    b = Basis.from_shell_list(configs.WATER_Q, configs.WATER_XYZ, specs, nelec=10, mult=1, maxit=400,
                              eps=1e-12, accel=2)
    return b


GRAD_COORDS = [(0, 2), (1, 1), (1, 2), (2, 0)]
GRAD_POS = (0.2, 0.4, 3.0)
GRAD_H = 1e-4


def ref_energy(b, pos=None):
    """The compiled reference's SCF energy (with pos: the DPM total energy at
    that positron position)."""
    if pos is None:
        out, _ = patref.run_ref(b, ["scf"])
        return json.loads(out.strip().splitlines()[-1])["e_total"]
    out, _ = patref.run_ref(b, ["scf"], posgrid=[pos])
    return json.loads(out.strip().splitlines()[-1])["dpm"][0]["e_total"]


def part_gradfd():
    b0 = gradfd_bases()
    recs = {"h": GRAD_H, "pos": list(GRAD_POS), "ground": [], "dpm": []}
    for c, d in GRAD_COORDS:
        ep = ref_energy(b0.displaced(c, d, GRAD_H))
        em = ref_energy(b0.displaced(c, d, -GRAD_H))
        recs["ground"].append({"center": c, "dim": d, "fd": (ep - em) / (2 * GRAD_H)})
        print("ground", recs["ground"][-1], flush=True)
    b1 = gradfd_bases()
    b1.dpm = 1
    for c, d in GRAD_COORDS:
        ep = ref_energy(b1.displaced(c, d, GRAD_H), GRAD_POS)
        em = ref_energy(b1.displaced(c, d, -GRAD_H), GRAD_POS)
        recs["dpm"].append({"center": c, "dim": d, "fd": (ep - em) / (2 * GRAD_H)})
        print("dpm", recs["dpm"][-1], flush=True)
    for d in (1, 2):   # the positron position
        pp = list(GRAD_POS)
        pm = list(GRAD_POS)
        pp[d] += GRAD_H
        pm[d] -= GRAD_H
        fd = (ref_energy(b1, tuple(pp)) - ref_energy(b1, tuple(pm))) / (2 * GRAD_H)
        recs["dpm"].append({"center": "positron", "dim": d, "fd": fd})
        print("dpm", recs["dpm"][-1], flush=True)
    merge("gradfd", recs)


MOM_DTYPE = np.dtype([("i", "<i4"), ("j", "<i4"), ("dip", "<f8", 3), ("quad", "<f8", 6)])


def ref_moments(basis):
    """The reference's MOMINTS.DAT records (momints.c:88-188) for a basis."""
    with tempfile.TemporaryDirectory(prefix="patref_mom_") as d:
        basis.write_patin(os.path.join(d, "patin.dat"))
        subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_harness"), "moments"], cwd=d, check=True,
                       capture_output=True)
        return np.fromfile(os.path.join(d, "MOMINTS.DAT"), dtype=MOM_DTYPE)


def part_moments():
    from golden.make_golden import mini_basis
    arrays = {}
    for name, b in (("mini", mini_basis()), ("water_spd", configs.water_spd())):
        r = ref_moments(b)
        arrays.update({f"{name}_i": r["i"], f"{name}_j": r["j"], f"{name}_dip": r["dip"], f"{name}_quad": r["quad"]})
        print(name, len(r), flush=True)
    np.savez_compressed(os.path.join(OUT, "moments.npz"), **arrays)


def part_org():
    from patmol_b200.scf import _RHFState
    natom, seed = int(os.environ.get("PINS_ORG_NATOM", "8")), int(os.environ.get("PINS_ORG_SEED", "3"))
    b = configs.organic_basis(natom, seed, with_f=True)
    O = patref.Oracle(b)
    S, _, H = O.oneints()
    st = _RHFState(b, S, H, ndiis=8, conv=1e-10)
    t = time.time()
    while st.it < 60 and not st.converged:
        st.step(O.gmat(st.packed_density()))
        print(f"it {st.it} E {st.e_old:.12f} {time.time() - t:.0f}s", flush=True)
    G = O.gmat(st.packed_density())
    res = st.finish(G)
    rec = {"natom": natom, "seed": seed, "n": b.norb, "e_total": res.energy, "iterations": res.iterations,
           "converged": bool(res.converged)}
    print(rec, flush=True)
    np.savez_compressed(os.path.join(OUT, f"org{natom}_pconv.npz"), P=res.P)
    merge("org", rec)


def main(argv):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", "restatement",
                    f"REF={reference_tree()}"], check=True)
    parts = {"c1": part_c1, "sf6": part_sf6, "mols": part_mols, "gradfd": part_gradfd, "org": part_org,
             "moments": part_moments}
    for p in argv or list(parts):
        parts[p]()


if __name__ == "__main__":
    main(sys.argv[1:])
