"""Generate the golden fixtures of tests/golden from the compiled reference.

Run in the build container (it needs the reference tree to build
oracle/_ref):
    PATMOL_REFERENCE=<reference tree> python tests/golden/make_golden.py
Every number stored here comes from the reference's own code
(oracle/_ref/ref_harness, oracle/_ref/ref_rysdump) run on seeded inputs, or
from the reference's shipped SF6 fixture (patin.dat, short.gs.dat).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from patmol_b200 import configs  # noqa: E402
from patmol_b200.basis import Basis  # noqa: E402
import patref  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("PATMOL_REFERENCE", "")


def mini_basis() -> Basis:
    """Two centres, every l up to f on centre 0 with contracted s and p."""
    specs = [(0, 0, [30.0, 5.0, 1.2], [0.2, 0.5, 0.4]), (1, 0, [2.5, 0.6], [0.6, 0.5]),
             (2, 0, [0.9], [1.0]), (3, 0, [0.7], [1.0]), (0, 1, [1.1], [1.0]), (1, 1, [0.45], [1.0])]
    return Basis.from_shell_list([2.0, 1.0], [[0, 0, 0], [0.3, -0.4, 1.1]], specs, nelec=4, mult=1)


def he_dpm_basis() -> Basis:
    specs = [(0, 0, [a], [1.0]) for a in (0.5, 2.0, 8.0)] + [(1, 0, [0.8], [1.0])]
    return Basis.from_shell_list([2.0], [[0.0, 0.0, 0.0]], specs, nelec=2, mult=1, dpm=1,
                                 maxit=200, eps=1e-10, accel=2)


def h2_sto3g() -> Basis:
    al = [3.42525091, 0.62391373, 0.16885540]
    co = [0.15432897, 0.53532814, 0.44463454]
    specs = [(0, 0, al, co), (0, 1, al, co)]
    return Basis.from_shell_list([1.0, 1.0], [[0, 0, 0], [0, 0, 1.4]], specs, nelec=2, mult=1,
                                 maxit=200, eps=1e-10, accel=2)


def seeded_density(n: int, seed: int) -> np.ndarray:
    """Symmetric packed matrix, values N(0, 0.1^2)."""
    rng = np.random.default_rng(seed)
    return rng.normal(scale=0.1, size=n * (n + 1) // 2)


def main():
    if not REFERENCE:
        raise SystemExit("set PATMOL_REFERENCE to the reference source tree")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REFERENCE}"], check=True)
    meta = {}

    # 1. mini basis: every ERI record, S, T, H, E_nuc
    b = mini_basis()
    _, o = patref.run_ref(b, ["ints"], outputs=["eri.bin", "S.bin", "T.bin", "H.bin", "info.txt"])
    eri = o["eri.bin"]
    np.savez_compressed(os.path.join(OUT, "mini_ints.npz"),
                        i=eri["i"], j=eri["j"], k=eri["k"], l=eri["l"], val=eri["val"],
                        S=o["S.bin"], T=o["T.bin"], H=o["H.bin"])
    meta["mini"] = {"enuc": float(o["info.txt"].split()[3]), "records": int(len(eri))}

    # 2. water s/p/d (51 shells, 132 functions): G(P) for seeded P, UHF G, S/T/H, SCF
    b = configs.water_spd()
    n = b.norb
    P = seeded_density(n, 11)
    PB = seeded_density(n, 12)
    _, g = patref.run_ref(b, ["gmat", "P.bin"], inputs={"P.bin": P}, outputs=["G.bin"])
    _, u = patref.run_ref(b, ["ugmat", "PA.bin", "PB.bin"], inputs={"PA.bin": P, "PB.bin": PB},
                          outputs=["GA.bin", "GB.bin"])
    _, s = patref.run_ref(b, ["ints"], outputs=["S.bin", "T.bin", "H.bin", "info.txt"])
    out, c = patref.run_ref(b, ["scf"], outputs=["Pconv.bin"])
    scf = json.loads(out.strip().splitlines()[-1])
    np.savez_compressed(os.path.join(OUT, "water_spd.npz"), G=g["G.bin"], GA=u["GA.bin"], GB=u["GB.bin"],
                        S=s["S.bin"], T=s["T.bin"], H=s["H.bin"], Pconv=c["Pconv.bin"])
    # first-order energy of exact integrals at the reference's converged
    # density: E + tr(P dG), dG = G_exact(P) - G_reference(P); the SCF energy
    # is stationary in P, so this is the exact-integral energy to second order
    Pc = c["Pconv.bin"]
    _, gc = patref.run_ref(b, ["gmat", "P.bin"], inputs={"P.bin": Pc}, outputs=["G.bin"])
    dG = patref.Oracle(b).gmat(Pc) - gc["G.bin"]
    from patmol_b200.basis import unpack
    de = float(np.sum(unpack(Pc, n) * unpack(dG, n)))
    meta["water_spd"] = {"P_seed": 11, "PB_seed": 12, "scf": scf, "nrec": int(s["info.txt"].split()[4]),
                         "e_total_exact_integrals": scf["e_total"] + de, "de_root_defect": de}

    # 3. He + DPM regression (positron at (0,0,3) bohr)
    b = he_dpm_basis()
    _, d = patref.run_ref(b, ["dpm", "0", "0", "3"], outputs=["H0.bin", "Hdpm.bin"])
    out, _ = patref.run_ref(b, ["scf"], posgrid=[(0.0, 0.0, 3.0)])
    np.savez_compressed(os.path.join(OUT, "he_dpm.npz"), H0=d["H0.bin"], Hdpm=d["Hdpm.bin"])
    meta["he_dpm"] = {"pos": [0.0, 0.0, 3.0], "scf": json.loads(out.strip().splitlines()[-1])}

    # 4. water s/p/d/f + ghost positron shells: DPM one-body at the centroid
    b = configs.water_spdf_positron()
    g0 = configs.water_centroid()
    _, d = patref.run_ref(b, ["dpm"] + ["%.17g" % x for x in g0], outputs=["H0.bin", "Hdpm.bin"])
    np.savez_compressed(os.path.join(OUT, "water_spdf_dpm.npz"), H0=d["H0.bin"], Vdpm=d["H0.bin"] - d["Hdpm.bin"])
    meta["water_spdf_dpm"] = {"pos": [float(x) for x in g0]}

    # 5. H2 / STO-3G at R = 1.4 bohr
    out, _ = patref.run_ref(h2_sto3g(), ["scf"])
    meta["h2_sto3g"] = {"scf": json.loads(out.strip().splitlines()[-1])}

    # 6. the reference's shipped SF6 fixture: input and its published energy
    src = os.path.join(REFERENCE, "patin.dat")
    with open(src) as f, open(os.path.join(OUT, "sf6_patin.dat"), "w") as g6:
        g6.write(f.read())
    with open(os.path.join(REFERENCE, "short.gs.dat")) as f:
        vals = [float(x) for x in f.read().split()]
    meta["sf6"] = {"enuc": vals[0], "e_total": vals[1], "ediff": vals[2], "iters": 43,
                   "source": "short.gs.dat:1-3, scfout.gs.dat:1-2"}

    # 7. the reference's Rys roots on a T grid (documents its fit accuracy)
    Ts = np.concatenate([np.linspace(0.0, 60.0, 601), [1e-7, 3e-7, 15.5, 20.0, 25.0, 31.0]])
    rr = {}
    for nr in range(1, 8):
        res = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_rysdump"), str(nr)],
                             input="\n".join("%.17g" % t for t in Ts), capture_output=True, text=True,
                             check=True).stdout.split("\n")
        rr[f"n{nr}"] = np.array([[float(v) for v in line.split()] for line in res[:len(Ts)]]).reshape(len(Ts), nr, 2)
    np.savez_compressed(os.path.join(OUT, "ref_rys.npz"), T=Ts, **rr)

    with open(os.path.join(OUT, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
