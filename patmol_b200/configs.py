"""Seeded synthetic molecules and even-tempered bases for the workloads.

All bases are uncontracted even-tempered Cartesian Gaussians with raw
coefficient 1.0 (normalised by the basis reader as shell.c:26-56 does).

* ``water_spd``      water, O(0,0,0), H(0,+-1.4305,1.1071) bohr; on every
                     centre s 0.08*2.5^k (k=0..7), p 0.1*2.5^k (k=0..5),
                     d 0.3*2.5^k (k=0..2).  51 shells, 132 functions, RHF.
* ``water_spdf_positron``  the same plus f 0.5*2.5^k (k=0,1) on every atom and
                     a q=0 ghost centre at the geometric centroid carrying
                     s/p/d shells 0.002*2.2^k (k=0..9); dpm on with the
                     positron at the centroid.  87 shells, 292 functions.
* ``random_organic`` seeded self-avoiding walk of C/N/O/H (p .35/.10/.10/.45),
                     bonds 2.6-2.9 bohr, non-bonded >= 4.0 bohr.
* ``alkane``         zig-zag CnH2n+2, C-C 2.91, C-H 2.06 bohr, tetrahedral
                     angles, seeded N(0, 0.05) bohr jitter.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from .basis import Basis

Z = {"H": 1.0, "C": 6.0, "N": 7.0, "O": 8.0}

WATER_XYZ = np.array([[0.0, 0.0, 0.0], [0.0, 1.4305, 1.1071], [0.0, -1.4305, 1.1071]])
WATER_Q = np.array([8.0, 1.0, 1.0])


def even_tempered(base: float, ratio: float, count: int) -> List[float]:
    return [base * ratio ** k for k in range(count)]


def spd_shells(cen: int, f: bool = False):
    sh = []
    for a in even_tempered(0.08, 2.5, 8):
        sh.append((0, cen, [a], [1.0]))
    for a in even_tempered(0.1, 2.5, 6):
        sh.append((1, cen, [a], [1.0]))
    for a in even_tempered(0.3, 2.5, 3):
        sh.append((2, cen, [a], [1.0]))
    if f:
        for a in even_tempered(0.5, 2.5, 2):
            sh.append((3, cen, [a], [1.0]))
    return sh


def ghost_shells(cen: int):
    sh = []
    for l in (0, 1, 2):
        for a in even_tempered(0.002, 2.2, 10):
            sh.append((l, cen, [a], [1.0]))
    return sh


def water_spd(**kw) -> Basis:
    specs = []
    for c in range(3):
        specs += spd_shells(c)
    return Basis.from_shell_list(WATER_Q, WATER_XYZ, specs, nelec=10, mult=1,
                                 maxit=kw.get("maxit", 200), eps=kw.get("eps", 1e-10), accel=2)


def water_centroid() -> np.ndarray:
    return WATER_XYZ.mean(axis=0)


def water_spdf_positron(mult: int = 1, nelec: int = 10, **kw) -> Basis:
    """mult=2, nelec=9 gives the open-shell (UHF) variant of the same basis."""
    g = water_centroid()
    q = np.concatenate([WATER_Q, [0.0]])
    xyz = np.vstack([WATER_XYZ, g[None, :]])
    specs = []
    for c in range(3):
        specs += spd_shells(c, f=True)
    specs += ghost_shells(3)
    return Basis.from_shell_list(q, xyz, specs, nelec=nelec, mult=mult,
                                 maxit=kw.get("maxit", 200), eps=kw.get("eps", 1e-10),
                                 accel=2, dpm=kw.get("dpm", 1))


def molecule_basis(symbols, xyz, with_f: bool, **kw) -> Basis:
    q = np.array([Z[s] for s in symbols])
    specs = []
    for c in range(len(symbols)):
        specs += spd_shells(c, f=with_f)
    nelec = int(round(q.sum())) + kw.pop("charge_shift", 0)
    mult = 1 if nelec % 2 == 0 else 2
    return Basis.from_shell_list(q, np.asarray(xyz), specs, nelec=nelec, mult=mult,
                                 maxit=kw.get("maxit", 200), eps=kw.get("eps", 1e-10), accel=2,
                                 dpm=kw.get("dpm", 0))


def random_organic(natom: int, seed: int) -> Tuple[List[str], np.ndarray]:
    """Self-avoiding random walk (bond 2.6-2.9 bohr, non-bonded >= 4.0 bohr)."""
    rng = np.random.default_rng(seed)
    elems = rng.choice(["C", "N", "O", "H"], size=natom, p=[0.35, 0.10, 0.10, 0.45])
    pos = [np.zeros(3)]
    tries = 0
    while len(pos) < natom:
        tries += 1
        if tries > 200000:
            raise RuntimeError("random walk stuck")
        anchor = pos[rng.integers(max(0, len(pos) - 3), len(pos))]
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        cand = anchor + v * rng.uniform(2.6, 2.9)
        d = np.linalg.norm(np.asarray(pos) - cand, axis=1)
        bonded = np.isclose(d, np.linalg.norm(cand - anchor))
        if np.all(d[~bonded] >= 4.0) and d.min() >= 2.6 - 1e-9:
            pos.append(cand)
    return list(elems), np.asarray(pos)


def organic_basis(natom: int, seed: int, with_f: bool = True, **kw) -> Basis:
    sym, xyz = random_organic(natom, seed)
    q = sum(Z[s] for s in sym)
    shift = 0 if int(q) % 2 == 0 else 1      # keep closed shell: add one electron
    return molecule_basis(sym, xyz, with_f, charge_shift=shift, **kw)


def alkane(ncarbon: int = 12, seed: int = 0) -> Tuple[List[str], np.ndarray]:
    rng = np.random.default_rng(seed)
    cc, ch = 2.91, 2.06
    half = math.radians(109.4712) / 2.0
    sym, xyz = [], []
    for i in range(ncarbon):
        x = i * cc * math.sin(half)
        y = (0.5 - (i % 2)) * cc * math.cos(half)
        sym.append("C")
        xyz.append([x, y, 0.0])
    carbons = np.array(xyz)
    for i in range(ncarbon):
        c = carbons[i]
        outward = np.array([0.0, 1.0 if i % 2 == 0 else -1.0, 0.0])
        for s in (+1, -1):
            d = outward * math.cos(half) + np.array([0.0, 0.0, s * math.sin(half)])
            sym.append("H")
            xyz.append(c + ch * d / np.linalg.norm(d))
        if i in (0, ncarbon - 1):
            d = np.array([-1.0 if i == 0 else 1.0, 0.0, 0.0])
            sym.append("H")
            xyz.append(c + ch * d)
    xyz = np.asarray(xyz) + rng.normal(scale=0.05, size=(len(xyz), 3))
    return sym, xyz
