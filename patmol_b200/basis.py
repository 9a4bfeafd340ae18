"""Basis model of the Patmol input: centres, shells and the Cartesian conventions.

Mirrors the reference's input layer so that the GPU library sees exactly the
data the reference's global accessors hand to its integral engines:

* ``patin.dat`` layout (basis.c:251-284, shell.c:8-20, center.c:4-8):
  line 1 ``nshell norb ncen``; line 2 ``maxit eps``; line 3 ``nelec mult``;
  line 4 ``dpm dft dft_x dft_c``; line 5 ``ffc scf_accel scf_guess``;
  line 6 three print flags; then ``ncen`` lines ``q x y z``; then per shell
  ``npr l cen`` followed by ``npr`` lines ``alpha coef``.
* Contraction coefficients are rescaled in place at read time
  (normalize_shell, shell.c:26-56), so ``Shell.coef`` holds the normalised
  values, as the reference's ``shells()`` accessor does.
* Cartesian component order per l: lx descending, then ly descending
  (basis.c:294-308); component factor 1/sqrt((2lx-1)!!(2ly-1)!!(2lz-1)!!)
  (basis.c:309-319).
* With ``dpm`` on the reference appends a +1 positron centre after the input
  centres (basis.c:283) and seven single-primitive DPM shells with no
  Cartesian components (basis.c:220-241; ``nst`` is never set there), so they
  contribute nothing to any integral.  ``Basis.dpm_augmented()`` reproduces
  that state.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

DFACT = (1.0, 1.0, 3.0, 15.0, 105.0, 945.0, 10395.0)


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def cart_components(l: int) -> List[tuple]:
    """(lx, ly, lz) in the reference's order (basis.c:294-308)."""
    out = []
    for lx in range(l, -1, -1):
        for ly in range(l - lx, -1, -1):
            out.append((lx, ly, l - lx - ly))
    return out


def component_factors(l: int) -> np.ndarray:
    return np.array([1.0 / math.sqrt(DFACT[a] * DFACT[b] * DFACT[c])
                     for (a, b, c) in cart_components(l)])


def normalize_coefficients(l: int, alpha: Sequence[float], coef: Sequence[float]) -> np.ndarray:
    """normalize_shell (shell.c:26-56): unit self-overlap of the contracted
    x^l-type function, then the primitive factor sqrt((2a)^(l+3/2)/pi^(3/2))."""
    twofact = 2.0 * math.sqrt(2.0)
    piterm = math.pi * math.sqrt(math.pi)
    lpow = 1.5 + l
    s = 0.0
    for a1, c1 in zip(alpha, coef):
        for a2, c2 in zip(alpha, coef):
            s += c1 * c2 * (math.sqrt(a1 * a2) / (a1 + a2)) ** lpow
    s = 1.0 / math.sqrt(s * twofact)
    return np.array([c * s * math.sqrt((2.0 * a) ** lpow / piterm) for a, c in zip(alpha, coef)])


@dataclass
class Shell:
    l: int
    cen: int
    alpha: np.ndarray
    coef: np.ndarray          # normalised (as after shell.c:21)
    off: int = 0
    nst: int = -1             # Cartesian components; 0 for the DPM shells

    def __post_init__(self):
        if self.nst < 0:
            self.nst = ncart(self.l)

    @property
    def npr(self) -> int:
        return len(self.alpha)


@dataclass
class Basis:
    charges: np.ndarray                      # (ncen,)
    coords: np.ndarray                       # (ncen, 3) bohr
    shells: List[Shell]
    nelec: int = 0
    mult: int = 1
    maxit: int = 200
    eps: float = 1e-10
    dpm: int = 0
    accel: int = 2
    guess: int = 0
    ffc: int = 0
    raw: List[tuple] = field(default_factory=list)   # (npr, l, cen, alphas, raw coefs)
    skipcen: int = -1

    def __post_init__(self):
        self.charges = np.asarray(self.charges, dtype=np.float64)
        self.coords = np.asarray(self.coords, dtype=np.float64).reshape(-1, 3)
        if self.skipcen < 0:
            self.skipcen = len(self.charges)
        off = 0
        for sh in self.shells:
            sh.off = off
            off += sh.nst

    @property
    def nshell(self) -> int:
        return len(self.shells)

    @property
    def norb(self) -> int:
        return sum(s.nst for s in self.shells)

    @property
    def ncen(self) -> int:
        return len(self.charges)

    @property
    def maxl(self) -> int:
        return max(s.l for s in self.shells)

    # ------------------------------------------------------------------
    @classmethod
    def from_shell_list(cls, charges, coords, shell_specs, **kw) -> "Basis":
        """shell_specs: iterable of (l, cen, alphas, raw coefs)."""
        shells, raw = [], []
        for (l, cen, al, co) in shell_specs:
            al = np.asarray(al, dtype=np.float64)
            co = np.asarray(co, dtype=np.float64)
            shells.append(Shell(l=int(l), cen=int(cen), alpha=al,
                                coef=normalize_coefficients(int(l), al, co)))
            raw.append((len(al), int(l), int(cen), al, co))
        return cls(charges=charges, coords=coords, shells=shells, raw=raw, **kw)

    @classmethod
    def read_patin(cls, path) -> "Basis":
        """Parse patin.dat as init_Basis does (basis.c:251-284)."""
        toks = open(path).read().split()
        it = iter(toks)
        nshell, norb, ncen = int(next(it)), int(next(it)), int(next(it))
        maxit, eps = int(next(it)), float(next(it))
        nelec, mult = int(next(it)), int(next(it))
        dpm, _dft, _dx, _dc = int(next(it)), int(next(it)), int(next(it)), int(next(it))
        ffc, accel, guess = int(next(it)), int(next(it)), int(next(it))
        for _ in range(3):
            next(it)
        q, xyz = [], []
        for _ in range(ncen):
            q.append(float(next(it)))
            xyz.append([float(next(it)) for _ in range(3)])
        specs = []
        for _ in range(nshell):
            npr, l, cen = int(next(it)), int(next(it)), int(next(it))
            al, co = [], []
            for _ in range(npr):
                al.append(float(next(it)))
                co.append(float(next(it)))
            specs.append((l, cen, al, co))
        b = cls.from_shell_list(q, xyz, specs, nelec=nelec, mult=mult, maxit=maxit,
                                eps=eps, dpm=dpm, accel=accel, guess=guess, ffc=ffc)
        if b.norb != norb:
            raise ValueError(f"patin.dat declares {norb} functions, shells give {b.norb}")
        return b

    def write_patin(self, path) -> None:
        lines = [f"{self.nshell} {self.norb} {self.ncen}",
                 f"{self.maxit} {self.eps:.10e}",
                 f"{self.nelec} {self.mult}",
                 f"{self.dpm} 0 0 0",
                 f"{self.ffc} {self.accel} {self.guess}",
                 "0 0 0"]
        for q, r in zip(self.charges, self.coords):
            lines.append(f"{q:.17g} {r[0]:.17g} {r[1]:.17g} {r[2]:.17g}")
        for (npr, l, cen, al, co) in self.raw:
            lines.append(f"{npr} {l} {cen}")
            for a, c in zip(al, co):
                lines.append(f"{a:.17g} {c:.17g}")
        with open(path, "w") as f:
            f.write("\n".join(lines) + "\n")

    def dpm_augmented(self, positron_xyz) -> "Basis":
        """State after dpm_augment + set_center_position (basis.c:220-241,
        323-329; rhfscf.c:232-235): a +1 centre at the positron and seven
        component-less DPM shells on it.  Function count is unchanged."""
        alf = (13.3615, 2.0133, 0.453757, 1.2331, 2.5719, 0.59976, 0.139365)
        lsh = (0, 0, 0, 0, 1, 1, 1)
        charges = np.concatenate([self.charges, [1.0]])
        coords = np.vstack([self.coords, np.asarray(positron_xyz, dtype=np.float64).reshape(1, 3)])
        pc = self.ncen
        shells = [Shell(l=s.l, cen=s.cen, alpha=s.alpha, coef=s.coef, nst=s.nst) for s in self.shells]
        for a, l in zip(alf, lsh):
            shells.append(Shell(l=l, cen=pc, alpha=np.array([a]), coef=np.array([1.0]), nst=0))
        out = Basis(charges=charges, coords=coords, shells=shells, raw=list(self.raw),
                    nelec=self.nelec, mult=self.mult, maxit=self.maxit, eps=self.eps,
                    dpm=self.dpm, accel=self.accel, guess=self.guess, ffc=self.ffc,
                    skipcen=self.ncen)
        return out

    def with_coords(self, coords) -> "Basis":
        """The same basis with every centre at new coordinates (ncen x 3);
        shells move with their centres (set_center_position, basis.c:163-166)."""
        shells = [Shell(l=s.l, cen=s.cen, alpha=s.alpha, coef=s.coef, nst=s.nst) for s in self.shells]
        return Basis(charges=self.charges.copy(), coords=np.array(coords, dtype=np.float64).reshape(-1, 3),
                     shells=shells, raw=list(self.raw), nelec=self.nelec, mult=self.mult, maxit=self.maxit,
                     eps=self.eps, dpm=self.dpm, accel=self.accel, guess=self.guess, ffc=self.ffc,
                     skipcen=self.skipcen)

    def displaced(self, center: int, dim: int, delta: float) -> "Basis":
        xyz = self.coords.copy()
        xyz[center, dim] += delta
        return self.with_coords(xyz)

    def is_uhf(self) -> bool:
        """patmol.c:18: RHF iff the electron count is even and mult == 1."""
        return not (self.nelec % 2 == 0 and self.mult == 1)

    def flat_arrays(self):
        """Plain arrays for the C ABI (patgpu_basis_create)."""
        nprim = np.array([s.npr for s in self.shells], dtype=np.int32)
        prim_off = np.zeros(self.nshell + 1, dtype=np.int32)
        prim_off[1:] = np.cumsum(nprim)
        return dict(
            l=np.array([s.l for s in self.shells], dtype=np.int32),
            cen=np.array([s.cen for s in self.shells], dtype=np.int32),
            off=np.array([s.off for s in self.shells], dtype=np.int32),
            nst=np.array([s.nst for s in self.shells], dtype=np.int32),
            prim_off=prim_off,
            alpha=np.concatenate([s.alpha for s in self.shells]).astype(np.float64),
            coef=np.concatenate([s.coef for s in self.shells]).astype(np.float64),
            charges=np.ascontiguousarray(self.charges, dtype=np.float64),
            coords=np.ascontiguousarray(self.coords, dtype=np.float64).reshape(-1),
        )


def packed_index(i: int, j: int) -> int:
    """Packed lower triangle, row-major (scfaux.c:452-456)."""
    if j > i:
        i, j = j, i
    return i * (i + 1) // 2 + j


def unpack(packed: np.ndarray, n: int) -> np.ndarray:
    m = np.zeros((n, n))
    il = np.tril_indices(n)
    # row-major lower triangle order matches np.tril_indices order
    m[il] = packed
    m = m + m.T - np.diag(np.diag(m))
    return m


def pack(full: np.ndarray) -> np.ndarray:
    n = full.shape[0]
    return full[np.tril_indices(n)].copy()
