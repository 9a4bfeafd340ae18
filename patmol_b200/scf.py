"""Closed-shell SCF over the GPU integral library, and its nuclear gradient.

The iteration is the one of rhf_scf_update (rhfscf.c:22-71): G[P] from the
GPU Fock build, F = H + G, X^T F X diagonalised on the host (the reference
keeps this step on the host too, spack_math.c:300-384), C = X W,
P = C_occ C_occ^T (scfaux.c:24-41) and E = 2 tr(P H) + tr(P G) + E_nuc
(rhfscf.c:49, scfaux.c:100-118).  The reference damps rising energies by
averaging or its Anderson step (scfaux.c:64-95); here DIIS on the
commutator F P S - S P F drives the energy to 1e-12 Eh, which finite
differences of energies need.  With ``dpm`` the distributed positron model
enters H as in rhf_dpm_calculation (rhfscf.c:232-240): H -= V_DPM.

The gradient (no reference counterpart) is patgpu_rhf_gradient at the
converged P and W = C_occ diag(e_occ) C_occ^T.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .basis import Basis, pack, unpack
from .gpu import GpuBasis


def nuclear_repulsion(basis: Basis) -> float:
    """Sum of q_i q_j / r_ij over centre pairs with a non-zero charge
    product (basis.c:174-195 sums every pair; a q=0 ghost may sit on the
    positron, where the reference's 0/0 gives NaN)."""
    e = 0.0
    q, r = basis.charges, basis.coords
    for i in range(basis.ncen):
        for j in range(i):
            if q[i] * q[j] != 0.0:
                e += q[i] * q[j] / float(np.linalg.norm(r[i] - r[j]))
    return e


@dataclass
class RHFResult:
    energy: float
    P: np.ndarray          # packed half density
    W: np.ndarray          # packed energy-weighted density
    C: np.ndarray          # MO coefficients (n x n)
    eps: np.ndarray        # orbital energies
    iterations: int
    converged: bool
    enuc: float


def orthogonalizer(S: np.ndarray, smin: float = 1e-10) -> np.ndarray:
    """Canonical orthogonalisation X = U s^-1/2 over overlap eigenvalues above smin."""
    s, U = np.linalg.eigh(S)
    keep = s > smin
    return U[:, keep] / np.sqrt(s[keep])


def rhf(basis: Basis, dpm: bool = False, gpu: GpuBasis | None = None, conv: float = 1e-12,
        maxit: int = 100, schwarz_tau: float = 1e-14, ndiis: int = 8) -> RHFResult:
    if basis.nelec % 2 or basis.mult != 1:
        raise ValueError("closed-shell SCF needs an even electron count and multiplicity 1")
    gb = gpu if gpu is not None else GpuBasis(basis, schwarz_tau=schwarz_tau)
    gb.two_electron_ints()
    Sp, _, Hp = gb.one_electron_ints()
    if dpm:
        Hp = gb.dpm_ints(Hp)
    n = basis.norb
    nocc = basis.nelec // 2
    S, H = unpack(Sp, n), unpack(Hp, n)
    X = orthogonalizer(S)
    enuc = nuclear_repulsion(basis)

    def diag(F):
        e, V = np.linalg.eigh(X.T @ F @ X)
        return e, X @ V

    eps, C = diag(H)
    P = C[:, :nocc] @ C[:, :nocc].T
    fs, es = [], []
    e_old = None
    converged = False
    it = 0
    for it in range(1, maxit + 1):
        G = unpack(gb.rhf_form_gmatrix(pack(P)), n)
        F = H + G
        energy = 2.0 * np.sum(P * H) + np.sum(P * G) + enuc
        err = F @ P @ S - S @ P @ F
        fs.append(F)
        es.append(X.T @ err @ X)
        fs, es = fs[-ndiis:], es[-ndiis:]
        if len(fs) > 1:
            m = len(fs)
            B = -np.ones((m + 1, m + 1))
            B[m, m] = 0.0
            for i in range(m):
                for j in range(m):
                    B[i, j] = np.sum(es[i] * es[j])
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            try:
                c = np.linalg.solve(B, rhs)[:m]
                F = sum(ci * Fi for ci, Fi in zip(c, fs))
            except np.linalg.LinAlgError:
                pass
        eps, C = diag(F)
        P_new = C[:, :nocc] @ C[:, :nocc].T
        dP = float(np.max(np.abs(P_new - P)))
        P = P_new
        if e_old is not None and abs(energy - e_old) < conv and float(np.max(np.abs(es[-1]))) < 1e-9 \
                and dP < 1e-8:
            converged = True
            break
        e_old = energy
    # energy and orbitals of the final density
    G = unpack(gb.rhf_form_gmatrix(pack(P)), n)
    F = H + G
    energy = 2.0 * np.sum(P * H) + np.sum(P * G) + enuc
    eps, C = diag(F)
    P = C[:, :nocc] @ C[:, :nocc].T
    W = (C[:, :nocc] * eps[:nocc]) @ C[:, :nocc].T
    if gpu is None:
        gb.close()
    return RHFResult(energy=float(energy), P=pack(P), W=pack(W), C=C, eps=eps, iterations=it,
                     converged=converged, enuc=enuc)


def rhf_gradient(basis: Basis, res: RHFResult, dpm: bool = False, gpu: GpuBasis | None = None,
                 parts: int = GpuBasis.GRAD_ALL, schwarz_tau: float = 1e-14) -> np.ndarray:
    """dE/dR (ncen x 3, Eh/bohr) of the converged closed-shell energy."""
    gb = gpu if gpu is not None else GpuBasis(basis, schwarz_tau=schwarz_tau)
    g = gb.rhf_gradient(res.P, res.W, parts=parts, with_dpm=dpm)
    if gpu is None:
        gb.close()
    return g
