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
from .gpu import GpuBasis, GpuBatch, GpuScfLinalg


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
    quartets_computed: list | None = None   # per iteration, incremental builds
    fock_seconds: float = 0.0              # device-timed Fock builds of the iterations


def orthogonalizer(S: np.ndarray, smin: float = 1e-10) -> np.ndarray:
    """Canonical orthogonalisation X = U s^-1/2 over overlap eigenvalues above smin."""
    s, U = np.linalg.eigh(S)
    keep = s > smin
    return U[:, keep] / np.sqrt(s[keep])


class _RHFState:
    """One molecule's closed-shell iteration (host side of rhf_scf_update)."""

    def __init__(self, basis: Basis, Sp, Hp, ndiis: int, conv: float, device_linalg: bool = False,
                 comm_tol: float = 1e-9, dp_tol: float = 1e-8, smin: float = 1e-10, level_shift: float = 0.0,
                 shift_tol: float = 1e-3, ediis: bool = False):
        if basis.nelec % 2 or basis.mult != 1:
            raise ValueError("closed-shell SCF needs an even electron count and multiplicity 1")
        self.n = basis.norb
        self.nocc = basis.nelec // 2
        self.S, self.H = unpack(Sp, self.n), unpack(Hp, self.n)
        self.X = orthogonalizer(self.S, smin)
        self.enuc = nuclear_repulsion(basis)
        self.ndiis, self.conv = ndiis, conv
        self.comm_tol, self.dp_tol = comm_tol, dp_tol
        # virtual-orbital level shift while the DIIS error is above shift_tol
        self.level_shift, self.shift_tol = level_shift, shift_tol
        self.err = np.inf
        # EDIIS (energy-DIIS) while the DIIS error is large: densities and
        # energies of the stored Fock matrices, and M[i, j] = tr(P_i F_j)
        self.ediis = ediis
        self.ps, self.ens = [], []
        self.M = np.zeros((0, 0))
        # the step of rhf_scf_update after F (X^T F X, diagonalise, C, P) on the
        # GPU (patgpu_scf_*) or on the host
        self.linalg = GpuScfLinalg(self.X, self.nocc) if device_linalg else None
        self.eps, C, self.P = self.diag_density(self.H)
        self.fs, self.es = [], []
        self.eov = np.zeros((0, 0))
        self.e_old = None
        self.converged = False
        self.it = 0

    def diag(self, F):
        e, V = np.linalg.eigh(self.X.T @ F @ self.X)
        return e, self.X @ V

    def diag_density(self, F):
        """Orbital energies, orbitals and the half density of the Fock matrix F."""
        if self.linalg is not None:
            e, C, Pp, _ = self.linalg.density(pack(F))
            return e, C, unpack(Pp, self.n)
        e, C = self.diag(F)
        return e, C, C[:, :self.nocc] @ C[:, :self.nocc].T

    def packed_density(self):
        return pack(self.P)

    def step(self, Gp):
        """Consume G[P] of the current density; DIIS-extrapolated F gives the next P."""
        self.it += 1
        G = unpack(Gp, self.n)
        F = self.H + G
        energy = 2.0 * np.sum(self.P * self.H) + np.sum(self.P * G) + self.enuc
        # F, P and S are symmetric, so S P F = (F P S)^T: two GEMMs, not four
        FPS = F @ self.P @ self.S
        err = FPS - FPS.T
        self.fs.append(F)
        e_new = self.X.T @ err @ self.X
        self.es.append(e_new)
        # the error overlaps <e_i, e_j>: one new row a step, the oldest
        # dropped with its vectors
        m0 = self.eov.shape[0]
        eov = np.zeros((m0 + 1, m0 + 1))
        eov[:m0, :m0] = self.eov
        for j in range(m0 + 1):
            eov[m0, j] = eov[j, m0] = np.sum(e_new * self.es[len(self.es) - 1 - m0 + j])
        if self.ediis:
            self._ediis_push(self.P, F, energy)
        self.fs, self.es = self.fs[-self.ndiis:], self.es[-self.ndiis:]
        self.eov = eov[-len(self.es):, -len(self.es):]
        F_last = F
        if len(self.fs) > 1:
            m = len(self.fs)
            B = -np.ones((m + 1, m + 1))
            B[m, m] = 0.0
            B[:m, :m] = self.eov
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            try:
                c = np.linalg.solve(B, rhs)[:m]
                F = sum(ci * Fi for ci, Fi in zip(c, self.fs))
            except np.linalg.LinAlgError:
                pass
        self.err = float(np.max(np.abs(self.es[-1])))
        if self.ediis and len(self.fs) > 1 and self.err > 1e-4:
            # energy-DIIS far from convergence, blended into DIIS between
            # DIIS errors 1e-1 and 1e-4 (weight 10 x error)
            Fe = self._ediis_fock(F_last)
            w = min(1.0, 10.0 * self.err)
            F = w * Fe + (1.0 - w) * F
        if self.level_shift > 0.0 and self.err > self.shift_tol:
            # F + s (S - S P S) raises the virtual space of the current
            # orbitals by s (P S P = P): damps occupied-virtual rotations and
            # orbital flips of small-gap molecules in the early iterations
            SP = self.S @ self.P
            F = F + self.level_shift * (self.S - SP @ self.S)
        self.eps, C, P_new = self.diag_density(F)
        dP = float(np.max(np.abs(P_new - self.P)))
        self.P = P_new
        self.dP = dP
        if self.e_old is not None and abs(energy - self.e_old) < self.conv and \
                self.err < self.comm_tol and dP < self.dp_tol:
            self.converged = True
        self.e_old = energy

    def _ediis_push(self, P, F, energy):
        self.ps.append(P)
        self.ens.append(energy)
        fs = self.fs[-len(self.ps):]
        m = len(self.ps)
        M = np.zeros((m, m))
        M[:m - 1, :m - 1] = self.M
        for j in range(m):
            M[m - 1, j] = np.sum(P * fs[j])
            M[j, m - 1] = np.sum(self.ps[j] * F)
        k = max(0, m - self.ndiis)
        self.ps, self.ens, self.M = self.ps[k:], self.ens[k:], M[k:, k:]

    def _ediis_fock(self, F_fallback):
        """sum_i c_i F_i with c on the simplex minimising the energy of the
        interpolated density, E(c) = sum c_i E_i - 1/2 sum c_i c_j
        tr((P_i - P_j)(F_i - F_j)) -- exact for the closed-shell energy,
        which is quadratic in P (Kudin, Scuseria and Cances, J. Chem. Phys.
        116, 8255 (2002)); c = t^2 / |t|^2 keeps c on the simplex."""
        from scipy.optimize import minimize
        E = np.array(self.ens)
        M = self.M
        d = np.diag(M)
        D = d[:, None] + d[None, :] - M - M.T
        m = len(E)
        fs = self.fs[-m:]

        def f(t):
            t2 = t * t
            s = t2.sum()
            c = t2 / s
            val = c @ E - 0.5 * c @ D @ c
            gc = E - D @ c
            return val, 2.0 * t * (gc - c @ gc) / s

        t0 = np.ones(m) / np.sqrt(m)
        t0[-1] *= 2.0
        try:
            r = minimize(f, t0, jac=True, method="BFGS", options={"maxiter": 200})
            c = r.x * r.x / np.sum(r.x * r.x)
        except Exception:
            return F_fallback
        return sum(ci * Fi for ci, Fi in zip(c, fs))

    def finish(self, Gp) -> RHFResult:
        """Energy and orbitals of the final density."""
        G = unpack(Gp, self.n)
        F = self.H + G
        energy = 2.0 * np.sum(self.P * self.H) + np.sum(self.P * G) + self.enuc
        o = self.nocc
        if self.linalg is not None:
            eps, C, Pp, Wp = self.linalg.density(pack(F))
            self.linalg.close()
        else:
            eps, C = self.diag(F)
            Pp = pack(C[:, :o] @ C[:, :o].T)
            Wp = pack((C[:, :o] * eps[:o]) @ C[:, :o].T)
        return RHFResult(energy=float(energy), P=Pp, W=Wp, C=C, eps=eps, iterations=self.it,
                         converged=self.converged, enuc=self.enuc)


def _setup(gb: GpuBasis, dpm: bool):
    gb.two_electron_ints()
    Sp, _, Hp = gb.one_electron_ints()
    if dpm:
        Hp = gb.dpm_ints(Hp)
    return Sp, Hp


class IncrementalFock:
    """G[P_n] = G[P_(n-1)] + G[P_n - P_(n-1)] with the density-screened
    difference build (patgpu_set_density_screening at tau_inc; the default
    1e-14 drops contributions at the level below which the reference stores
    no integral, twoints.c:375), and a full unscreened build every
    `full_every` iterations.  tau32 > 0: while the density still changes by
    more than fp32_dp_min (early iterations), quartets of a difference build
    whose density-weighted bound is below tau32 run in FP32; the difference
    builds of the final iterations stay FP64.  Records the quartets each
    build computed."""

    def __init__(self, gb: GpuBasis, tau_inc: float = 1e-14, full_every: int = 8, tau32: float = 0.0,
                 fp32_dp_min: float = 1e-4):
        self.gb, self.tau_inc, self.full_every = gb, tau_inc, full_every
        self.tau32, self.fp32_dp_min = tau32, fp32_dp_min
        self.P = self.G = None
        self.n = 0
        self.computed = []

    def __call__(self, Pp, full: bool = False):
        gb = self.gb
        if full or self.G is None or self.n % self.full_every == 0:
            gb.set_density_screening(0.0)
            G = gb.rhf_form_gmatrix(Pp)
        else:
            dP = Pp - self.P
            gb.set_density_screening(self.tau_inc)
            gb.set_density_precision(self.tau32 if float(np.abs(dP).max()) > self.fp32_dp_min else 0.0)
            G = self.G + gb.rhf_form_gmatrix(dP)
            gb.set_density_screening(0.0)
            gb.set_density_precision(0.0)
        self.computed.append(gb.last_computed())
        self.n += 1
        self.P, self.G = Pp.copy(), G
        return G


def rhf(basis: Basis, dpm: bool = False, gpu: GpuBasis | None = None, conv: float = 1e-12,
        maxit: int = 100, schwarz_tau: float = 1e-14, ndiis: int = 8, incremental: bool = False,
        tau_inc: float = 1e-14, device_linalg: bool = False, tau_fp32: float = 0.0, tau_inc32: float = 0.0,
        comm_tol: float = 1e-9, dp_tol: float = 1e-8, smin: float = 1e-10, level_shift: float = 0.0,
        shift_tol: float = 1e-3, full_every: int = 8, ediis: bool = False) -> RHFResult:
    """Closed-shell SCF.  incremental=True builds G from density differences
    (IncrementalFock) during the iterations; the final energy always comes
    from a full build.  device_linalg=True diagonalises on the GPU.
    tau_fp32 > 0 runs quartets whose Rys-term bound is below it in FP32
    (mixed precision) in every build.  level_shift > 0 raises the virtual
    orbitals by that many Eh while the DIIS error exceeds shift_tol.
    ediis=True blends energy-DIIS into DIIS while the DIIS error is above
    1e-4 (_RHFState._ediis_fock)."""
    gb = gpu if gpu is not None else GpuBasis(basis, schwarz_tau=schwarz_tau)
    Sp, Hp = _setup(gb, dpm)
    if tau_fp32 > 0.0:
        gb.set_mixed_precision(tau_fp32)
    st = _RHFState(basis, Sp, Hp, ndiis, conv, device_linalg=device_linalg, comm_tol=comm_tol, dp_tol=dp_tol,
                   smin=smin, level_shift=level_shift, shift_tol=shift_tol, ediis=ediis)
    fock = IncrementalFock(gb, tau_inc, full_every=full_every, tau32=tau_inc32) if incremental else None
    fock_ns = 0.0
    while st.it < maxit and not st.converged:
        Pp = st.packed_density()
        G = fock(Pp) if fock else gb.rhf_form_gmatrix(Pp)
        fock_ns += gb.last_timing()[0]
        st.step(G)
    res = st.finish(gb.rhf_form_gmatrix(st.packed_density()))
    res.quartets_computed = fock.computed if fock else None
    res.fock_seconds = fock_ns * 1e-9
    if tau_fp32 > 0.0:
        gb.set_mixed_precision(0.0)
    if gpu is None:
        gb.close()
    return res


def rhf_batch(bases, dpm: bool = False, tau_fp32: float = 0.0, conv: float = 1e-12, maxit: int = 100,
              schwarz_tau: float = 1e-14, ndiis: int = 8, incremental: bool = False, tau_inc: float = 1e-11,
              tau_inc32: float = 0.0, fp32_dp_min: float = 1e-4, full_every: int = 8, comm_tol: float = 1e-9,
              dp_tol: float = 1e-8, computed: list | None = None, smin: float = 1e-10,
              device_linalg: bool = False, fock_seconds: list | None = None, level_shift: float = 0.0,
              shift_tol: float = 1e-3, tau_full: float = 0.0, tau_rel: float = 0.0, tau_max: float = 1e-8,
              ediis: bool = False):
    """Closed-shell SCF of many molecules in lock step: every iteration is one
    batched Fock build (one CUDA graph over all molecules, patgpu_batch_*),
    then each molecule's host step.  Converged molecules keep their density.
    tau_fp32 > 0 runs quartets with Rys-term bound below it in FP32.
    incremental=True: between full builds (the first and every full_every-th
    iteration) the graph builds G[P_n - P_(n-1)] of every molecule with
    density screening at tau_inc (the filter runs inside the graph) and adds
    it to the previous G; while a molecule's density still changes by more
    than fp32_dp_min, tau_inc32 > 0 also runs its kept quartets with a
    density-weighted bound below tau_inc32 in FP32 (the difference builds of
    the final iterations stay FP64).  A converged molecule's difference is
    zero, so the filter drops all of its quartets.  tau_full > 0 screens the
    full builds of the iterations by the density as well, at that bound, and
    gives converged molecules a zero density there, so that they cost
    nothing after convergence.  The final energies come from an unscreened
    full build.  tau_rel > 0 tightens the screening with the SCF: each
    molecule's build is screened at tau_rel times its own DIIS error,
    clipped to [tau_inc, tau_max] (the first build at tau_max): early
    iterations, whose Fock matrices are far from self-consistent anyway,
    drop many more quartets, and the error each build's screening adds stays
    far below the error the molecule's SCF has left; the full builds of the
    iterations use the same thresholds.  level_shift /
    shift_tol / ediis as in rhf().  computed, if given, receives the quartets of
    every build, and fock_seconds the device-timed seconds of every batched
    build."""
    gbs = [GpuBasis(b, schwarz_tau=schwarz_tau) for b in bases]
    states = []
    for b, gb in zip(bases, gbs):
        Sp, Hp = _setup(gb, dpm)
        states.append(_RHFState(b, Sp, Hp, ndiis, conv, comm_tol=comm_tol, dp_tol=dp_tol, smin=smin,
                                device_linalg=device_linalg, level_shift=level_shift, shift_tol=shift_tol,
                                ediis=ediis))
    batch = GpuBatch(gbs)
    if tau_fp32 > 0.0:
        batch.set_mixed_precision(tau_fp32)
    it = 0
    Gprev = Pprev = None

    def thresholds(floor):
        # per molecule: adaptive (tau_rel > 0: its own DIIS error) or fixed
        out = []
        for st in states:
            e = st.err
            out.append(floor if tau_rel <= 0.0 else
                       (tau_max if not np.isfinite(e) else min(tau_max, max(floor, tau_rel * e))))
        return out

    while it < maxit and not all(st.converged for st in states):
        it += 1
        Ps = [st.packed_density() for st in states]
        if not incremental or Gprev is None or (it - 1) % full_every == 0:
            if tau_rel > 0.0 and Gprev is None:
                batch.set_density_screening(tau_max)
                Gs = batch.rhf_form_gmatrix(Ps)
            elif (tau_full > 0.0 or tau_rel > 0.0) and Gprev is not None:
                batch.set_density_thresholds(thresholds(max(tau_full, 1e-14)))
                Gn = batch.rhf_form_gmatrix([np.zeros_like(P) if st.converged else P
                                             for P, st in zip(Ps, states)])
                Gs = [Gp if st.converged else G for G, Gp, st in zip(Gn, Gprev, states)]
            else:
                batch.set_density_screening(0.0)
                Gs = batch.rhf_form_gmatrix(Ps)
        else:
            dPs = [P - Pp for P, Pp in zip(Ps, Pprev)]
            t32 = [tau_inc32 if float(np.abs(d).max()) > fp32_dp_min else 0.0 for d in dPs]
            batch.set_density_thresholds(thresholds(tau_inc), t32)
            Gs = [Gp + dG for Gp, dG in zip(Gprev, batch.rhf_form_gmatrix(dPs))]
        if computed is not None:
            computed.append(batch.last_computed())
        if fock_seconds is not None:
            fock_seconds.append(batch.last_timing_ns() * 1e-9)
        Gprev, Pprev = Gs, Ps
        for st, G in zip(states, Gs):
            if not st.converged:
                st.step(G)
    batch.set_density_screening(0.0)
    Gs = batch.rhf_form_gmatrix([st.packed_density() for st in states])
    out = [st.finish(G) for st, G in zip(states, Gs)]
    batch.close()
    for gb in gbs:
        gb.close()
    return out


@dataclass
class UHFResult:
    energy: float
    PA: np.ndarray         # packed alpha density
    PB: np.ndarray         # packed beta density
    WA: np.ndarray         # packed energy-weighted alpha density
    WB: np.ndarray
    iterations: int
    converged: bool
    enuc: float


def uhf(basis: Basis, dpm: bool = False, gpu: GpuBasis | None = None, conv: float = 1e-12,
        maxit: int = 150, schwarz_tau: float = 1e-14, ndiis: int = 8) -> UHFResult:
    """Open-shell SCF: the iteration of uhf_scf_update (uhfscf.c:23-78) with
    G_s = J[Pa+Pb] - K[P_s] from the GPU (uhf_form_gmatrix), occupations of
    uhfscf.c:120-122 (n_b = (N - (2S+1) + 1)/2, n_a = N - n_b), energy
    E = sum_s [tr(P_s H) + tr(P_s G_s)/2] + E_nuc (uhfscf.c:54-55,
    scfaux.c:100-118), and DIIS over both spins' commutators."""
    gb = gpu if gpu is not None else GpuBasis(basis, schwarz_tau=schwarz_tau)
    Sp, Hp = _setup(gb, dpm)
    n = basis.norb
    nb = (basis.nelec - (basis.mult - 1)) // 2
    na = basis.nelec - nb
    S, H = unpack(Sp, n), unpack(Hp, n)
    X = orthogonalizer(S)
    enuc = nuclear_repulsion(basis)

    def diag(F):
        e, V = np.linalg.eigh(X.T @ F @ X)
        return e, X @ V

    e0, C0 = diag(H)
    P = [C0[:, :na] @ C0[:, :na].T, C0[:, :nb] @ C0[:, :nb].T]
    occ = (na, nb)
    hist_f, hist_e = [], []
    e_old, converged, it = None, False, 0
    for it in range(1, maxit + 1):
        GA, GB = gb.uhf_form_gmatrix(pack(P[0]), pack(P[1]))
        G = [unpack(GA, n), unpack(GB, n)]
        F = [H + G[0], H + G[1]]
        energy = sum(np.sum(P[s] * H) + 0.5 * np.sum(P[s] * G[s]) for s in range(2)) + enuc
        FPS = [F[s] @ P[s] @ S for s in range(2)]
        errs = [X.T @ (FPS[s] - FPS[s].T) @ X for s in range(2)]   # S P F = (F P S)^T
        hist_f.append(F)
        hist_e.append(errs)
        hist_f, hist_e = hist_f[-ndiis:], hist_e[-ndiis:]
        if len(hist_f) > 1:
            m = len(hist_f)
            B = -np.ones((m + 1, m + 1))
            B[m, m] = 0.0
            for i in range(m):
                for j in range(m):
                    B[i, j] = sum(np.sum(hist_e[i][s] * hist_e[j][s]) for s in range(2))
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            try:
                c = np.linalg.solve(B, rhs)[:m]
                F = [sum(ci * Fi[s] for ci, Fi in zip(c, hist_f)) for s in range(2)]
            except np.linalg.LinAlgError:
                pass
        newP = []
        for s in range(2):
            e, C = diag(F[s])
            newP.append(C[:, :occ[s]] @ C[:, :occ[s]].T)
        dP = max(float(np.abs(newP[s] - P[s]).max()) for s in range(2))
        P = newP
        if e_old is not None and abs(energy - e_old) < conv and dP < 1e-8 and \
                max(float(np.abs(x).max()) for x in errs) < 1e-9:
            converged = True
            break
        e_old = energy
    GA, GB = gb.uhf_form_gmatrix(pack(P[0]), pack(P[1]))
    G = [unpack(GA, n), unpack(GB, n)]
    energy = sum(np.sum(P[s] * H) + 0.5 * np.sum(P[s] * G[s]) for s in range(2)) + enuc
    out_P, out_W = [], []
    for s in range(2):
        e, C = diag(H + G[s])
        o = occ[s]
        out_P.append(pack(C[:, :o] @ C[:, :o].T))
        out_W.append(pack((C[:, :o] * e[:o]) @ C[:, :o].T))
    if gpu is None:
        gb.close()
    return UHFResult(energy=float(energy), PA=out_P[0], PB=out_P[1], WA=out_W[0], WB=out_W[1], iterations=it,
                     converged=converged, enuc=enuc)


def uhf_gradient(basis: Basis, res: UHFResult, dpm: bool = False, gpu: GpuBasis | None = None,
                 parts: int = GpuBasis.GRAD_ALL, schwarz_tau: float = 1e-14) -> np.ndarray:
    """dE/dR (ncen x 3, Eh/bohr) of the converged open-shell energy."""
    gb = gpu if gpu is not None else GpuBasis(basis, schwarz_tau=schwarz_tau)
    g = gb.uhf_gradient(res.PA, res.PB, res.WA, res.WB, parts=parts, with_dpm=dpm)
    if gpu is None:
        gb.close()
    return g


def rhf_gradient(basis: Basis, res: RHFResult, dpm: bool = False, gpu: GpuBasis | None = None,
                 parts: int = GpuBasis.GRAD_ALL, schwarz_tau: float = 1e-14) -> np.ndarray:
    """dE/dR (ncen x 3, Eh/bohr) of the converged closed-shell energy."""
    gb = gpu if gpu is not None else GpuBasis(basis, schwarz_tau=schwarz_tau)
    g = gb.rhf_gradient(res.P, res.W, parts=parts, with_dpm=dpm)
    if gpu is None:
        gb.close()
    return g
