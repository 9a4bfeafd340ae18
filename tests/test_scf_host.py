"""Host-side SCF logic that needs no GPU: the energy-DIIS step of
scf._RHFState (the coefficients on the simplex that minimise the
closed-shell energy of the interpolated density, which is exact because the
energy is quadratic in P), checked on a model problem against a brute-force
search of the simplex and against the energy evaluated directly."""
import itertools

import numpy as np

from patmol_b200 import scf


def _model(n=6, m=4, seed=3):
    """A closed-shell model: H, a symmetric positive two-electron operator
    G[P] (linear in P), and m random densities with their Fock matrices
    F_i = H + G[P_i] and energies E_i = tr(P_i (H + F_i))."""
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n))
    H = -(A @ A.T) / n
    W = rng.normal(size=(n * n, n * n)) * 0.05
    W = W @ W.T

    def G(P):
        return (W @ P.reshape(-1)).reshape(n, n)

    Ps, Fs, Es = [], [], []
    for _ in range(m):
        B = rng.normal(size=(n, 2))
        P = B @ B.T * 0.3
        F = H + G(P)
        Ps.append(P)
        Fs.append(F)
        Es.append(float(np.sum(P * (H + F))))

    def energy(P):
        return float(np.sum(P * (H + H + G(P))))

    return Ps, Fs, Es, energy


def _state(Ps, Fs, Es):
    st = scf._RHFState.__new__(scf._RHFState)
    st.ndiis = len(Ps)
    st.fs, st.ps, st.ens, st.M = [], [], [], np.zeros((0, 0))
    for P, F, E in zip(Ps, Fs, Es):
        st.fs.append(F)
        st._ediis_push(P, F, E)
    return st


def test_ediis_energy_model_is_exact():
    Ps, Fs, Es, energy = _model()
    st = _state(Ps, Fs, Es)
    E = np.array(st.ens)
    d = np.diag(st.M)
    D = d[:, None] + d[None, :] - st.M - st.M.T
    rng = np.random.default_rng(0)
    for _ in range(5):
        c = rng.dirichlet(np.ones(len(Ps)))
        model = c @ E - 0.5 * c @ D @ c
        assert abs(model - energy(sum(ci * P for ci, P in zip(c, Ps)))) < 1e-10


def test_ediis_minimises_over_the_simplex():
    Ps, Fs, Es, energy = _model()
    st = _state(Ps, Fs, Es)
    F = st._ediis_fock(None)
    # recover the coefficients from F = sum c_i F_i (the F_i are independent)
    A = np.stack([f.reshape(-1) for f in Fs], axis=1)
    c = np.linalg.lstsq(A, F.reshape(-1), rcond=None)[0]
    assert abs(c.sum() - 1.0) < 1e-8 and c.min() > -1e-8
    got = energy(sum(ci * P for ci, P in zip(c, Ps)))
    best = np.inf
    steps = 40
    for k in itertools.product(range(steps + 1), repeat=len(Ps) - 1):
        if sum(k) > steps:
            continue
        w = np.array(list(k) + [steps - sum(k)], dtype=float) / steps
        best = min(best, energy(sum(wi * P for wi, P in zip(w, Ps))))
    assert got <= best + 1e-9, (got, best)
