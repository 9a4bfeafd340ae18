"""Generate the Rys root/weight tables used by the GPU kernels (rys_table.h).

The Rys quadrature of order n at argument T is the n-point Gauss rule, in
x = t^2 on [0, 1], for the weight exp(-T x) / (2 sqrt(x)); its moments are
the Boys values F_m(T).  This script computes nodes and weights in 50-digit
arithmetic (mpmath): moments by the Boys series, recurrence coefficients by
the Chebyshev algorithm, nodes and weights by the symmetric tridiagonal
eigenproblem (Golub-Welsch).  It then fits, for every n <= NMAX, each node
and weight on unit-width intervals of T in [0, TMAX(n)) by a Chebyshev
series of degree DEG.  Above TMAX(n) the kernels use the large-T limit, in
which the rule becomes generalised Gauss-Laguerre (alpha = -1/2) scaled by
1/T: x_i = s_i / T, w_i = W_i / (2 sqrt(T)); TMAX(n) is chosen here as the
first T beyond which that limit is exact to 1e-16 relative.

Run:  python patmol_b200/csrc/gen_rys_table.py   (about two minutes)
Writes rys_table.h (C arrays) and rys_table.npz (the same numbers, for the
host-side accuracy test).
"""
from __future__ import annotations

import os
import sys
from multiprocessing import Pool

import mpmath as mp
import numpy as np

NMAX = 9          # up to (gg|gg); the kernels instantiate up to (ff|ff)
DEG = 11          # Chebyshev degree per unit interval (fit error ~2.5e-15 relative)
DPS = 50
HERE = os.path.dirname(os.path.abspath(__file__))


def boys_mp(mmax, T):
    T = mp.mpf(T)
    if T == 0:
        return [mp.mpf(1) / (2 * m + 1) for m in range(mmax + 1)]
    e = mp.exp(-T)
    if T > 60:
        st = mp.sqrt(T)
        F = [mp.sqrt(mp.pi) / 2 * mp.erf(st) / st]
        for m in range(mmax):
            F.append(((2 * m + 1) * F[m] - e) / (2 * T))
        return F
    term = mp.mpf(1) / (2 * mmax + 1)
    s = term
    i = 1
    while True:
        term *= 2 * T / (2 * mmax + 2 * i + 1)
        s += term
        i += 1
        if term < mp.mpf(10) ** (-DPS - 5) * s:
            break
    F = [mp.mpf(0)] * (mmax + 1)
    F[mmax] = e * s
    for m in range(mmax - 1, -1, -1):
        F[m] = (2 * T * F[m + 1] + e) / (2 * m + 1)
    return F


def rys_mp(n, T):
    mp.mp.dps = DPS
    mu = boys_mp(2 * n, T)
    al = [mp.mpf(0)] * n
    be = [mp.mpf(0)] * n
    lev = [[mp.mpf(0)] * (2 * n + 1) for _ in range(n + 1)]
    for l in range(2 * n):
        lev[0][l] = mu[l]
    al[0] = mu[1] / mu[0]
    be[0] = mu[0]
    for k in range(1, n):
        for l in range(k, 2 * n - k):
            prev2 = lev[k - 2][l] if k >= 2 else 0
            lev[k][l] = lev[k - 1][l + 1] - al[k - 1] * lev[k - 1][l] - be[k - 1] * prev2
        al[k] = lev[k][k + 1] / lev[k][k] - lev[k - 1][k] / lev[k - 1][k - 1]
        be[k] = lev[k][k] / lev[k - 1][k - 1]
    J = mp.matrix(n, n)
    for k in range(n):
        J[k, k] = al[k]
    for k in range(n - 1):
        J[k, k + 1] = J[k + 1, k] = mp.sqrt(be[k + 1])
    E, Q = mp.eigsy(J)
    pairs = sorted([(E[i], be[0] * Q[0, i] ** 2) for i in range(n)], key=lambda p: p[0])
    return [p[0] for p in pairs], [p[1] for p in pairs]


def laguerre_half(n):
    """Nodes and weights of Gauss-Laguerre with alpha = -1/2 (= squared
    positive Gauss-Hermite nodes of order 2n)."""
    mp.mp.dps = DPS
    # Jacobi matrix of generalised Laguerre: a_k = 2k + alpha + 1, b_k = k (k + alpha)
    a = -mp.mpf(1) / 2
    J = mp.matrix(n, n)
    for k in range(n):
        J[k, k] = 2 * k + a + 1
    for k in range(1, n):
        J[k, k - 1] = J[k - 1, k] = mp.sqrt(k * (k + a))
    E, Q = mp.eigsy(J)
    mu0 = mp.gamma(a + 1)
    pairs = sorted([(E[i], mu0 * Q[0, i] ** 2) for i in range(n)], key=lambda p: p[0])
    return [p[0] for p in pairs], [p[1] for p in pairs]


def asym(n, T, lag):
    s, W = lag
    T = mp.mpf(T)
    return [x / T for x in s], [w / (2 * mp.sqrt(T)) for w in W]


def find_tmax(n, lag):
    T = 20
    while True:
        x, w = rys_mp(n, T)
        xa, wa = asym(n, T, lag)
        err = max(max(abs(a / b - 1) for a, b in zip(xa, x)), max(abs(a / b - 1) for a, b in zip(wa, w)))
        if err < 1e-17:
            return T
        T += 1


def cheb_nodes(deg):
    k = np.arange(deg + 1)
    return np.cos(np.pi * (k + 0.5) / (deg + 1))


def fit_interval(args):
    n, t0 = args
    mp.mp.dps = DPS
    u = cheb_nodes(DEG)
    vals = []
    for uu in u:
        T = mp.mpf(t0) + (mp.mpf(float(uu)) + 1) / 2
        x, w = rys_mp(n, T)
        vals.append([float(v) for v in x] + [float(v) for v in w])
    vals = np.array(vals)                      # (DEG+1, 2n)
    # Chebyshev coefficients by the discrete cosine transform at the nodes
    k = np.arange(DEG + 1)
    theta = np.pi * (k + 0.5) / (DEG + 1)
    C = np.zeros((2 * n, DEG + 1))
    for j in range(DEG + 1):
        C[:, j] = 2.0 / (DEG + 1) * (vals * np.cos(j * theta)[:, None]).sum(axis=0)
    C[:, 0] *= 0.5
    return n, t0, C


def main():
    mp.mp.dps = DPS
    lags = {n: laguerre_half(n) for n in range(1, NMAX + 1)}
    tmax = {}
    with Pool(min(8, os.cpu_count() or 1)) as pool:
        tm = pool.starmap(find_tmax, [(n, lags[n]) for n in range(1, NMAX + 1)])
    for n, t in zip(range(1, NMAX + 1), tm):
        tmax[n] = int(t)
    jobs = [(n, t0) for n in range(1, NMAX + 1) for t0 in range(tmax[n])]
    with Pool(min(8, os.cpu_count() or 1)) as pool:
        res = pool.map(fit_interval, jobs, chunksize=4)
    coefs = {}
    for n, t0, C in res:
        coefs[(n, t0)] = C
    # flatten: per n, intervals, per function (n roots then n weights), DEG+1
    offs = [0]
    flat = []
    for n in range(1, NMAX + 1):
        for t0 in range(tmax[n]):
            flat.append(coefs[(n, t0)].reshape(-1))
        offs.append(offs[-1] + tmax[n] * 2 * n * (DEG + 1))
    flat = np.concatenate(flat)
    lag_x = np.zeros((NMAX + 1, NMAX))
    lag_w = np.zeros((NMAX + 1, NMAX))
    for n in range(1, NMAX + 1):
        lag_x[n, :n] = [float(v) for v in lags[n][0]]
        lag_w[n, :n] = [float(v) / 2 for v in lags[n][1]]     # includes the 1/2 of w = W/(2 sqrt T)
    np.savez(os.path.join(HERE, "rys_table.npz"), coef=flat, off=np.array(offs[:-1]),
             tmax=np.array([0] + [tmax[n] for n in range(1, NMAX + 1)]), deg=DEG,
             lag_x=lag_x, lag_w=lag_w)
    with open(os.path.join(HERE, "rys_table.h"), "w") as f:
        f.write("/* Generated by gen_rys_table.py: Chebyshev fits (degree %d, unit\n" % DEG)
        f.write(" * intervals in T) of the Rys nodes x = t^2 and weights for n <= %d,\n" % NMAX)
        f.write(" * plus the large-T Laguerre(alpha=-1/2) limits.  Do not edit. */\n")
        f.write("#pragma once\n")
        f.write("#define RYS_NMAX %d\n#define RYS_DEG %d\n" % (NMAX, DEG))
        f.write("static const int rys_tmax[RYS_NMAX + 1] = {%s};\n" %
                ", ".join(str(v) for v in [0] + [tmax[n] for n in range(1, NMAX + 1)]))
        f.write("static const int rys_off[RYS_NMAX + 1] = {0, %s};\n" % ", ".join(str(v) for v in offs[:-1]))
        f.write("static const int rys_ncoef = %d;\n" % len(flat))
        f.write("static const double rys_lag_x[RYS_NMAX + 1][RYS_NMAX] = {\n")
        for n in range(NMAX + 1):
            f.write("  {%s},\n" % ", ".join("%.17e" % v for v in lag_x[n]))
        f.write("};\nstatic const double rys_lag_w[RYS_NMAX + 1][RYS_NMAX] = {\n")
        for n in range(NMAX + 1):
            f.write("  {%s},\n" % ", ".join("%.17e" % v for v in lag_w[n]))
        f.write("};\nstatic const double rys_coef_host[%d] = {\n" % len(flat))
        for i in range(0, len(flat), 4):
            f.write("  " + ", ".join("%.17e" % v for v in flat[i:i + 4]) + ",\n")
        f.write("};\n")
    print("tmax", tmax, "coefs", len(flat))


if __name__ == "__main__":
    sys.exit(main())
