/*
 * patref.c -- CPU restatement of the Patmol SCF hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the GPU library is
 * checked against; nothing in the product links, loads or calls it, and the
 * GPU library has no CPU fallback to it.  It is pinned against the compiled
 * reference (oracle/_ref) through the fixtures in tests/golden.
 *
 * Reference functions restated (file:line in the Patmol tree):
 *   Boys function            mdr.c:6-35            patref_boys
 *   Rys roots and weights    rys.c:2217-2244 (role), rys.c:245-323 (moment
 *                            method of rootN)      patref_rys
 *   2-D Rys recursion        rys.c:2269-2293       rys_vrr
 *   binomial transfer (HRR)  rys.c:2295-2336       rys_shift
 *   primitive quartet loop   twoints.c:23-186      patref_eri_block
 *   quartet enumeration      twoints.c:228-404     patref_gmat
 *   G digestion RHF / UHF    scfaux.c:446-495, 575-650
 *   MD E coefficients        mdd.c:3-43            md_e
 *   MD R integrals           mdr.c:37-2163         md_r (recursive form)
 *   one-electron S, T, V     oneints.c:12-234      patref_oneints
 *   DPM potential            dpmints.c:18-199      patref_dpm
 *   nuclear repulsion        basis.c:174-195       patref_enuc
 */
#include "patref.h"

#include <math.h>
#include <pthread.h>
#include <quadmath.h>
#include <unistd.h>
#include <stdlib.h>
#include <string.h>

#define MAXLS 5                 /* pconfig.h:9 */
#define MAXR (2 * MAXLS + 1)    /* rys.h:7, MAXROOTS */
#define LT (4 * MAXLS + 1)

typedef __float128 quad;

/* ---------------------------------------------------------------- basis */
static struct {
    int nsh, ncen, skip;
    int *l, *cen, *off, *nst, *poff;
    double *al, *co, *q, *xyz;
} B;

static const double dfact[] = {1., 1., 3., 15., 105., 945., 10395., 135135.};

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

/* Cartesian order of basis.c:294-308 (lx descending, then ly descending) */
static void comp(int l, int k, int *lx, int *ly, int *lz)
{
    int a, b, n = 0;
    for (a = l; a >= 0; --a)
        for (b = l - a; b >= 0; --b) {
            if (n == k) { *lx = a; *ly = b; *lz = l - a - b; return; }
            ++n;
        }
}

static double comp_norm(int l, int k)   /* basis.c:309-319 */
{
    int x, y, z;
    comp(l, k, &x, &y, &z);
    return 1.0 / sqrt(dfact[x] * dfact[y] * dfact[z]);
}

static void *pr_dup(const void *p, size_t n)
{
    void *q = malloc(n ? n : 1);
    memcpy(q, p, n);
    return q;
}

void patref_set_basis(int nshell, const int *l, const int *cen, const int *off,
                      const int *nst, const int *poff, const double *al,
                      const double *co, int ncen, const double *q,
                      const double *xyz, int skipcen)
{
    free(B.l); free(B.cen); free(B.off); free(B.nst); free(B.poff);
    free(B.al); free(B.co); free(B.q); free(B.xyz);
    B.nsh = nshell;
    B.ncen = ncen;
    B.skip = skipcen;
    B.l = pr_dup(l, sizeof(int) * nshell);
    B.cen = pr_dup(cen, sizeof(int) * nshell);
    B.off = pr_dup(off, sizeof(int) * nshell);
    B.nst = pr_dup(nst, sizeof(int) * nshell);
    B.poff = pr_dup(poff, sizeof(int) * (nshell + 1));
    B.al = pr_dup(al, sizeof(double) * poff[nshell]);
    B.co = pr_dup(co, sizeof(double) * poff[nshell]);
    B.q = pr_dup(q, sizeof(double) * ncen);
    B.xyz = pr_dup(xyz, sizeof(double) * 3 * ncen);
}

/* ---------------------------------------------------------- Boys (FP64) */
/* mdr.c:6-35: Taylor series at m, downward recursion; the asymptotic
 * form above T = 36 + 2m. */
void patref_boys(int m, double T, double *F)
{
    int i;
    if (T > 36.0 + 2.0 * m) {
        F[0] = 0.88622692545275801365 / sqrt(T);
        for (i = 1; i <= m; ++i) F[i] = F[i - 1] * (i - 0.5) / T;
        return;
    }
    {
        double mh = m + 0.5, term = 0.5 / mh, sum = term, e = exp(-T);
        for (i = 1; i <= 500; ++i) {
            term *= T / (mh + i);
            sum += term;
            if (term < 1e-17 * sum) break;
        }
        F[m] = sum * e;
        for (i = m - 1; i >= 0; --i) F[i] = (2.0 * T * F[i + 1] + e) / (2.0 * i + 1.0);
    }
}

/* ------------------------------------------------- Rys roots (quad) */
/* Boys moments F_0..F_mmax in quad precision: series + downward recursion
 * below T = max(30, mmax), upward recursion from erf above (stable there). */
static void boys_quad(int mmax, quad T, quad *F)
{
    int i;
    if (T >= 30.0Q && T >= (quad)mmax) {
        quad e = expq(-T), st = sqrtq(T);
        F[0] = 0.5Q * sqrtq(M_PIq) * erfq(st) / st;
        for (i = 0; i < mmax; ++i) F[i + 1] = ((2 * i + 1) * F[i] - e) / (2.0Q * T);
        return;
    }
    {
        quad term = 1.0Q / (2 * mmax + 1), sum = term, e = expq(-T);
        for (i = 1; i < 4000; ++i) {
            term *= 2.0Q * T / (2 * mmax + 2 * i + 1);
            sum += term;
            if (term < 1e-40Q * sum) break;
        }
        F[mmax] = e * sum;
        for (i = mmax - 1; i >= 0; --i) F[i] = (2.0Q * T * F[i + 1] + e) / (2 * i + 1);
    }
}

static int sturm_count(int n, const double *a, const double *b2, double x)
{
    int k, c = 0;
    double q = a[0] - x;
    if (q < 0) ++c;
    for (k = 1; k < n; ++k) {
        if (q == 0.0) q = 1e-300;
        q = (a[k] - x) - b2[k] / q;
        if (q < 0) ++c;
    }
    return c;
}

/* Gauss quadrature in x = t^2 for the weight exp(-T x)/(2 sqrt x) on [0,1]
 * (the Rys weight; its moments are the Boys values F_m(T)).  Returns the
 * roots as t^2 (the reference stores u = t^2/(1-t^2), rys.c:317-321, and
 * converts back with drt = u/(1+u), twoints.c:122) and the weights, whose
 * sum is F_0(T).  Moments -> recurrence by the Chebyshev algorithm in quad,
 * nodes by Sturm bisection then Newton on the monic orthogonal polynomial,
 * weights by the Christoffel formula (the reference's rootN also uses
 * Christoffel weights, rys.c:290-305). */
int patref_rys(int n, double Td, double *xr, double *wr)
{
    quad mu[2 * MAXR + 2], lev[MAXR + 1][2 * MAXR + 2], al[MAXR + 1], be[MAXR + 1];
    double ad[MAXR + 1], b2d[MAXR + 1];
    quad T = Td;
    int k, l, i;
    if (n < 1 || n > MAXR) return -1;
    boys_quad(2 * n, T, mu);
    /* Chebyshev algorithm on the ordinary moments: lev[k][l] = sigma_{k,l} */
    for (l = 0; l < 2 * n; ++l) lev[0][l] = mu[l];
    al[0] = mu[1] / mu[0];
    be[0] = mu[0];
    for (k = 1; k < n; ++k) {
        for (l = k; l < 2 * n - k; ++l) {
            quad prev2 = (k >= 2) ? lev[k - 2][l] : 0.0Q;
            lev[k][l] = lev[k - 1][l + 1] - al[k - 1] * lev[k - 1][l] - be[k - 1] * prev2;
        }
        al[k] = lev[k][k + 1] / lev[k][k] - lev[k - 1][k] / lev[k - 1][k - 1];
        be[k] = lev[k][k] / lev[k - 1][k - 1];
    }
    for (k = 0; k < n; ++k) { ad[k] = (double)al[k]; b2d[k] = (double)be[k]; }
    for (i = 0; i < n; ++i) {
        double lo = 0.0, hi = 1.0, x0;
        int it;
        for (it = 0; it < 64; ++it) {
            double mid = 0.5 * (lo + hi);
            if (sturm_count(n, ad, b2d, mid) > i) hi = mid; else lo = mid;
        }
        x0 = 0.5 * (lo + hi);
        {
            quad x = x0;
            for (it = 0; it < 3; ++it) {
                quad p0 = 1, p1 = x - al[0], d0 = 0, d1 = 1;
                for (k = 1; k < n; ++k) {
                    quad p2 = (x - al[k]) * p1 - be[k] * p0;
                    quad d2 = p1 + (x - al[k]) * d1 - be[k] * d0;
                    p0 = p1; p1 = p2; d0 = d1; d1 = d2;
                }
                if (n == 1) { p1 = x - al[0]; d1 = 1; }
                if (d1 != 0) x -= p1 / d1;
            }
            {
                /* Christoffel: 1/w = sum_k phat_k(x)^2, phat orthonormal */
                quad s = 0, pm1 = 0, pk = 1.0Q / sqrtq(be[0]), nrm;
                s = pk * pk;
                for (k = 0; k < n - 1; ++k) {
                    quad sb = sqrtq(be[k + 1]);
                    quad pn = ((x - al[k]) * pk - (k ? sqrtq(be[k]) : 0.0Q) * pm1) / sb;
                    pm1 = pk; pk = pn;
                    s += pk * pk;
                }
                nrm = 1.0Q / s;
                xr[i] = (double)x;
                wr[i] = (double)nrm;
            }
        }
    }
    return 0;
}

/* ------------------------------------------------ Rys VRR and transfer */
/* rys.c:2269-2293: G[i][j], i <= l12 (bra), j <= l34 (ket) */
static void rys_vrr(double G[LT][LT], int l12, int l34, double B00, double B1,
                    double B1p, double C, double Cp)
{
    int i, j;
    G[0][0] = 1.0;
    if (l12 > 0) G[1][0] = C;
    for (i = 1; i < l12; ++i) G[i + 1][0] = i * B1 * G[i - 1][0] + C * G[i][0];
    for (j = 0; j < l34; ++j) {
        for (i = 0; i <= l12; ++i) {
            double v = Cp * G[i][j];
            if (j > 0) v += j * B1p * G[i][j - 1];
            if (i > 0) v += i * B00 * G[i - 1][j];
            G[i][j + 1] = v;
        }
    }
}

static double binom[LT][LT];

static void init_binom(void)
{
    int i, j;
    if (binom[0][0] == 1.0) return;
    for (i = 0; i < LT; ++i) {
        binom[i][0] = 1.0;
        for (j = 1; j <= i; ++j) binom[i][j] = binom[i - 1][j - 1] + (j <= i - 1 ? binom[i - 1][j] : 0.0);
    }
}

/* rys.c:2295-2336: I(l1,l2;l3,l4) = sum_i C(l2,i) AB^i sum_j C(l4,j) CD^j
 * G[l1+l2-i][l3+l4-j] */
static double rys_shift(double ab, double cd, double G[LT][LT], int l1, int l2, int l3, int l4)
{
    int i, j;
    double s = 0.0, abp = 1.0;
    for (i = 0; i <= l2; ++i) {
        double cdp = 1.0, t = 0.0;
        for (j = 0; j <= l4; ++j) {
            t += binom[l4][j] * cdp * G[l1 + l2 - i][l3 + l4 - j];
            cdp *= cd;
        }
        s += binom[l2][i] * abp * t;
        abp *= ab;
    }
    return s;
}

/* ------------------------------------------------------- ERI block */
/* One contracted shell quartet, every component combination, in the
 * requested (a b | c d) order: out[((ia*nb + ib)*nc + ic)*nd + id].
 * Follows calc_pteints (twoints.c:23-186): larger l first in each pair
 * (twoints.c:249-266,297-314), prefactor 2 pi^(5/2) s12 s34/(p q sqrt(p+q)),
 * primitive cut 1e-15 before the contraction coefficients
 * (twoints.c:109-111), T = rho |PQ|^2, nroots = L/2 + 1 (twoints.c:46). */
int patref_eri_block(int a, int b, int c, int d, double *out)
{
    const double SR = 34.9868366552497250;   /* 2 pi^(5/2) */
    int sw12 = B.l[a] < B.l[b], sw34 = B.l[c] < B.l[d];
    int s1 = sw12 ? b : a, s2 = sw12 ? a : b, s3 = sw34 ? d : c, s4 = sw34 ? c : d;
    int l1 = B.l[s1], l2 = B.l[s2], l3 = B.l[s3], l4 = B.l[s4];
    int n1 = ncart(l1), n2 = ncart(l2), n3 = ncart(l3), n4 = ncart(l4);
    int na = ncart(B.l[a]), nb = ncart(B.l[b]), nc = ncart(B.l[c]), nd = ncart(B.l[d]);
    int nroots = (l1 + l2 + l3 + l4) / 2 + 1, L12 = l1 + l2, L34 = l3 + l4;
    const double *A = B.xyz + 3 * B.cen[s1], *Bc = B.xyz + 3 * B.cen[s2];
    const double *C = B.xyz + 3 * B.cen[s3], *D = B.xyz + 3 * B.cen[s4];
    double AB[3], CD[3], ab2 = 0, cd2 = 0, *tmp;
    int ntot = n1 * n2 * n3 * n4, i, j, k, l, r, x;
    static __thread double G[MAXR][3][LT][LT];
    init_binom();
    if (nroots > MAXR) return -1;
    for (x = 0; x < 3; ++x) {
        AB[x] = A[x] - Bc[x];
        CD[x] = C[x] - D[x];
        ab2 += AB[x] * AB[x];
        cd2 += CD[x] * CD[x];
    }
    tmp = calloc(ntot, sizeof(double));
    for (i = B.poff[s1]; i < B.poff[s1 + 1]; ++i)
        for (j = B.poff[s2]; j < B.poff[s2 + 1]; ++j) {
            double ea = B.al[i], eb = B.al[j], p = ea + eb, s12 = exp(-ea * eb * ab2 / p);
            double P[3], PA[3];
            for (x = 0; x < 3; ++x) {
                P[x] = (ea * A[x] + eb * Bc[x]) / p;
                PA[x] = P[x] - A[x];
            }
            for (k = B.poff[s3]; k < B.poff[s3 + 1]; ++k)
                for (l = B.poff[s4]; l < B.poff[s4 + 1]; ++l) {
                    double ec = B.al[k], ed = B.al[l], q = ec + ed, s34 = exp(-ec * ed * cd2 / q);
                    double Qv[3], QC[3], PQ[3], pq2 = 0, pqs = p + q, sr, T;
                    double rt[MAXR], wt[MAXR];
                    int ia, ib, ic, id, kc;
                    sr = SR * s12 * s34 / (p * q * sqrt(pqs));
                    if (sr < 1e-15) continue;
                    sr *= B.co[i] * B.co[j] * B.co[k] * B.co[l];
                    for (x = 0; x < 3; ++x) {
                        Qv[x] = (ec * C[x] + ed * D[x]) / q;
                        QC[x] = Qv[x] - C[x];
                        PQ[x] = P[x] - Qv[x];
                        pq2 += PQ[x] * PQ[x];
                    }
                    T = pq2 * p * q / pqs;
                    patref_rys(nroots, T, rt, wt);
                    for (r = 0; r < nroots; ++r) {
                        double f = rt[r] / pqs, B00 = 0.5 * f;
                        double B1 = (0.5 - B00 * q) / p, B1p = (0.5 - B00 * p) / q;
                        for (x = 0; x < 3; ++x)
                            rys_vrr(G[r][x], L12, L34, B00, B1, B1p, PA[x] - q * PQ[x] * f,
                                    QC[x] + p * PQ[x] * f);
                    }
                    kc = 0;
                    for (ia = 0; ia < n1; ++ia)
                        for (ib = 0; ib < n2; ++ib)
                            for (ic = 0; ic < n3; ++ic)
                                for (id = 0; id < n4; ++id, ++kc) {
                                    int e1[3], e2[3], e3[3], e4[3];
                                    double s = 0.0;
                                    comp(l1, ia, e1, e1 + 1, e1 + 2);
                                    comp(l2, ib, e2, e2 + 1, e2 + 2);
                                    comp(l3, ic, e3, e3 + 1, e3 + 2);
                                    comp(l4, id, e4, e4 + 1, e4 + 2);
                                    for (r = 0; r < nroots; ++r)
                                        s += rys_shift(AB[0], CD[0], G[r][0], e1[0], e2[0], e3[0], e4[0]) *
                                             rys_shift(AB[1], CD[1], G[r][1], e1[1], e2[1], e3[1], e4[1]) *
                                             rys_shift(AB[2], CD[2], G[r][2], e1[2], e2[2], e3[2], e4[2]) * wt[r];
                                    tmp[kc] += s * sr;
                                }
                }
        }
    /* back to the requested order, with the component factors */
    for (i = 0; i < na; ++i)
        for (j = 0; j < nb; ++j)
            for (k = 0; k < nc; ++k)
                for (l = 0; l < nd; ++l) {
                    int i1 = sw12 ? j : i, i2 = sw12 ? i : j, i3 = sw34 ? l : k, i4 = sw34 ? k : l;
                    double v = tmp[((i1 * n2 + i2) * n3 + i3) * n4 + i4];
                    out[((i * nb + j) * nc + k) * nd + l] =
                        v * comp_norm(B.l[a], i) * comp_norm(B.l[b], j) * comp_norm(B.l[c], k) *
                        comp_norm(B.l[d], l);
                }
    free(tmp);
    return 0;
}

/* --------------------------------------------------------- G build */
/* Digest one canonical integral (i>=j, i>=k>=l, l<=j when i==k) into G with
 * the scatter of scfaux.c:446-495 (RHF, P = half density, G = 2J - K) or
 * scfaux.c:575-650 (UHF). */
static void digest(int uhf, double val, int i, int j, int k, int l, const double *PA,
                   const double *PB, double *GA, double *GB)
{
    int ii = i * (i + 1) / 2, ij = ii + j, ik = ii + k, il = ii + l, kl = k * (k + 1) / 2 + l;
    int jk = j > k ? j * (j + 1) / 2 + k : k * (k + 1) / 2 + j;
    int jl = j > l ? j * (j + 1) / 2 + l : l * (l + 1) / 2 + j;
    if (!uhf) {
        double da = val * 2.0 * PA[ij], db = val * 2.0 * PA[kl];
        double sjl = val * PA[ik], sjk = val * PA[il], sik = val * PA[jl], sil = val * PA[jk];
        if (k != l) {
            db += db;
            GA[ik] -= sik;
            if (i != j && j >= k) GA[jk] -= sjk;
        }
        GA[il] -= sil;
        GA[ij] += db;
        if (i != j && j >= l) GA[jl] -= sjl;
        if (ij != kl) {
            if (i != j) da += da;
            if (j <= k) {
                GA[jk] -= sjk;
                if (i != j && i <= k) GA[ik] -= sik;
                if (k != l && j <= l) GA[jl] -= sjl;
            }
            GA[kl] += da;
        }
    } else {
        double da = val * (PA[ij] + PB[ij]), db = val * (PA[kl] + PB[kl]);
        double sjlA = val * PA[ik], sjkA = val * PA[il], sikA = val * PA[jl], silA = val * PA[jk];
        double sjlB = val * PB[ik], sjkB = val * PB[il], sikB = val * PB[jl], silB = val * PB[jk];
        if (k != l) {
            db += db;
            GA[ik] -= sikA; GB[ik] -= sikB;
            if (i != j && j >= k) { GA[jk] -= sjkA; GB[jk] -= sjkB; }
        }
        GA[il] -= silA; GA[ij] += db;
        GB[il] -= silB; GB[ij] += db;
        if (i != j && j >= l) { GA[jl] -= sjlA; GB[jl] -= sjlB; }
        if (ij != kl) {
            if (i != j) da += da;
            if (j <= k) {
                GA[jk] -= sjkA; GB[jk] -= sjkB;
                if (i != j && i <= k) { GA[ik] -= sikA; GB[ik] -= sikB; }
                if (k != l && j <= l) { GA[jl] -= sjlA; GB[jl] -= sjlB; }
            }
            GA[kl] += da; GB[kl] += da;
        }
    }
}

/* Direct G build over the reference's quartet enumeration
 * (twoints.c:228-404: ish >= start, jsh <= ish, ksh <= ish, lsh <= ksh and the
 * function-level restriction of twoints.c:316-337), keeping integrals with
 * |v| > 1e-14 (twoints.c:375).  Accumulates into GA/GB (the caller zeroes,
 * rhfscf.c:26-28).  Returns the number of integrals digested.  Worker threads
 * take outer shells from a shared counter and keep private G copies. */
typedef struct {
    int uhf, start, no2;
    const double *PA, *PB;
    double *ga, *gb;
    long long count;
} GJob;

static int g_next;
static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;

static void gmat_shell(GJob *J, int ish, double *blk)
{
    int jsh, ksh, lsh;
    if (!B.nst[ish]) return;
    for (jsh = 0; jsh <= ish; ++jsh) {
        if (!B.nst[jsh]) continue;
        for (ksh = 0; ksh <= ish; ++ksh) {
            if (!B.nst[ksh]) continue;
            for (lsh = 0; lsh <= ksh; ++lsh) {
                int a, bb, c, d, nb, nc, nd;
                if (!B.nst[lsh]) continue;
                patref_eri_block(ish, jsh, ksh, lsh, blk);
                nb = B.nst[jsh]; nc = B.nst[ksh]; nd = B.nst[lsh];
                for (a = 0; a < B.nst[ish]; ++a)
                    for (bb = 0; bb < nb; ++bb)
                        for (c = 0; c < nc; ++c)
                            for (d = 0; d < nd; ++d) {
                                int ir = B.off[ish] + a, jr = B.off[jsh] + bb;
                                int kr = B.off[ksh] + c, lr = B.off[lsh] + d;
                                double v;
                                if (jr > ir || kr > ir || lr > kr || (ir == kr && lr > jr)) continue;
                                v = blk[((a * nb + bb) * nc + c) * nd + d];
                                if (fabs(v) > 1e-14) {
                                    digest(J->uhf, v, ir, jr, kr, lr, J->PA, J->PB, J->ga, J->gb);
                                    ++J->count;
                                }
                            }
            }
        }
    }
}

static void *gmat_worker(void *arg)
{
    GJob *J = (GJob *)arg;
    double *blk = malloc(sizeof(double) * 28 * 28 * 28 * 28);
    for (;;) {
        int ish;
        pthread_mutex_lock(&g_lock);
        ish = g_next--;
        pthread_mutex_unlock(&g_lock);
        if (ish < J->start) break;
        gmat_shell(J, ish, blk);
    }
    free(blk);
    return NULL;
}

long long patref_gmat(int uhf, const double *PA, const double *PB, double *GA, double *GB, int start)
{
    int n = 0, s, t, nth;
    long long total = 0;
    GJob jobs[64];
    pthread_t th[64];
    const char *env = getenv("PATREF_THREADS");
    nth = env ? atoi(env) : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nth < 1) nth = 1;
    if (nth > 64) nth = 64;
    for (s = 0; s < B.nsh; ++s) n += B.nst[s];
    g_next = B.nsh - 1;
    for (t = 0; t < nth; ++t) {
        jobs[t].uhf = uhf; jobs[t].start = start; jobs[t].no2 = n * (n + 1) / 2;
        jobs[t].PA = PA; jobs[t].PB = PB; jobs[t].count = 0;
        jobs[t].ga = calloc(jobs[t].no2, sizeof(double));
        jobs[t].gb = calloc(jobs[t].no2, sizeof(double));
        pthread_create(&th[t], NULL, gmat_worker, &jobs[t]);
    }
    for (t = 0; t < nth; ++t) {
        int k;
        pthread_join(th[t], NULL);
        for (k = 0; k < jobs[t].no2; ++k) {
            GA[k] += jobs[t].ga[k];
            if (uhf) GB[k] += jobs[t].gb[k];
        }
        total += jobs[t].count;
        free(jobs[t].ga); free(jobs[t].gb);
    }
    return total;
}

/* ------------------------------------------------------ MD one-body */
/* mdd.c:3-43: E^{ij}_t for i <= l1, j <= l2 with 1/(2p) and PA, PB */
#define EL (MAXLS + 2)
static void md_e(double E[EL][EL][2 * EL + 1], double h, double pa, double pb, int l1, int l2)
{
    int i, j, t;
    memset(E, 0, sizeof(double) * EL * EL * (2 * EL + 1));
    E[0][0][0] = 1.0;
    for (j = 0; j < l2; ++j)
        for (t = 0; t <= j + 1; ++t) {
            double v = pb * (t <= j ? E[0][j][t] : 0.0) + (t + 1 <= j ? (t + 1) * E[0][j][t + 1] : 0.0);
            if (t > 0) v += h * E[0][j][t - 1];
            E[0][j + 1][t] = v;
        }
    for (i = 0; i < l1; ++i)
        for (j = 0; j <= l2; ++j)
            for (t = 0; t <= i + j + 1; ++t) {
                double v = pa * (t <= i + j ? E[i][j][t] : 0.0) +
                           (t + 1 <= i + j ? (t + 1) * E[i][j][t + 1] : 0.0);
                if (t > 0) v += h * E[i][j][t - 1];
                E[i + 1][j][t] = v;
            }
}

/* R_{tuv} of mdr.c:37-2163 (there unrolled, here the recursion
 * R^n_{t+1,u,v} = t R^{n+1}_{t-1,u,v} + X R^{n+1}_{t,u,v}), scaled by
 * sr (-2w)^n F_n(T) at the base. */
#define RL (2 * MAXLS + 3)
static void md_r(double R[RL][RL][RL], double sr, double T, double w, const double *pq, int L)
{
    static __thread double Rn[RL + 1][RL][RL][RL];
    double F[RL + 2];
    int n, t, u, v;
    patref_boys(L, T, F);
    for (n = 0; n <= L; ++n) Rn[n][0][0][0] = sr * pow(-2.0 * w, n) * F[n];
    for (n = L - 1; n >= 0; --n) {
        int top = L - n;
        for (t = 0; t <= top; ++t)
            for (u = 0; u <= top - t; ++u)
                for (v = 0; v <= top - t - u; ++v) {
                    double val;
                    if (t + u + v == 0) continue;
                    if (t > 0) {
                        val = pq[0] * Rn[n + 1][t - 1][u][v];
                        if (t > 1) val += (t - 1) * Rn[n + 1][t - 2][u][v];
                    } else if (u > 0) {
                        val = pq[1] * Rn[n + 1][t][u - 1][v];
                        if (u > 1) val += (u - 1) * Rn[n + 1][t][u - 2][v];
                    } else {
                        val = pq[2] * Rn[n + 1][t][u][v - 1];
                        if (v > 1) val += (v - 1) * Rn[n + 1][t][u][v - 2];
                    }
                    Rn[n][t][u][v] = val;
                }
    }
    for (t = 0; t <= L; ++t)
        for (u = 0; u <= L - t; ++u)
            for (v = 0; v <= L - t - u; ++v) R[t][u][v] = Rn[0][t][u][v];
}

/* oneints.c:12-234: S, T and H = T + V (all centres but skipcen) by MD. */
void patref_oneints(double *S, double *Tm, double *H)
{
    const double piterm = 5.5683279968317079;   /* pi^(3/2) */
    int ish, jsh;
    static double E[3][EL][EL][2 * EL + 1];
    static double R[RL][RL][RL], Rs[RL][RL][RL];
    for (ish = 0; ish < B.nsh; ++ish) {
        for (jsh = 0; jsh <= ish; ++jsh) {
            int l1 = B.l[ish], l2 = B.l[jsh], n1 = B.nst[ish], n2 = B.nst[jsh], L = l1 + l2;
            const double *A = B.xyz + 3 * B.cen[ish], *Bv = B.xyz + 3 * B.cen[jsh];
            double ab2 = 0, sv[441], tv[441], vv[441];
            int i, j, x, ia, ib, kc;
            if (!n1 || !n2) continue;
            for (x = 0; x < 3; ++x) ab2 += (A[x] - Bv[x]) * (A[x] - Bv[x]);
            memset(sv, 0, sizeof sv); memset(tv, 0, sizeof tv); memset(vv, 0, sizeof vv);
            for (i = B.poff[ish]; i < B.poff[ish + 1]; ++i)
                for (j = B.poff[jsh]; j < B.poff[jsh + 1]; ++j) {
                    double ea = B.al[i], eb = B.al[j], p = ea + eb, c12 = B.co[i] * B.co[j];
                    double s12 = piterm * exp(-ea * eb * ab2 / p) / (p * sqrt(p)), P[3], sr;
                    int c, t, u, v;
                    for (x = 0; x < 3; ++x) {
                        P[x] = (ea * A[x] + eb * Bv[x]) / p;
                        md_e(E[x], 0.5 / p, P[x] - A[x], P[x] - Bv[x], l1 + 1, l2 + 1);
                    }
                    sr = 2.0 * s12 * sqrt(p / M_PI);
                    memset(Rs, 0, sizeof Rs);
                    for (c = 0; c < B.ncen; ++c) {
                        double pc[3];
                        if (c == B.skip) continue;
                        for (x = 0; x < 3; ++x) pc[x] = P[x] - B.xyz[3 * c + x];
                        md_r(R, sr, p * (pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2]), p, pc, L);
                        for (t = 0; t <= L; ++t)
                            for (u = 0; u <= L - t; ++u)
                                for (v = 0; v <= L - t - u; ++v) Rs[t][u][v] -= B.q[c] * R[t][u][v];
                    }
                    kc = 0;
                    for (ia = 0; ia < n1; ++ia)
                        for (ib = 0; ib < n2; ++ib, ++kc) {
                            int e1[3], e2[3];
                            double nf = c12 * comp_norm(l1, ia) * comp_norm(l2, ib), kin = 0.0, pot = 0.0;
                            comp(l1, ia, e1, e1 + 1, e1 + 2);
                            comp(l2, ib, e2, e2 + 1, e2 + 2);
                            sv[kc] += nf * s12 * E[0][e1[0]][e2[0]][0] * E[1][e1[1]][e2[1]][0] *
                                      E[2][e1[2]][e2[2]][0];
                            for (x = 0; x < 3; ++x) {
                                int a1 = e1[x], b1 = e2[x];
                                double tx = 2.0 * ea * eb * E[x][a1 + 1][b1 + 1][0], o = 1.0;
                                int y;
                                if (a1) tx -= a1 * eb * E[x][a1 - 1][b1 + 1][0];
                                if (b1) {
                                    tx -= b1 * ea * E[x][a1 + 1][b1 - 1][0];
                                    if (a1) tx += 0.5 * a1 * b1 * E[x][a1 - 1][b1 - 1][0];
                                }
                                for (y = 0; y < 3; ++y)
                                    if (y != x) o *= E[y][e1[y]][e2[y]][0];
                                kin += tx * o;
                            }
                            tv[kc] += nf * s12 * kin;
                            for (t = 0; t <= e1[0] + e2[0]; ++t)
                                for (u = 0; u <= e1[1] + e2[1]; ++u)
                                    for (v = 0; v <= e1[2] + e2[2]; ++v)
                                        pot += E[0][e1[0]][e2[0]][t] * E[1][e1[1]][e2[1]][u] *
                                               E[2][e1[2]][e2[2]][v] * Rs[t][u][v];
                            vv[kc] += nf * pot;
                        }
                }
            kc = 0;
            for (ia = 0; ia < n1; ++ia)
                for (ib = 0; ib < n2; ++ib, ++kc) {
                    int ir = B.off[ish] + ia, jr = B.off[jsh] + ib, ij;
                    if (jr > ir) continue;
                    ij = ir * (ir + 1) / 2 + jr;
                    S[ij] = sv[kc];
                    Tm[ij] = tv[kc];
                    H[ij] = tv[kc] + vv[kc];
                }
        }
    }
}

/* dpmints.c:18-199: H -= V_DPM, the attraction of every basis pair to the
 * six-Gaussian model charge at the positron centre (skipcen).  The model
 * exponents and weights are the reference's (dpmints.c:30-36). */
void patref_dpm(double *H)
{
    const double SR = 34.9868366552497250;
    const double palf[6] = {6.8505018000, 4.0491646000, 3.5941062989,
                            1.2478274000, 0.7927690989, 0.3377107978};
    const double pcof[6] = {0.0766926784, 0.1483475912, 0.0462334641,
                            0.0717376427, 0.0447149792, 0.0069678529};
    const double *Qp = B.xyz + 3 * B.skip;
    static double E[3][EL][EL][2 * EL + 1];
    static double R[RL][RL][RL];
    int ish, jsh;
    for (ish = 0; ish < B.nsh; ++ish)
        for (jsh = 0; jsh <= ish; ++jsh) {
            int l1 = B.l[ish], l2 = B.l[jsh], n1 = B.nst[ish], n2 = B.nst[jsh], L = l1 + l2;
            const double *A = B.xyz + 3 * B.cen[ish], *Bv = B.xyz + 3 * B.cen[jsh];
            double ab2 = 0, vv[441];
            int i, j, x, ia, ib, kc, g;
            if (!n1 || !n2) continue;
            for (x = 0; x < 3; ++x) ab2 += (A[x] - Bv[x]) * (A[x] - Bv[x]);
            memset(vv, 0, sizeof vv);
            for (i = B.poff[ish]; i < B.poff[ish + 1]; ++i)
                for (j = B.poff[jsh]; j < B.poff[jsh + 1]; ++j) {
                    double ea = B.al[i], eb = B.al[j], p = ea + eb, c12 = B.co[i] * B.co[j];
                    double s12 = exp(-ea * eb * ab2 / p), P[3], pq[3];
                    for (x = 0; x < 3; ++x) {
                        P[x] = (ea * A[x] + eb * Bv[x]) / p;
                        md_e(E[x], 0.5 / p, P[x] - A[x], P[x] - Bv[x], l1, l2);
                        pq[x] = P[x] - Qp[x];
                    }
                    for (g = 0; g < 6; ++g) {
                        double qx = palf[g], tx = p + qx;
                        double sr = 2.0 * c12 * pcof[g] * SR * s12 * (0.5 / p) * (1.0 / qx) / sqrt(tx);
                        double w = p * qx / tx, pq2 = pq[0] * pq[0] + pq[1] * pq[1] + pq[2] * pq[2];
                        md_r(R, sr, w * pq2, w, pq, L);
                        kc = 0;
                        for (ia = 0; ia < n1; ++ia)
                            for (ib = 0; ib < n2; ++ib, ++kc) {
                                int e1[3], e2[3], t, u, v;
                                double s = 0.0;
                                comp(l1, ia, e1, e1 + 1, e1 + 2);
                                comp(l2, ib, e2, e2 + 1, e2 + 2);
                                for (t = 0; t <= e1[0] + e2[0]; ++t)
                                    for (u = 0; u <= e1[1] + e2[1]; ++u)
                                        for (v = 0; v <= e1[2] + e2[2]; ++v)
                                            s += E[0][e1[0]][e2[0]][t] * E[1][e1[1]][e2[1]][u] *
                                                 E[2][e1[2]][e2[2]][v] * R[t][u][v];
                                vv[kc] += s * comp_norm(l1, ia) * comp_norm(l2, ib);
                            }
                    }
                }
            kc = 0;
            for (ia = 0; ia < n1; ++ia)
                for (ib = 0; ib < n2; ++ib, ++kc) {
                    int ir = B.off[ish] + ia, jr = B.off[jsh] + ib;
                    if (jr > ir) continue;
                    H[ir * (ir + 1) / 2 + jr] -= vv[kc];
                }
        }
}

/* basis.c:174-195 over centre pairs with a nonzero charge product (a q=0
 * ghost on the positron makes the reference's sum 0/0). */
double patref_enuc(void)
{
    int i, j;
    double s = 0.0;
    for (i = 0; i < B.ncen; ++i)
        for (j = i + 1; j < B.ncen; ++j) {
            double qq = B.q[i] * B.q[j], r2 = 0.0;
            int x;
            if (qq == 0.0) continue;
            for (x = 0; x < 3; ++x) r2 += (B.xyz[3 * i + x] - B.xyz[3 * j + x]) * (B.xyz[3 * i + x] - B.xyz[3 * j + x]);
            s += qq / sqrt(r2);
        }
    return s;
}
