/*
 * ref_harness.c -- test-infrastructure driver linked against the reference's
 * own objects (every Patmol source of Makefile.am:11-12 except patmol.c).
 * It calls only the reference's public functions and writes raw binary
 * dumps into the current directory, which must hold patin.dat (and
 * posgrid.dat for "scf" with dpm on).  Nothing in the product links this.
 *
 *   ref_harness moments         MOMINTS.DAT (the reference's momints, momints.c:88-188)
 *   ref_harness ints            S.bin T.bin H.bin (packed lower triangle),
 *                               eri.bin (ERINT records, erifs.h:19-22),
 *                               info.txt (norb nshell ncen enuc nrec)
 *   ref_harness gmat P.bin      G.bin  = rhf_form_gmatrix(P) (scfaux.c:429)
 *   ref_harness ugmat PA PB     GA.bin GB.bin = uhf_form_gmatrix (scfaux.c:555)
 *   ref_harness dpm x y z       H0.bin (T+V, positron centre skipped) and
 *                               Hdpm.bin (after dpm_ints, dpmints.c:121)
 *                               for the positron at (x,y,z)
 *   ref_harness scf             RHF/UHF SCF re-created from the public
 *                               functions (rhfscf.c:22-118, uhfscf.c:23-110),
 *                               then, if the input has dpm on, the DPM stage
 *                               of rhfscf.c:218-263 at every posgrid point,
 *                               printing the DPM total energy the reference
 *                               never writes.  E_nuc skips pairs with
 *                               q_i*q_j == 0 (basis.c:174-195 divides 0 by 0
 *                               when a ghost centre sits on the positron).
 *   ref_harness bench K         times two_electron_ints once and K calls of
 *                               rhf_form_gmatrix, prints one JSON line.
 *   ref_harness bench1 K W      the same, but each call digests only the
 *                               first ERI file (a bounded sample of the
 *                               Fock build), after W untimed calls.
 */
#include "momints.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <time.h>
#include "basis.h"
#include "oneints.h"
#include "twoints.h"
#include "dpmints.h"
#include "scfaux.h"
#include "spack_math.h"
#include "erifs.h"

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void write_bin(const char *name, const void *p, size_t bytes)
{
    FILE *f = fopen(name, "wb");
    if (!f || fwrite(p, 1, bytes, f) != bytes) {
        fprintf(stderr, "cannot write %s\n", name);
        exit(2);
    }
    fclose(f);
}

static void read_bin(const char *name, void *p, size_t bytes)
{
    FILE *f = fopen(name, "rb");
    if (!f || fread(p, 1, bytes, f) != bytes) {
        fprintf(stderr, "cannot read %s\n", name);
        exit(2);
    }
    fclose(f);
}

/* E_nuc over centre pairs with a nonzero charge product. */
static double enuc_nonzero(void)
{
    const Center *c = centers();
    int n = number_of_centers(), i, j;
    double s = 0.0;
    for (i = 0; i < n; ++i)
        for (j = i + 1; j < n; ++j) {
            double qq = c[i].q * c[j].q;
            if (qq != 0.0) s += qq / sqrt(distSqr(c[i].r, c[j].r));
        }
    return s;
}

static ERIFS *make_eris(int start, const char *base, double *secs)
{
    ERIFS *e = init_ERIFS(0, number_of_orbitals(), base);
    double t0 = now_s();
    two_electron_ints(e, start);
    if (secs) *secs = now_s() - t0;
    return e;
}

static size_t dump_eris(const ERIFS *e, const char *out)
{
    FILE *fo = fopen(out, "wb");
    size_t nrec = 0;
    int f;
    for (f = 0; f < e->nfiles; ++f) {
        FILE *fi = openERIFile(e->rank, f, e->basename);
        ERINT buf[4096];
        size_t got;
        while ((got = fread(buf, sizeof(ERINT), 4096, fi)) > 0) {
            fwrite(buf, sizeof(ERINT), got, fo);
            nrec += got;
        }
        fclose(fi);
    }
    fclose(fo);
    return nrec;
}

/* ---- SCF re-created from the public functions ------------------------- */
typedef struct {
    int n, no2, nocc_a, nocc_b, uhf, accel, maxit;
    double eps, enuc;
    double *h, *s, *t, *x, *w, *work, *fock, *ev;
    double *pa, *pa1, *pa2, *pb, *pb1, *pb2, *ga, *gb, *ca, *cb;
    ERIFS *mints;
} Scf;

static void scf_alloc(Scf *S)
{
    int n = S->n, no2 = S->no2;
    S->h = dalloc(no2); S->s = dalloc(no2); S->t = dalloc(no2);
    S->fock = dalloc(no2);
    S->x = dalloc(n * n); S->w = dalloc(n * n); S->work = dalloc(n * n);
    S->ev = dalloc(n);
    S->pa = dalloc(no2); S->pa1 = dalloc(no2); S->pa2 = dalloc(no2);
    S->pb = dalloc(no2); S->pb1 = dalloc(no2); S->pb2 = dalloc(no2);
    S->ga = dalloc(no2); S->gb = dalloc(no2);
    S->ca = dalloc(n * n); S->cb = dalloc(n * n);
    memset(S->pa1, 0, sizeof(double) * no2); memset(S->pa2, 0, sizeof(double) * no2);
    memset(S->pb1, 0, sizeof(double) * no2); memset(S->pb2, 0, sizeof(double) * no2);
}

/* rhfscf.c:433-452 */
static void scf_orth_matrix(Scf *S)
{
    int i, j, n = S->n;
    memcpy(S->fock, S->s, sizeof(double) * S->no2);
    spack_diag(n, S->fock, S->w, S->ev, S->work);
    for (i = 0; i < n; ++i) {
        if (S->ev[i] <= DBL_EPSILON) fatalError("overlap not positive definite");
        S->ev[i] = 1.0 / sqrt(S->ev[i]);
    }
    for (i = 0; i < n; ++i)
        for (j = 0; j < n; ++j) S->x[i * n + j] = S->w[i * n + j] * S->ev[j];
}

/* rhfscf.c:455-471 core-Hamiltonian guess */
static void scf_core_guess(Scf *S)
{
    memcpy(S->fock, S->h, sizeof(double) * S->no2);
    spack_trans(S->n, S->fock, S->x, S->work);
    spack_diag(S->n, S->fock, S->w, S->ev, S->work);
    form_cmatrix(S->n, S->ca, S->x, S->w);
    form_pmatrix(S->n, S->nocc_a, S->ca, S->pa);
    if (S->uhf) form_pmatrix(S->n, S->nocc_b, S->ca, S->pb);
}

static void spin_update(Scf *S, const double *g, double *c, int nocc,
                        double *p, double *p1, double *p2)
{
    int i;
    for (i = 0; i < S->no2; ++i) S->fock[i] = S->h[i] + g[i];
    spack_trans(S->n, S->fock, S->x, S->work);
    spack_diag(S->n, S->fock, S->w, S->ev, S->work);
    form_cmatrix(S->n, c, S->x, S->w);
    memcpy(p2, p1, sizeof(double) * S->no2);
    memcpy(p1, p, sizeof(double) * S->no2);
    form_pmatrix(S->n, nocc, c, p);
}

/* one iteration: rhfscf.c:22-71 (RHF) or uhfscf.c:23-78 (UHF) */
static int scf_update(Scf *S, int *iteration, double *eold, double *enrg)
{
    int i;
    double pdiff, ediff;
    ++(*iteration);
    memset(S->ga, 0, sizeof(double) * S->no2);
    memset(S->gb, 0, sizeof(double) * S->no2);
    if (!S->uhf) {
        rhf_form_gmatrix(S->mints, S->pa, S->ga);
        spin_update(S, S->ga, S->ca, S->nocc_a, S->pa, S->pa1, S->pa2);
        pdiff = pdiffNorm(S->n, S->pa, S->pa1);
        *enrg = 2.0 * calc_energy(S->n, S->pa1, S->h, S->ga);
    } else {
        uhf_form_gmatrix(S->mints, S->pa, S->pb, S->ga, S->gb);
        spin_update(S, S->ga, S->ca, S->nocc_a, S->pa, S->pa1, S->pa2);
        pdiff = pdiffNorm(S->n, S->pa, S->pa1);
        spin_update(S, S->gb, S->cb, S->nocc_b, S->pb, S->pb1, S->pb2);
        pdiff += pdiffNorm(S->n, S->pb, S->pb1);
        *enrg = calc_energy(S->n, S->pa1, S->h, S->ga) +
                calc_energy(S->n, S->pb1, S->h, S->gb);
    }
    ediff = *enrg - *eold;
    *eold = *enrg;
    if (*iteration == 1) return 0;
    if (fabs(ediff) < 10 * DBL_EPSILON) return 1;
    if (pdiff < S->eps) return 1;
    if (ediff > 0.0) {
        if (S->accel == 1) {
            for (i = 0; i < S->no2; ++i) {
                S->pa[i] = 0.5 * (S->pa1[i] + S->pa2[i]);
                S->pb[i] = 0.5 * (S->pb1[i] + S->pb2[i]);
            }
        }
        if (S->accel == 2) {
            scfAccelerator(*iteration, S->no2, S->pa, S->pa1, S->pa2);
            if (S->uhf) scfAccelerator(*iteration, S->no2, S->pb, S->pb1, S->pb2);
        }
    }
    return 0;
}

/* ---- DIIS driver (closed shell; REF_HARNESS_DIIS=1) ----------------------
 * The reference's averaging/Anderson damping (scfaux.c:64-95) stalls on many
 * random molecules.  This driver keeps every reference computation -- G from
 * rhf_form_gmatrix over the reference's own ERI files, spack_trans /
 * spack_diag / form_cmatrix / form_pmatrix, calc_energy -- and only replaces
 * the damping by Pulay's DIIS on the commutator FPS - SPF (in the
 * orthogonalised basis), so that the reference's SCF energy exists for
 * them.  Converged when |dE| < 1e-11 and max|error| < 1e-8. */
#define DIIS_MAX 8
static void unpack_full(int n, const double *p, double *f)
{
    int i, j;
    for (i = 0; i < n; ++i)
        for (j = 0; j <= i; ++j) f[i * n + j] = f[j * n + i] = p[i * (i + 1) / 2 + j];
}

static void matmul(int n, const double *a, const double *b, double *c)
{
    int i, j, k;
    memset(c, 0, sizeof(double) * n * n);
    for (i = 0; i < n; ++i)
        for (k = 0; k < n; ++k) {
            double aik = a[i * n + k];
            if (aik == 0.0) continue;
            for (j = 0; j < n; ++j) c[i * n + j] += aik * b[k * n + j];
        }
}

/* x^T a x with x = S->x (full) */
static void orth_transform(int n, const double *x, const double *a, double *out, double *tmp)
{
    int i, j, k;
    matmul(n, a, x, tmp);
    memset(out, 0, sizeof(double) * n * n);
    for (k = 0; k < n; ++k)
        for (i = 0; i < n; ++i) {
            double xki = x[k * n + i];
            if (xki == 0.0) continue;
            for (j = 0; j < n; ++j) out[i * n + j] += xki * tmp[k * n + j];
        }
}

/* Gaussian elimination with partial pivoting, m <= DIIS_MAX + 1 */
static int solve_small(int m, double *A, double *b)
{
    int i, j, k;
    for (k = 0; k < m; ++k) {
        int piv = k;
        for (i = k + 1; i < m; ++i)
            if (fabs(A[i * m + k]) > fabs(A[piv * m + k])) piv = i;
        if (fabs(A[piv * m + k]) < 1e-300) return -1;
        if (piv != k) {
            double t;
            for (j = 0; j < m; ++j) { t = A[k * m + j]; A[k * m + j] = A[piv * m + j]; A[piv * m + j] = t; }
            t = b[k]; b[k] = b[piv]; b[piv] = t;
        }
        for (i = k + 1; i < m; ++i) {
            double f = A[i * m + k] / A[k * m + k];
            for (j = k; j < m; ++j) A[i * m + j] -= f * A[k * m + j];
            b[i] -= f * b[k];
        }
    }
    for (k = m - 1; k >= 0; --k) {
        double s = b[k];
        for (j = k + 1; j < m; ++j) s -= A[k * m + j] * b[j];
        b[k] = s / A[k * m + k];
    }
    return 0;
}

static double scf_run_diis(Scf *S, int *iters)
{
    int n = S->n, no2 = S->no2, it, i, j, nh = 0, head = 0;
    double *fh[DIIS_MAX], *eh[DIIS_MAX];
    double *Pf = dalloc(n * n), *Ff = dalloc(n * n), *Sf = dalloc(n * n), *t1 = dalloc(n * n);
    double *t2 = dalloc(n * n), *err = dalloc(n * n), *fx = dalloc(no2);
    double eold = 0.0, enrg = 0.0, emax = 0.0;
    for (i = 0; i < DIIS_MAX; ++i) { fh[i] = dalloc(no2); eh[i] = dalloc(n * n); }
    unpack_full(n, S->s, Sf);
    for (it = 1; it <= S->maxit; ++it) {
        memset(S->ga, 0, sizeof(double) * no2);
        rhf_form_gmatrix(S->mints, S->pa, S->ga);
        enrg = 2.0 * calc_energy(n, S->pa, S->h, S->ga);
        for (i = 0; i < no2; ++i) fx[i] = S->h[i] + S->ga[i];
        /* error FPS - SPF in the orthogonalised basis */
        unpack_full(n, fx, Ff);
        unpack_full(n, S->pa, Pf);
        matmul(n, Ff, Pf, t1);
        matmul(n, t1, Sf, t2);
        for (i = 0; i < n; ++i)
            for (j = 0; j < n; ++j) t1[i * n + j] = t2[i * n + j] - t2[j * n + i];
        orth_transform(n, S->x, t1, err, t2);
        emax = 0.0;
        for (i = 0; i < n * n; ++i) emax = fabs(err[i]) > emax ? fabs(err[i]) : emax;
        if (it > 1 && fabs(enrg - eold) < 1e-11 && emax < 1e-8) break;
        eold = enrg;
        memcpy(fh[head], fx, sizeof(double) * no2);
        memcpy(eh[head], err, sizeof(double) * n * n);
        head = (head + 1) % DIIS_MAX;
        if (nh < DIIS_MAX) ++nh;
        if (nh > 1) {
            double B[(DIIS_MAX + 1) * (DIIS_MAX + 1)], c[DIIS_MAX + 1];
            int m = nh + 1, a, b2;
            for (a = 0; a < nh; ++a)
                for (b2 = 0; b2 < nh; ++b2) {
                    double s = 0.0;
                    for (i = 0; i < n * n; ++i) s += eh[a][i] * eh[b2][i];
                    B[a * m + b2] = s;
                }
            for (a = 0; a < nh; ++a) { B[a * m + nh] = B[nh * m + a] = -1.0; c[a] = 0.0; }
            B[nh * m + nh] = 0.0;
            c[nh] = -1.0;
            if (solve_small(m, B, c) == 0) {
                for (i = 0; i < no2; ++i) {
                    double s = 0.0;
                    for (a = 0; a < nh; ++a) s += c[a] * fh[a][i];
                    fx[i] = s;
                }
            }
        }
        /* rhfscf.c:36-47 on the extrapolated Fock matrix */
        memcpy(S->fock, fx, sizeof(double) * no2);
        spack_trans(n, S->fock, S->x, S->work);
        spack_diag(n, S->fock, S->w, S->ev, S->work);
        form_cmatrix(n, S->ca, S->x, S->w);
        form_pmatrix(n, S->nocc_a, S->ca, S->pa);
    }
    *iters = it;
    fprintf(stderr, "ref_harness: DIIS SCF %d iterations, max|FPS-SPF| %.3e\n", it, emax);
    for (i = 0; i < DIIS_MAX; ++i) { free(fh[i]); free(eh[i]); }
    free(Pf); free(Ff); free(Sf); free(t1); free(t2); free(err); free(fx);
    return enrg;
}

/* rhfscf.c:74-118: returns the final electronic energy */
static double scf_run(Scf *S, int *iters)
{
    int it = 0, done = 0;
    double eold = 0.0, enrg = 0.0;
    const char *diis = getenv("REF_HARNESS_DIIS");
    if (diis && diis[0] == '1' && !S->uhf) return scf_run_diis(S, iters);
    scf_update(S, &it, &eold, &enrg);
    it = 0;
    while (!done && it < S->maxit) done = scf_update(S, &it, &eold, &enrg);
    *iters = it;
    return enrg;
}

static int cmd_scf(void)
{
    Scf S;
    int ne = number_of_electrons(), sm = spin_multiplicity(), iters;
    double e_gs;
    memset(&S, 0, sizeof(S));
    S.n = number_of_orbitals();
    S.no2 = S.n * (S.n + 1) / 2;
    S.uhf = !((ne % 2 == 0) && sm == 1);         /* patmol.c:18 */
    S.nocc_b = S.uhf ? (ne - (sm - 1)) / 2 : ne / 2;
    S.nocc_a = S.uhf ? ne - S.nocc_b : ne / 2;
    S.accel = scf_acceleration();
    S.maxit = max_scf_iterations();
    S.eps = scf_convergence();
    if (S.eps < 10 * DBL_EPSILON * S.n * S.n) S.eps = 10 * DBL_EPSILON * S.n * S.n;
    scf_alloc(&S);
    one_electron_ints(S.s, S.t, S.h);
    S.mints = make_eris(0, "MINTS.DAT", NULL);
    S.enuc = enuc_nonzero();
    scf_orth_matrix(&S);
    scf_core_guess(&S);
    e_gs = scf_run(&S, &iters);
    write_bin("Pconv.bin", S.pa, sizeof(double) * S.no2);
    if (S.uhf) write_bin("PconvB.bin", S.pb, sizeof(double) * S.no2);
    write_bin("Hcore.bin", S.h, sizeof(double) * S.no2);
    printf("{\"kind\": \"%s\", \"e_total\": %.17g, \"e_elec\": %.17g, \"enuc\": %.17g, \"iters\": %d",
           S.uhf ? "uhf" : "rhf", e_gs + S.enuc, e_gs, S.enuc, iters);
    if (do_dpm_calculation()) {
        /* rhfscf.c:218-263 with the fixed-N dimension of the reference */
        FILE *in = openFile("posgrid.dat", "r");
        int npts, ipt, poscen = number_of_centers(), onsh = number_of_shells();
        double *pa_gs = dalloc(S.no2), *pb_gs = dalloc(S.no2);
        ERIFS *xints;
        memcpy(pa_gs, S.pa, sizeof(double) * S.no2);
        memcpy(pb_gs, S.pb, sizeof(double) * S.no2);
        xints = init_ERIFS(S.n, total_number_of_orbitals(), "XINTS.DAT");
        dpm_augment();
        if (fscanf(in, "%d", &npts) != 1) npts = 0;
        printf(", \"dpm\": [");
        for (ipt = 0; ipt < npts; ++ipt) {
            double rp[3], e1;
            int it1;
            if (fscanf(in, "%lg %lg %lg", rp, rp + 1, rp + 2) != 3) break;
            set_center_position(poscen, rp);
            one_electron_ints(S.s, S.t, S.h);
            dpm_ints(S.h);
            two_electron_ints(xints, onsh);
            S.enuc = enuc_nonzero();
            memcpy(S.pa, pa_gs, sizeof(double) * S.no2);
            memcpy(S.pb, pb_gs, sizeof(double) * S.no2);
            scf_orth_matrix(&S);
            {
                int it = 0, done = 0;
                double eold = 0.0, enrg = 0.0, efirst;
                scf_update(&S, &it, &eold, &enrg);
                efirst = enrg;
                it = 0;
                while (!done && it < S.maxit) done = scf_update(&S, &it, &eold, &enrg);
                e1 = enrg;
                it1 = it;
                printf("%s{\"pos\": [%.17g, %.17g, %.17g], \"e_total\": %.17g, \"vpol\": %.17g, \"enuc\": %.17g, \"iters\": %d, \"xints_files\": %d}",
                       ipt ? ", " : "", rp[0], rp[1], rp[2], e1 + S.enuc, e1 - efirst, S.enuc, it1,
                       xints->nfiles);
            }
        }
        printf("]");
        fclose(in);
    }
    printf("}\n");
    return 0;
}

int main(int argc, char **argv)
{
    int n, no2;
    if (argc < 2) {
        fprintf(stderr, "usage: ref_harness ints|gmat|ugmat|dpm|scf|bench ...\n");
        return 2;
    }
    init_Basis();
    n = number_of_orbitals();
    no2 = n * (n + 1) / 2;
    if (!strcmp(argv[1], "ints")) {
        double *S = dalloc(no2), *T = dalloc(no2), *H = dalloc(no2), secs;
        ERIFS *e;
        size_t nrec;
        FILE *f;
        one_electron_ints(S, T, H);
        write_bin("S.bin", S, sizeof(double) * no2);
        write_bin("T.bin", T, sizeof(double) * no2);
        write_bin("H.bin", H, sizeof(double) * no2);
        e = make_eris(0, "MINTS.DAT", &secs);
        nrec = dump_eris(e, "eri.bin");
        f = fopen("info.txt", "w");
        fprintf(f, "%d %d %d %.17g %zu %.6f\n", n, number_of_shells(), number_of_centers(),
                enuc_nonzero(), nrec, secs);
        fclose(f);
        clean_ERIFS(e);
        return 0;
    }
    if (!strcmp(argv[1], "moments")) {
        /* the reference's moment integrals (momints.c:88-188), MOMINTS.DAT */
        momints();
        return 0;
    }
    if (!strcmp(argv[1], "gmat") && argc >= 3) {
        double *P = dalloc(no2), *G = dalloc(no2);
        ERIFS *e = make_eris(0, "MINTS.DAT", NULL);
        read_bin(argv[2], P, sizeof(double) * no2);
        memset(G, 0, sizeof(double) * no2);
        rhf_form_gmatrix(e, P, G);
        write_bin("G.bin", G, sizeof(double) * no2);
        clean_ERIFS(e);
        return 0;
    }
    if (!strcmp(argv[1], "ugmat") && argc >= 4) {
        double *PA = dalloc(no2), *PB = dalloc(no2), *GA = dalloc(no2), *GB = dalloc(no2);
        ERIFS *e = make_eris(0, "MINTS.DAT", NULL);
        read_bin(argv[2], PA, sizeof(double) * no2);
        read_bin(argv[3], PB, sizeof(double) * no2);
        memset(GA, 0, sizeof(double) * no2);
        memset(GB, 0, sizeof(double) * no2);
        uhf_form_gmatrix(e, PA, PB, GA, GB);
        write_bin("GA.bin", GA, sizeof(double) * no2);
        write_bin("GB.bin", GB, sizeof(double) * no2);
        clean_ERIFS(e);
        return 0;
    }
    if (!strcmp(argv[1], "dpm") && argc >= 5) {
        double rp[3], *S = dalloc(no2), *T = dalloc(no2), *H = dalloc(no2);
        int poscen = number_of_centers();
        rp[0] = atof(argv[2]); rp[1] = atof(argv[3]); rp[2] = atof(argv[4]);
        dpm_augment();
        set_center_position(poscen, rp);
        one_electron_ints(S, T, H);
        write_bin("H0.bin", H, sizeof(double) * no2);
        dpm_ints(H);
        write_bin("Hdpm.bin", H, sizeof(double) * no2);
        return 0;
    }
    if (!strcmp(argv[1], "scf")) return cmd_scf();
    if (!strcmp(argv[1], "bench") && argc >= 3) {
        int k, K = atoi(argv[2]);
        double *P = dalloc(no2), *G = dalloc(no2), secs, t0, tg;
        ERIFS *e = make_eris(0, "MINTS.DAT", &secs);
        size_t nrec = 0;
        for (k = 0; k < e->nfiles; ++k) nrec += e->numints[k];
        for (k = 0; k < no2; ++k) P[k] = 1.0 / (1.0 + k % 7);
        t0 = now_s();
        for (k = 0; k < K; ++k) {
            memset(G, 0, sizeof(double) * no2);
            rhf_form_gmatrix(e, P, G);
        }
        tg = (now_s() - t0) / (K > 0 ? K : 1);
        printf("{\"eri_seconds\": %.6f, \"gmat_seconds_per_call\": %.6f, \"records\": %zu, \"norb\": %d, \"nshell\": %d}\n",
               secs, tg, nrec, n, number_of_shells());
        clean_ERIFS(e);
        return 0;
    }
    if (!strcmp(argv[1], "bench1") && argc >= 4) {
        int k, K = atoi(argv[2]), W = atoi(argv[3]);
        double *P = dalloc(no2), *G = dalloc(no2), secs, t0, tg;
        ERIFS *e = make_eris(0, "MINTS.DAT", &secs), view;
        size_t nrec = 0;
        for (k = 0; k < e->nfiles; ++k) nrec += e->numints[k];
        view = *e;
        view.nfiles = e->nfiles > 0 ? 1 : 0;      /* file 0 only */
        for (k = 0; k < no2; ++k) P[k] = 1.0 / (1.0 + k % 7);
        for (k = 0; k < W; ++k) {
            memset(G, 0, sizeof(double) * no2);
            rhf_form_gmatrix(&view, P, G);
        }
        t0 = now_s();
        for (k = 0; k < K; ++k) {
            memset(G, 0, sizeof(double) * no2);
            rhf_form_gmatrix(&view, P, G);
        }
        tg = (now_s() - t0) / (K > 0 ? K : 1);
        printf("{\"eri_seconds\": %.6f, \"gmat_seconds_per_call\": %.6f, \"records\": %zu, \"file_records\": %d, \"nfiles\": %d, \"norb\": %d}\n",
               secs, tg, nrec, e->nfiles ? e->numints[0] : 0, e->nfiles, n);
        clean_ERIFS(e);
        return 0;
    }
    fprintf(stderr, "unknown command %s\n", argv[1]);
    return 2;
}
