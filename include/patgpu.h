/*
 * patgpu.h -- C ABI of libpatgpu.so, the B200 (sm_100a) implementation of
 * Patmol's SCF hot path: two-electron integrals over shell quartets (Rys
 * quadrature) fused with their digestion into the G matrix, and the
 * distributed-positron-model / one-electron integrals.
 *
 * Two layers:
 *
 *  1. Drop-in entry points with the reference's exact signatures.  A
 *     program built from the reference's host sources links these instead
 *     of twoints.c, dpmints.c and the two G builds of scfaux.c.  They read
 *     the basis through the reference's accessors (shells(), centers(),
 *     number_of_shells(), ... basis.h:16-50), which the host program
 *     provides.  Matrices are packed lower triangles, row-major
 *     (ij = i(i+1)/2 + j, scfaux.c:452-456); P is the RHF half density.
 *
 *  2. Explicit entry points (patgpu_*) taking plain arrays, used by the
 *     drop-in layer, the Python host mirror and the tests.  Every one
 *     returns 0 on success or a negative PATGPU_E* code; the message of the
 *     last failure on the calling thread is patgpu_error_message().
 *
 * No entry point has a CPU fallback: without a usable CUDA device they fail
 * with PATGPU_ENODEV.
 */
#ifndef PATGPU_H
#define PATGPU_H
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- drop-in */
/* The reference's ERI file handle (erifs.h:14-18).  The GPU library keeps
 * integral-direct state keyed by the handle's address and writes no files:
 * after two_electron_ints, tfiles->nfiles is 0. */
#ifndef _ERIFS_H_
typedef struct {
    int rank, nproc, nfiles;
    int *numints;
    char *basename;
} ERIFS;
#endif

/* Replaces two_electron_ints (twoints.h:14, twoints.c:188-418): snapshots the
 * current basis (shells with nst == 0 contribute nothing), builds shell
 * pairs, Schwarz bounds and the screened quartet list of every shell
 * quartet whose largest shell index is >= start, and binds them to tfiles. */
void two_electron_ints(ERIFS *tfiles, int start);

/* Replaces rhf_form_gmatrix (scfaux.h:22-23, scfaux.c:429-552):
 * Gmat += 2 J[P] - K[P] over the quartets bound to tfiles. */
void rhf_form_gmatrix(const ERIFS *tfiles, const double *Pmat, double *Gmat);

/* Replaces uhf_form_gmatrix (scfaux.h:24-26, scfaux.c:555-714):
 * GmatA += J[PA+PB] - K[PA], GmatB += J[PA+PB] - K[PB]. */
void uhf_form_gmatrix(const ERIFS *tfiles, const double *PmatA, const double *PmatB,
                      double *GmatA, double *GmatB);

/* Replaces dpm_ints (dpmints.h:12, dpmints.c:121-199): hmat -= V_DPM, the
 * six-Gaussian model potential centred on centre skip_center(). */
void dpm_ints(double *hmat);

/* Replaces one_electron_ints (oneints.h:10, oneints.c:139-234):
 * S, T and H = T + V (all centres but skip_center()). */
void one_electron_ints(double *Smat, double *Tmat, double *Hmat);

/* Replaces clean_ERIFS (erifs.h:28, erifs.c:68-81): frees the device state
 * bound to e, then runs the host program's own file clean-up and frees e
 * through clean_ERIFS_files, the reference's clean_ERIFS compiled under that
 * name (-Dclean_ERIFS=clean_ERIFS_files on erifs.c).  A host without it
 * keeps e allocated. */
void clean_ERIFS(ERIFS *e);

/* Replaces momints (momints.h:11, momints.c:88-188): writes MOMINTS.DAT in
 * the working directory with the reference's records -- per shell pair
 * (ish >= jsh) and component pair (j <= i), int i, int j, the three dipole
 * and six quadrupole integrals -- computed on the GPU. */
void momints(void);

/* ------------------------------------------------------------- explicit */
typedef struct patgpu_basis *patgpu_handle;

enum {
    PATGPU_OK = 0,
    PATGPU_EINVAL = -1,      /* bad argument */
    PATGPU_ENODEV = -2,      /* no CUDA device */
    PATGPU_ECUDA = -3,       /* a CUDA call failed */
    PATGPU_EUNSUPPORTED = -4,/* angular momentum above f */
    PATGPU_ENOMEM = -5,
    PATGPU_ESTATE = -6,      /* call order (e.g. no quartets built) */
};

int patgpu_last_error(void);
const char *patgpu_error_message(void);

/* Basis snapshot.  Per shell: l, centre, first basis function, Cartesian
 * component count (0 = contributes nothing, as the reference's DPM shells),
 * primitive range [prim_off[s], prim_off[s+1]) into alpha/coef; coef holds
 * the normalised contraction coefficients (what shells() returns after
 * normalize_shell, shell.c:26-56).  Per centre charge and xyz (bohr).
 * skipcen is left out of V and carries the DPM potential.  schwarz_tau:
 * quartets with Q_ab Q_cd < tau are skipped (0 disables screening).
 * Builds pairs and Schwarz bounds on the current CUDA device; every later
 * call on the handle must run with that device current (PATGPU_ESTATE
 * otherwise).  One process may drive several devices, one handle each. */
int patgpu_basis_create(int nshell, const int *l, const int *cen, const int *off, const int *nst,
                        const int *prim_off, const double *alpha, const double *coef, int ncen,
                        const double *charge, const double *xyz, int skipcen, double schwarz_tau,
                        patgpu_handle *out);
/* The same, owning from the start only the quartets patgpu_set_quartets
 * would select (start_shell, rank, nranks): one quartet-list build and one
 * tuning pass instead of two. */
int patgpu_basis_create_quartets(int nshell, const int *l, const int *cen, const int *off, const int *nst,
                                 const int *prim_off, const double *alpha, const double *coef, int ncen,
                                 const double *charge, const double *xyz, int skipcen, double schwarz_tau,
                                 int start_shell, int rank, int nranks, patgpu_handle *out);
int patgpu_basis_destroy(patgpu_handle h);

/* Which quartets this handle owns: those whose largest shell index is
 * >= start_shell (the reference's `start`, twoints.c:228), and of those
 * every nranks-th of each class starting at rank (static split across
 * GPUs).  Rebuilds the quartet list. */
int patgpu_set_quartets(patgpu_handle h, int start_shell, int rank, int nranks);

/* Host-buffer Fock builds (packed lower triangles; outputs accumulate). */
int patgpu_rhf_gmatrix(patgpu_handle h, const double *P, double *G);
int patgpu_uhf_gmatrix(patgpu_handle h, const double *PA, const double *PB, double *GA, double *GB);
/* J[P] and K[P] separately (packed; accumulate). */
int patgpu_jk(patgpu_handle h, const double *P, double *J, double *K);

/* No counterpart in the reference (its G build is a serial, hence
 * deterministic, scatter: scfaux.c:446-495).  on = 1 (the default; the
 * environment variable PATGPU_DETERMINISTIC=0 changes the default for new
 * handles): every J/K contribution is rounded once to a fixed-point grid of
 * 2^-60 and summed with 64-bit integer adds, which are exact and
 * order-independent, so G is bitwise identical from run to run and across
 * any split of the quartets over GPUs.  The accumulator then holds n x n
 * elements of 16 bytes (two 64-bit integers).  on = 0: FP64 atomic adds,
 * n x n doubles, last bits depend on the order the GPU's threads add in. */
int patgpu_set_deterministic(patgpu_handle h, int on);
/* Bytes of the n x n accumulator that patgpu_rhf_accumulate_device fills:
 * 16 n^2 with deterministic accumulation, 8 n^2 without. */
int patgpu_accumulator_bytes(patgpu_handle h, size_t *bytes);

/* Device-resident Fock build: dP and dG are device pointers to packed
 * triangles; dG is overwritten (not accumulated).  stream is the
 * cudaStream_t to enqueue on, used as given (NULL = the legacy default
 * stream).  Enqueues only; the caller synchronises. */
int patgpu_rhf_gmatrix_device(patgpu_handle h, const double *dP, double *dG, void *stream);
/* Same, leaving the unsymmetrised n x n accumulator in dA (G = A + A^T,
 * patgpu_accumulator_bytes(h) bytes), for callers that reduce partial
 * results across GPUs before finishing: sum the partials elementwise, as
 * doubles without deterministic accumulation, as 64-bit integers (wrapping)
 * with it, then call patgpu_finish_gmatrix_device on the sum. */
int patgpu_rhf_accumulate_device(patgpu_handle h, const double *dP, double *dA, void *stream);
int patgpu_finish_gmatrix_device(patgpu_handle h, const double *dA, double *dG, void *stream);

/* No counterpart in the reference.  The same device-resident RHF Fock build
 * as patgpu_rhf_gmatrix_device, for callers that must not allocate GPU
 * memory once they are running: a solver embedded in a host program that
 * owns all device memory through its own pool, or code on a path where a
 * cudaMalloc would synchronise the device or fail.  Its two n x n working
 * matrices (the density, and the accumulator at up to 16 bytes an element)
 * live in a fixed 6 MiB array compiled into the library (every GPU that
 * loads the library holds it until the process exits), so the basis must
 * have at most 512 functions; larger bases are rejected with
 * PATGPU_EINVAL.  The handle itself is built beforehand by
 * patgpu_basis_create, which does allocate.  The first call on a device
 * looks up the array's device address there, so make that first call before
 * any stream capture.  All calls share the one array: calls that overlap on
 * the GPU (different streams, or different handles on one device at the
 * same time) race and give wrong G.  dP, dG and stream as for
 * patgpu_rhf_gmatrix_device; dG is overwritten. */
int patgpu_rhf_gmatrix_device_noalloc(patgpu_handle h, const double *dP, double *dG, void *stream);

/* Integrals of arbitrary shell quartets (a b | c d), nq x 4 shell indices;
 * out receives, per quartet in order, na*nb*nc*nd values indexed
 * ((ia nb + ib) nc + ic) nd + id with the reference's component order and
 * factors.  Host buffers. */
int patgpu_eri_quartets(patgpu_handle h, int nq, const int *shells4, double *out);

/* One-electron S, T, H = T + V (packed, overwritten) and H -= V_DPM. */
int patgpu_oneints(patgpu_handle h, double *S, double *T, double *H);
int patgpu_dpm(patgpu_handle h, double *H);
/* The same without a handle (no pair or quartet set-up): any of S/T/H may
 * be NULL together (then only Hdpm is formed), Hdpm may be NULL. */
int patgpu_onebody(int nshell, const int *l, const int *cen, const int *off, const int *nst,
                   const int *prim_off, const double *alpha, const double *coef, int ncen,
                   const double *charge, const double *xyz, int skipcen, double *S, double *T,
                   double *H, double *Hdpm);

/* Moment integrals about the coordinate origin, replacing the integrals of
 * momints (momints.h:11, momints.c:13-188): dip[3][no2] (x, y, z) and
 * quad[6][no2] (xx, xy, xz, yy, yz, zz), packed lower triangles with the
 * reference's component order and factors, overwritten.  No handle. */
int patgpu_moments(int nshell, const int *l, const int *cen, const int *off, const int *nst, const int *prim_off,
                   const double *alpha, const double *coef, int ncen, const double *xyz, double *dip, double *quad);

/* Nuclear gradient of the closed-shell SCF energy (no counterpart in the
 * reference, which has no gradients):
 *   E = 2 tr(P H) + tr(P G[P]) + E_nuc,  H -= V_DPM when with_dpm,
 * at a converged half density P (P = C_occ C_occ^T, packed lower triangle)
 * and its energy-weighted density W = sum_occ e_i c_i c_i^T (packed, may be
 * NULL when PATGPU_GRAD_1E is not asked for).  grad[3*ncen] (x, y, z per
 * centre, ghost and positron centres included) is overwritten with the sum
 * of the parts selected by the mask: PATGPU_GRAD_2E (derivative ERIs
 * contracted with the density products on the GPU, over this handle's
 * screened quartets -- with a rank split, only this rank's share),
 * PATGPU_GRAD_1E (overlap/Pulay, kinetic, nuclear attraction including the
 * moving charges, and DPM when with_dpm; GPU) and PATGPU_GRAD_NUC (nuclear
 * repulsion over centre pairs whose charge product is non-zero; host). */
#define PATGPU_GRAD_2E 1
#define PATGPU_GRAD_1E 2
#define PATGPU_GRAD_NUC 4
#define PATGPU_GRAD_ALL 7
int patgpu_rhf_gradient(patgpu_handle h, const double *P, const double *W, int parts, int with_dpm,
                        double *grad);
/* The open-shell form: E = sum_s [tr(P_s H) + tr(P_s G_s)/2] + E_nuc with
 * G_s = J[Pa+Pb] - K[P_s] (uhfscf.c:29-55), at converged spin densities
 * PA, PB and W_s = sum_occ e_i c_i c_i^T per spin (all packed). */
int patgpu_uhf_gradient(patgpu_handle h, const double *PA, const double *PB, const double *WA, const double *WB,
                        int parts, int with_dpm, double *grad);

/* The reference's ERI files from the GPU integrals: the record stream of
 * two_electron_ints (twoints.c:188-418) -- 16-byte ERINT records
 * (erifs.h:19-22) of every canonical function quartet with |v| > 1e-14, in
 * the reference's shell-quartet and component order, MPI rank `rank` of
 * `nproc` taking the reference's card-dealt share (twoints.c:280-288), a
 * new file after max_records records (the reference uses
 * MAXFILESIZE / 16, pconfig.h:7).  For callers that keep the reference's
 * file-reading G build (rhf_form_gmatrix in scfaux.c, e.g. in patmpi) and
 * only take the integrals from the GPU.  patgpu_write_eri_files names the
 * files prefix + rank + file number + basename, as create_filename does
 * (erifs.c:54-73); patgpu_write_eri_files_with opens them through the
 * caller's function (the reference's createERIFile, erifs.c:84-90).
 * numints[f] receives file f's record count (capacity max_files), *nfiles
 * the file count.  The drop-in two_electron_ints writes them too when
 * PATGPU_ERI_FILES=1. */
int patgpu_write_eri_files(patgpu_handle h, int start, int rank, int nproc, const char *prefix,
                           const char *basename, long long max_records, int max_files, int *numints, int *nfiles);
int patgpu_write_eri_files_with(patgpu_handle h, int start, int rank, int nproc,
                                FILE *(*open_file)(int rank, int file_no, const char *basename),
                                const char *basename, long long max_records, int max_files, int *numints,
                                int *nfiles);

/* SCF linear algebra on the GPU (the reference does it on the host:
 * spack_trans, spack_diag, form_cmatrix, form_pmatrix; rhfscf.c:36-47).
 * patgpu_scf_create takes the orthogonaliser X (host, n x nx, row-major --
 * the reference's xmat, or any X with X^T S X = 1) and the occupied-orbital
 * count, and allocates every work array once.  patgpu_scf_density takes a
 * packed Fock matrix on the device and forms F' = X^T F X, its eigenpairs
 * (cuSOLVER syevd, ascending), C = X V and the packed half density
 * P = C_occ C_occ^T on the device; optionally W = C_occ e_occ C_occ^T
 * (device, packed), the eigenvalues (host, nx) and C (host, n x nx
 * column-major, i.e. C[i + n a] is orbital a on function i).  It
 * synchronises `stream` before returning. */
typedef struct patgpu_scf_s *patgpu_scf;
int patgpu_scf_create(int n, int nx, int nocc, const double *X, patgpu_scf *out);
int patgpu_scf_destroy(patgpu_scf s);
int patgpu_scf_density(patgpu_scf s, const double *dF, double *dP, double *dW, double *eps, double *C,
                       void *stream);
/* The same with packed host buffers (F in; P and, if not NULL, W out). */
int patgpu_scf_density_host(patgpu_scf s, const double *F, double *P, double *W, double *eps, double *C);

/* Density-weighted screening (no counterpart in the reference, which
 * screens nothing at run time): with tau_dens > 0 the host-buffer builds
 * (patgpu_rhf_gmatrix, patgpu_uhf_gmatrix, patgpu_jk) skip every quartet
 * whose bound Q_ab Q_cd max(4|D_ab|, 4|D_cd|, |D_ac|, |D_ad|, |D_bc|, |D_bd|)
 * (shell-block maxima of the build's density) is below tau_dens.  Meant for
 * incremental builds G[P_n] = G[P_(n-1)] + G[P_n - P_(n-1)], whose density
 * difference shrinks as the SCF converges.  Needs the compacted lists (a
 * handle without them computes every quartet).  0 (the default) turns it
 * off.  patgpu_last_computed: quartets computed by the last host-buffer build. */
int patgpu_set_density_screening(patgpu_handle h, double tau_dens);
int patgpu_last_computed(patgpu_handle h, long long *quartets);
/* Density-weighted precision of density-screened builds (no counterpart in
 * the reference): a quartet kept by the screening whose density-weighted
 * term bound (the term bound of patgpu_set_mixed_precision times the same
 * max|D|) is below tau32 is computed in FP32 arithmetic with FP64 roots,
 * prefactors and J/K sums -- in a difference build G[P_n - P_(n-1)] the
 * density factor makes most contributions small, so their FP32 error
 * (about 1e-7 of the bound) stays far below the screening threshold's
 * scale.  0 (the default) turns it off.  The first non-zero
 * value times the FP32 kernels per class. */
int patgpu_set_density_precision(patgpu_handle h, double tau32);

/* Batches (no counterpart in the reference, which runs one molecule per
 * process): many molecules advanced in lock step.  A batch holds the
 * molecules' handles (which must outlive it and must not be used
 * elsewhere while a batch launch runs: the batch uses their work buffers)
 * and, per molecule, packed device buffers dP and dG.  patgpu_batch_launch
 * computes dG_m = G[dP_m] (RHF, overwritten) for every molecule as ONE
 * CUDA graph launch on `stream`; the graph is captured on the first launch
 * (after one plain build per molecule) and holds each molecule's class
 * launches, spread over parallel capture streams or kept on one: the first
 * capture of each graph kind (plain, density-screened) times both forms once
 * on the buffers' densities and keeps the faster.  patgpu_batch_rhf_gmatrix
 * is the host-buffer form (G_m += G[P_m]).  Mixed precision is per
 * molecule; patgpu_batch_set_mixed_precision sets it for all and drops the
 * graph.  Stats: [0] molecules, [1] quartets, [2] FP32 quartets, [3]
 * graph nodes.  Timing: nanoseconds of the last graph launch (events). */
typedef struct patgpu_batch_s *patgpu_batch;
int patgpu_batch_create(int nmol, const patgpu_handle *mols, patgpu_batch *out);
int patgpu_batch_destroy(patgpu_batch b);
int patgpu_batch_buffers(patgpu_batch b, int m, double **dP, double **dG);
int patgpu_batch_set_mixed_precision(patgpu_batch b, double tau_fp32);
/* Density screening (and density-weighted precision, tau32) of every
 * molecule's build, for incremental SCF: tau_dens > 0 makes launches use a
 * second graph holding each molecule's density filter ahead of its class
 * launches (the filtered work counts stay on the device, so the graph
 * replays whatever densities the buffers hold); 0 returns to the plain
 * graph.  The second graph copies both thresholds from host memory when it
 * starts, so they may change from one launch to the next (an SCF that
 * tightens its screening as it converges) without a new capture; change
 * them only while no launch of the batch is pending.  The first tau32 > 0
 * captures the graph once more with the FP32 sublist launches in it.
 * patgpu_batch_last_computed: quartets computed by the last launch
 * (synchronises the batch's stream). */
int patgpu_batch_set_density_screening(patgpu_batch b, double tau_dens, double tau32);
/* The same with a threshold pair per molecule (arrays of the batch's
 * molecule count; tau32 may be NULL for zeros), so that each molecule of an
 * SCF can tighten its own screening as it converges.  Screening is on when
 * any tau_dens is positive; a molecule at 0 then keeps every quartet. */
int patgpu_batch_set_density_thresholds(patgpu_batch b, const double *tau_dens, const double *tau32);
int patgpu_batch_last_computed(patgpu_batch b, long long *quartets);
int patgpu_batch_launch(patgpu_batch b, void *stream);
int patgpu_batch_rhf_gmatrix(patgpu_batch b, const double *const *P, double *const *G);
int patgpu_batch_stats(patgpu_batch b, long long *out4);
int patgpu_batch_last_timing(patgpu_batch b, double *kernel_ns);

/* Mixed precision (no counterpart in the reference, which is FP64
 * throughout): screened-in quartets whose term bound lies below tau_fp32
 * are computed with FP32 recursion, transfer and assembly, while roots,
 * weights, prefactors and every J/K product and sum stay FP64.  The term
 * bound is an upper estimate of the terms the Rys scheme sums for the
 * quartet (prefactor times, per side, (2|A-B| + share of |P-Q| +
 * sqrt((L+1)/2p))^L), not the Schwarz bound Q_ab Q_cd: distant diffuse
 * distributions have small integrals made of large cancelling root terms,
 * and FP32 rounding scales with the terms.  The absolute error per
 * integral is then about 1e-7 tau_fp32.  0 turns it off
 * (the default).  Per quartet class the library times the FP32 kernels
 * against the class's FP64 kernel on that window and keeps the fastest, so
 * a class whose window is too small to repay FP32 stays FP64 (one launch).
 * patgpu_mixed_stats returns how many quartets of this handle run in FP32.
 * The FP32 window runs over the handle's compacted quartet lists; a handle
 * without lists (not enough device memory, or PATGPU_LISTS=0) stays FP64 and
 * reports 0. */
int patgpu_set_mixed_precision(patgpu_handle h, double tau_fp32);
int patgpu_mixed_stats(patgpu_handle h, long long *n_fp32);

/* Sizes of the handle: [0] basis functions, [1] shell pairs, [2] quartets
 * owned, [3] classes with work, [4] quartets before screening. */
int patgpu_stats(patgpu_handle h, long long *out5);
/* Per class with work: l of the four shells and the quartet count. */
int patgpu_class_counts(patgpu_handle h, int max, int *l4, long long *counts);
/* Nanoseconds of the last Fock build's class kernels (CUDA events on the
 * handle's stream, first kernel start to last kernel end), and the number
 * of kernels it launched. */
int patgpu_last_timing(patgpu_handle h, double *kernel_ns, int *launches);

/* Measured dense FP64 FMA throughput of the current device (TFLOP/s), the
 * denominator of the kernels' roofline fraction. */
int patgpu_fp64_peak(double *tflops);
/* Dense FP64 matrix-instruction rate of the current GPU in TFLOP/s
 * (mma.sync m8n8k4, 8 independent accumulators per thread), to set beside
 * patgpu_fp64_peak: on sm_100a this is the only FP64 tensor-core form. */
int patgpu_dmma_peak(double *tflops);

/* Host evaluation of the Rys root tables the kernels use (no device
 * needed): x = t^2 nodes and weights of the n-point rule at T. */
int patgpu_rys_host(int n, double T, double *x, double *w);

/* Make device (index modulo the device count) current for this thread. The
 * drop-in layer calls it once with PATGPU_DEVICE or the launcher's
 * node-local rank (OMPI_COMM_WORLD_LOCAL_RANK, MPI_LOCALRANKID,
 * SLURM_LOCALID, LOCAL_RANK) when one is set. */
int patgpu_select_device(int index);

/* Drop every handle the drop-in layer created. */
void patgpu_release_all(void);

#ifdef __cplusplus
}
#endif
#endif
