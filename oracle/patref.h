/*
 * patref.h -- CPU restatement of the Patmol SCF hot path (test
 * infrastructure: the checker for the GPU library, never shipped in it).
 *
 * Every routine restates the reference's algorithm in plain C and cites
 * the reference file:line it follows.  Integer index work is exact; the
 * floating-point work is FP64 except the Rys roots, which are computed in
 * __float128 from the Boys moments (the reference uses polynomial fits for
 * n <= 5 and a long-double moment method for n > 5, rys.c:245-323,
 * 328-2214), so the restatement's ERIs are at least as accurate as the
 * reference's.
 */
#ifndef PATREF_H
#define PATREF_H
#ifdef __cplusplus
extern "C" {
#endif

/* Basis snapshot, the data the reference reads through shells()/centers():
 * per shell l, centre, first function, Cartesian component count (0 for the
 * DPM shells), primitive range [poff[s], poff[s+1]) into al/co (normalised
 * coefficients, shell.c:21); per centre charge and xyz.  skipcen is the
 * centre left out of V (oneints.c:51-53) and carrying the DPM potential. */
void patref_set_basis(int nshell, const int *l, const int *cen, const int *off,
                      const int *nst, const int *poff, const double *al,
                      const double *co, int ncen, const double *q,
                      const double *xyz, int skipcen);

void patref_boys(int m, double T, double *F);                 /* mdr.c:6-35 */
int patref_rys(int n, double T, double *x, double *w);        /* rys.c:2217-2244 */
int patref_eri_block(int a, int b, int c, int d, double *out); /* twoints.c:23-186 */
long long patref_gmat(int uhf, const double *PA, const double *PB,
                      double *GA, double *GB, int start);      /* scfaux.c:429-714 */
void patref_oneints(double *S, double *T, double *H);         /* oneints.c:139-234 */
void patref_dpm(double *H);                                   /* dpmints.c:121-199 */
double patref_enuc(void);                                     /* basis.c:174-195 */

#ifdef __cplusplus
}
#endif
#endif
