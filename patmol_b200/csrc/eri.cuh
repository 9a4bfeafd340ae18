// eri.cuh -- interfaces between the host orchestration and the shell-quartet
// kernels of eri.cu.
#pragma once
#include "common.cuh"

namespace pg {

enum EriMode : int {
    MODE_EXPORT = 0,   // write every Cartesian integral of each quartet
    MODE_RHF = 1,      // A += contributions of G = 2J[P] - K[P]  (P = half density)
    MODE_UHF = 2,      // A0/A1 += contributions of G_a = J[Pa+Pb] - K[Pa], G_b likewise
    MODE_JK = 3,       // A0 += J[P] part, A1 += K[P] part
};

// Shell pairs, structure of arrays.  The first shell of a pair has the
// larger angular momentum (the orientation twoints.c:249-266 uses).
struct PairDev {
    const int *sa, *sb;          // shell indices
    const int *fa, *fb;          // first basis function of each shell
    const double *ax, *ay, *az;  // centre of the first shell
    const double *abx, *aby, *abz;  // A - B
    const int *pstart, *pnum;    // primitive-pair range
};

// Primitive pairs: p = a + b, P, K = c_a c_b exp(-ab/p |AB|^2) / p and the
// same without the contraction coefficients (for the primitive cut).
struct PrimDev {
    const double *p, *px, *py, *pz, *K, *cut;
};

struct EriArgs {
    PairDev pr;
    PrimDev pp;
    const int2 *quart;      // (bra pair, ket pair), bra class >= ket class
    long long nquart;
    int mode;
    int swap;               // 1: quart[] holds (ket pair, bra pair) of this kernel's class
    int n;                  // basis functions
    const double *D0, *D1;  // full n x n densities
    double *A0, *A1;        // n x n accumulators
    double *out;            // export buffer
    const long long *out_off;
    const double *rys_coef;
    double prim_cut;        // skip primitive quartets whose coefficient-free
                            // prefactor is below this (1e-15 = twoints.c:110)
    int *err;               // device error word (0 = ok)
};

// Launch the kernel of class (la lb | lc ld) on `stream`.  Returns a CUDA
// error code (cudaSuccess on success).
// variant 0: the lane-per-ket-component team kernel (eri_kernel.cuh, every
// class); 1: the register-only kernel (eri_reg.cuh, the classes of
// eri_reg_classes.inc); 2: the shared-memory team kernel (eri_smem.cuh,
// every class).
cudaError_t launch_eri_class(int la, int lb, int lc, int ld, const EriArgs &a, cudaStream_t stream,
                             int num_sms, int variant = 0);
bool eri_has_variant(int la, int lb, int lc, int ld, int variant);

cudaError_t upload_rys_constants(const RysConst &rc);

}  // namespace pg
