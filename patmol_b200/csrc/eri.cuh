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
    const int2 *quart;      // list mode: (bra pair, ket pair), bra class >= ket class
    long long nquart;       // work items of this launch
    // implicit mode (no list): item qi is quartet k = qi*nranks + rank of the
    // class's bra x ket pair space -- pairs u0+i, v0+j with (i, j) = (k / nv,
    // k % nv), or the triangle j <= i when bra and ket are the same class --
    // kept when tau_lo <= Q_u Q_v < tau_hi and its largest shell index is at
    // least start_shell.
    int implicit;
    int u0, nu, v0, nv, same, rank, nranks, start_shell;
    // compacted mode (implicit and klist set): item qi is the quartet
    // klist[qi] = bra pair | ket pair << 32 (global pair indices), already
    // screened and partitioned; no window test
    const unsigned long long *klist;
    const double *Q;
    double tau_lo, tau_hi;
    int mode;
    int swap;               // 1: quart[] holds (ket pair, bra pair) of this kernel's class
    int n;                  // basis functions
    const double *D0, *D1;  // full n x n densities
    double *A0, *A1;        // n x n accumulators
    double *out;            // export buffer
    const long long *out_off;
    const double *rys_coef;
    int single_prim;        // 1: every shell pair has one primitive pair
    double prim_cut;        // skip primitive quartets whose coefficient-free
                            // prefactor is below this (1e-15 = twoints.c:110)
    int *err;               // device error word (0 = ok)
    // one-primitive handles: per pair 16 doubles in one 128-byte line -- p,
    // P (3), K, the coefficient-free prefactor, A (3), A - B (3), then the
    // first functions fa | fb << 32 and the shells sa | sb << 32 as 64-bit
    // integers (read by the warp kernel)
    const double *ppk;
    int det;                // 1: A0/A1 are fixed-point accumulators (acc_add)
    // device work count: with nq_dev set, the launch runs *nq_dev items (a
    // count an earlier kernel on the stream wrote; nquart is then only the
    // launch's upper bound), the last ones of [0, nquart) when from_end is set
    const unsigned long long *nq_dev;
    int from_end;
};

// Launch the kernel of class (la lb | lc ld) on `stream`.  Returns a CUDA
// error code (cudaSuccess on success).
// variant 0: the lane-per-ket-component team kernel (eri_kernel.cuh, every
// class); 1: the register-only kernel (eri_reg.cuh, the classes of
// eri_reg_classes.inc); 2: the shared-memory team kernel (eri_smem.cuh,
// every class); 3 and 4: the FP32 forms of 2 and 0 (mixed precision; 4
// takes one density set and runs as 3 for UHF); 5: the occupancy-hinted
// FP64 form of 2 (the classes whose shared memory leaves room for it);
// 6 and 7: the warp-synchronous kernel (eri_warp.cuh) in FP64 and FP32, for
// the classes of eri_warp_classes.inc on one-primitive handles (RHF and JK;
// UHF, export and contracted handles run 0 and 3 instead).
cudaError_t launch_eri_class(int la, int lb, int lc, int ld, const EriArgs &a, cudaStream_t stream,
                             int num_sms, int variant = 0);
bool eri_has_variant(int la, int lb, int lc, int ld, int variant);

cudaError_t upload_rys_constants(const RysConst &rc);

#ifdef __CUDACC__
// Fixed-point accumulation (det = 1).  Each element of the accumulator is a
// signed fixed-point number with 60 fraction bits held in two 64-bit
// counters: word 1 counts units of 2^-28, word 0 units of 2^-60 (each addend
// of word 0 lies in [-2^31, 2^31], so 2^32 additions fit; both words add as
// two's complement integers).  A contribution is rounded once to the 2^-60
// grid and added with integer arithmetic, which is exact and associative:
// the accumulated value, and G, do not depend on the order in which threads
// add.  Rounding to integers uses the 1.5 * 2^52 shift (the sum's low
// mantissa bits are the rounded integer).  Contributions must stay below
// 2^23 in magnitude; a larger or non-finite one sets *err, and the
// finishing step then writes NaN.  det = 0: a plain FP64 atomic add.
constexpr double kFixHi = 268435456.0;            // 2^28
constexpr double kFixLo = 4294967296.0;           // 2^32
constexpr double kFixShift = 6755399441055744.0;  // 1.5 * 2^52
__device__ __forceinline__ void acc_add(double *A, size_t idx, double v, int det, int *err)
{
    if (!det) {
        atomicAdd(A + idx, v);
        return;
    }
    if (!(fabs(v) < 8388608.0)) {      // 2^23, also NaN
        if (err) atomicOr(err, 1);
        return;
    }
    unsigned long long *U = reinterpret_cast<unsigned long long *>(A) + 2 * idx;
    const double sc = v * kFixHi;                 // |sc| < 2^51
    const double t = sc + kFixShift;
    const long long hi = __double_as_longlong(t) - __double_as_longlong(kFixShift);
    const double r = sc - (t - kFixShift);        // exact, |r| <= 1/2
    const long long lo = __double_as_longlong(fma(r, kFixLo, kFixShift)) - __double_as_longlong(kFixShift);
    atomicAdd(U, (unsigned long long)lo);
    atomicAdd(U + 1, (unsigned long long)hi);
}

// Value of a fixed-point element (signed words lo, hi) as a double, rounded once.
__device__ __forceinline__ double fix_value(long long lo, long long hi)
{
    const long long h = hi + (lo >> 32);          // arithmetic shift: floor(lo / 2^32)
    return (double)h * (1.0 / kFixHi) + (double)(lo & 0xffffffffll) * (1.0 / (kFixHi * kFixLo));
}

// Sum of two fixed-point elements as a double, rounded once.
__device__ __forceinline__ double fix_sum(const unsigned long long *x, const unsigned long long *y)
{
    return fix_value((long long)x[0] + (long long)y[0], (long long)x[1] + (long long)y[1]);
}

// Number of work items of a launch and the first one (see nq_dev).
__device__ __forceinline__ long long eri_work_count(const EriArgs &a)
{
    return a.nq_dev ? (long long)*a.nq_dev : a.nquart;
}
__device__ __forceinline__ long long eri_work_first(const EriArgs &a, long long nq)
{
    return (a.nq_dev && a.from_end) ? a.nquart - nq : 0;
}

// Work item qi -> (bra pair u, ket pair v) in this kernel's orientation;
// false when the item is screened out.
__device__ __forceinline__ bool eri_quartet_at(const EriArgs &a, long long qi, int &u, int &v)
{
    int ub, vk;
    if (!a.implicit) {
        const int2 q = a.quart[qi];
        ub = q.x;
        vk = q.y;
    } else if (a.klist) {
        const unsigned long long e = __ldg(a.klist + qi);
        ub = (int)(unsigned)(e & 0xffffffffull);
        vk = (int)(unsigned)(e >> 32);
    } else {
        const long long k = qi * a.nranks + a.rank;
        long long i, j;
        if (a.same) {
            i = (long long)((sqrt(8.0 * (double)k + 1.0) - 1.0) * 0.5);
            while (i * (i + 1) / 2 > k) --i;
            while ((i + 1) * (i + 2) / 2 <= k) ++i;
            j = k - i * (i + 1) / 2;
            if (i >= a.nu) return false;
        } else {
            i = k / a.nv;
            j = k - i * a.nv;
            if (i >= a.nu) return false;
        }
        ub = a.u0 + (int)i;
        vk = a.v0 + (int)j;
        const double b = __ldg(a.Q + ub) * __ldg(a.Q + vk);
        if (!(b >= a.tau_lo && b < a.tau_hi)) return false;
        if (a.start_shell > 0 &&
            max(max(a.pr.sa[ub], a.pr.sb[ub]), max(a.pr.sa[vk], a.pr.sb[vk])) < a.start_shell)
            return false;
    }
    u = a.swap ? vk : ub;
    v = a.swap ? ub : vk;
    return true;
}
#endif

}  // namespace pg
