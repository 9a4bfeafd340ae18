// eri.cu -- constant tables of the shell-quartet kernels and the class
// dispatcher.  The kernel template is in eri_kernel.cuh; every kernel of
// eri_kernels.inc is instantiated in its own translation unit (generated by
// the Makefile), so the 110 instantiations compile in parallel.
#include "eri_kernel.cuh"
#include "eri_reg.cuh"
#include "eri_smem.cuh"
#include "eri_warp.cuh"

namespace pg {

__constant__ RysConst c_rys;
__constant__ int c_cart[4][10];
__constant__ double c_norm[4][10];

cudaError_t upload_rys_constants(const RysConst &rc)
{
    int cart[4][10] = {};
    double nrm[4][10] = {};
    for (int l = 0; l <= 3; ++l)
        for (int k = 0; k < ncart(l); ++k) {
            cart[l][k] = kCart.e[l][k];
            int x = cart_x(l, k), y = cart_y(l, k), z = cart_z(l, k);
            nrm[l][k] = 1.0 / sqrt(dfact_odd(x) * dfact_odd(y) * dfact_odd(z));
        }
    cudaError_t e = cudaMemcpyToSymbol(c_rys, &rc, sizeof(RysConst));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_cart, cart, sizeof(cart));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_norm, nrm, sizeof(nrm));
    return e;
}

#define PG_KERNEL(la, lb, lc, ld, sw)                                                              \
    extern template cudaError_t launch_one<la, lb, lc, ld, 1>(const EriArgs &, cudaStream_t, int); \
    extern template cudaError_t launch_one<la, lb, lc, ld, 2>(const EriArgs &, cudaStream_t, int); \
    extern template cudaError_t launch_one<la, lb, lc, ld, 1, float>(const EriArgs &, cudaStream_t, int);
#include "eri_kernels.inc"
#undef PG_KERNEL

// Quartet class (LA LB | LC LD) of a list whose entries are (bra, ket) pairs;
// classes listed with swap = 1 run on the kernel of (LC LD | LA LB).
#define PG_KERNEL(la, lb, lc, ld, sw)                                                        \
    if ((sw == 0 && LA == la && LB == lb && LC == lc && LD == ld) ||                        \
        (sw == 1 && LA == lc && LB == ld && LC == la && LD == lb)) {                        \
        EriArgs b = a;                                                                       \
        b.swap = sw;                                                                         \
        if (variant == 4) return launch_one<la, lb, lc, ld, 1, float>(b, stream, num_sms);  \
        return a.mode == MODE_UHF ? launch_one<la, lb, lc, ld, 2>(b, stream, num_sms)       \
                                  : launch_one<la, lb, lc, ld, 1>(b, stream, num_sms);      \
    }

#define PG_REG(la, lb, lc, ld)                                                                    \
    extern template cudaError_t launch_reg<la, lb, lc, ld, 1>(const EriArgs &, cudaStream_t, int); \
    extern template cudaError_t launch_reg<la, lb, lc, ld, 2>(const EriArgs &, cudaStream_t, int);
#include "eri_reg_classes.inc"
#undef PG_REG

#define PG_CLASS(la, lb, lc, ld)                                                                       \
    extern template cudaError_t launch_smem<la, lb, lc, ld, double>(const EriArgs &, cudaStream_t, int); \
    extern template cudaError_t launch_smem<la, lb, lc, ld, float>(const EriArgs &, cudaStream_t, int);  \
    extern template cudaError_t launch_smem_occ<la, lb, lc, ld>(const EriArgs &, cudaStream_t, int);
#include "eri_classes.inc"
#undef PG_CLASS

#define PG_WARP(la, lb, lc, ld, sw)                                                                    \
    extern template cudaError_t launch_warp<la, lb, lc, ld, 1, double>(const EriArgs &, cudaStream_t, int); \
    extern template cudaError_t launch_warp<la, lb, lc, ld, 1, float>(const EriArgs &, cudaStream_t, int);
#include "eri_warp_classes.inc"
#undef PG_WARP

bool eri_has_variant(int LA, int LB, int LC, int LD, int variant)
{
    if (variant == 6 || variant == 7) {
#define PG_WARP(la, lb, lc, ld, sw)                                          \
        if ((sw == 0 && LA == la && LB == lb && LC == lc && LD == ld) ||    \
            (sw == 1 && LA == lc && LB == ld && LC == la && LD == lb))      \
            return true;
#include "eri_warp_classes.inc"
#undef PG_WARP
        return false;
    }
    if (variant == 0 || variant == 2 || variant == 3 || variant == 4) return true;
    if (variant == 5) {
#define PG_CLASS(la, lb, lc, ld) \
        if (LA == la && LB == lb && LC == lc && LD == ld) return SmemShape<la, lb, lc, ld, double>::HAS_OCC;
#include "eri_classes.inc"
#undef PG_CLASS
        return false;
    }
#define PG_REG(la, lb, lc, ld) \
    if (LA == la && LB == lb && LC == lc && LD == ld) return variant == 1;
#include "eri_reg_classes.inc"
#undef PG_REG
    return false;
}

cudaError_t launch_eri_class(int LA, int LB, int LC, int LD, const EriArgs &a, cudaStream_t stream,
                             int num_sms, int variant)
{
    if (variant == 4 && a.mode == MODE_UHF) variant = 3;   // the FP32 lane kernel has one density set
    if (variant == 6 || variant == 7) {
        // the warp kernels take one density set, Fock modes only and one
        // primitive pair per shell pair; elsewhere the lane kernel (FP64) or
        // the shared-memory kernel (FP32) serves
        if (a.mode != MODE_UHF && a.mode != MODE_EXPORT && a.single_prim && a.ppk) {
#define PG_WARP(la, lb, lc, ld, sw)                                                             \
    if ((sw == 0 && LA == la && LB == lb && LC == lc && LD == ld) ||                           \
        (sw == 1 && LA == lc && LB == ld && LC == la && LD == lb)) {                           \
        EriArgs b = a;                                                                          \
        b.swap = sw;                                                                            \
        return variant == 6 ? launch_warp<la, lb, lc, ld, 1, double>(b, stream, num_sms)      \
                            : launch_warp<la, lb, lc, ld, 1, float>(b, stream, num_sms);      \
    }
#include "eri_warp_classes.inc"
#undef PG_WARP
        }
        variant = variant == 6 ? 0 : 3;
    }
    if (variant == 2 || variant == 3) {
#define PG_CLASS(la, lb, lc, ld)                                                     \
    if (LA == la && LB == lb && LC == lc && LD == ld) {                             \
        EriArgs b = a;                                                                \
        b.swap = 0;                                                                   \
        return variant == 2 ? launch_smem<la, lb, lc, ld, double>(b, stream, num_sms) \
                            : launch_smem<la, lb, lc, ld, float>(b, stream, num_sms); \
    }
#include "eri_classes.inc"
#undef PG_CLASS
        return cudaErrorInvalidValue;
    }
    if (variant == 5) {
#define PG_CLASS(la, lb, lc, ld)                                      \
    if (LA == la && LB == lb && LC == lc && LD == ld) {              \
        EriArgs b = a;                                                 \
        b.swap = 0;                                                    \
        return launch_smem_occ<la, lb, lc, ld>(b, stream, num_sms);   \
    }
#include "eri_classes.inc"
#undef PG_CLASS
        return cudaErrorInvalidValue;
    }
    if (variant == 1) {
#define PG_REG(la, lb, lc, ld)                                                            \
    if (LA == la && LB == lb && LC == lc && LD == ld) {                                  \
        EriArgs b = a;                                                                     \
        b.swap = 0;                                                                        \
        return a.mode == MODE_UHF ? launch_reg<la, lb, lc, ld, 2>(b, stream, num_sms)     \
                                  : launch_reg<la, lb, lc, ld, 1>(b, stream, num_sms);    \
    }
#include "eri_reg_classes.inc"
#undef PG_REG
        return cudaErrorInvalidValue;
    }
#include "eri_kernels.inc"
    return cudaErrorInvalidValue;
}

}  // namespace pg
