// eri_smem_all.cu -- instantiations of the shared-memory team kernel
// (eri_smem.cuh) for every class of eri_classes.inc, in FP64 and in FP32.
#include "eri_smem.cuh"

namespace pg {
#define PG_CLASS(la, lb, lc, ld)                                                                \
    template cudaError_t launch_smem<la, lb, lc, ld, double>(const EriArgs &, cudaStream_t, int); \
    template cudaError_t launch_smem<la, lb, lc, ld, float>(const EriArgs &, cudaStream_t, int);
#include "eri_classes.inc"
#undef PG_CLASS
}  // namespace pg
