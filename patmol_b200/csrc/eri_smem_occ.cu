// eri_smem_occ.cu -- instantiations of the occupancy-hinted FP64 form of the
// shared-memory team kernel (eri_smem.cuh, kernel variant 5) for every class
// of eri_classes.inc where shared memory leaves room for it.
#include "eri_smem.cuh"

namespace pg {
#define PG_CLASS(la, lb, lc, ld) \
    template cudaError_t launch_smem_occ<la, lb, lc, ld>(const EriArgs &, cudaStream_t, int);
#include "eri_classes.inc"
#undef PG_CLASS
}  // namespace pg
