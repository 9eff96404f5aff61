// smcrt_kernels.cu -- one kernel variant per build: SMCRT_R (float|double),
// SMCRT_TAG (f32|f64), SMCRT_K (smcrt_kernel_kind).  Compiled six times so the
// variants build in parallel.
#include "smcrt_launch.h"

#if !defined(SMCRT_R) || !defined(SMCRT_TAG) || !defined(SMCRT_K)
#error "define SMCRT_R, SMCRT_TAG and SMCRT_K"
#endif

#define SMCRT_CAT_(a, b, c) a##_##b##_##c
#define SMCRT_CAT(a, b, c) SMCRT_CAT_(a, b, c)

namespace smcrt {

// smem: dynamic shared memory of the launch (the privatized detector bins).
cudaError_t SMCRT_CAT(launch, SMCRT_TAG, SMCRT_K)(const Params<SMCRT_R>& P, const Buffers& B, bool replay, int blocks,
                                                   int block, cudaStream_t s) {
    const size_t smem = sizeof(unsigned) * (size_t)P.sbins;
    if (replay) transport_kernel<SMCRT_R, SMCRT_K, true><<<blocks, block, smem, s>>>(P, B);
    else transport_kernel<SMCRT_R, SMCRT_K, false><<<blocks, block, smem, s>>>(P, B);
    return cudaGetLastError();
}

cudaError_t SMCRT_CAT(occupancy, SMCRT_TAG, SMCRT_K)(int block, size_t smem, int* per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, transport_kernel<SMCRT_R, SMCRT_K, false>, block,
                                                         smem);
}

}  // namespace smcrt
