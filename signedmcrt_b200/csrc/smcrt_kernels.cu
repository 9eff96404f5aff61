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

// Dynamic shared memory of a launch: the CTA's packet slots, then the
// privatized detector bins.  The kernel needs more than the default 48 KiB
// opt-in limit, set once per kernel.  Scenes whose primitives carry no
// modifiers run the instantiation compiled without the modifier code
// (MODS = false); replays always run the general one.
template <bool REPLAY, bool MODS = true>
static cudaError_t allow_smem() {
    static const cudaError_t e = cudaFuncSetAttribute(transport_kernel<SMCRT_R, SMCRT_K, REPLAY, false, false, MODS>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)(slots_bytes<SMCRT_R>() + sizeof(unsigned) * kMaxSharedBins));
    return e;
}

cudaError_t SMCRT_CAT(launch, SMCRT_TAG, SMCRT_K)(const Params<SMCRT_R>& P, const Buffers& B, bool replay, int blocks,
                                                   int block, cudaStream_t s) {
    if (block != kBlock) return cudaErrorInvalidConfiguration;
    const size_t smem = slots_bytes<SMCRT_R>() + sizeof(unsigned) * (size_t)P.sbins;
    const bool mods = P.sc.has_mods != 0;
    cudaError_t e = replay ? allow_smem<true>() : mods ? allow_smem<false>() : allow_smem<false, false>();
    if (e != cudaSuccess) return e;
    if (replay) transport_kernel<SMCRT_R, SMCRT_K, true><<<blocks, kBlock, smem, s>>>(P, B);
    else if (mods) transport_kernel<SMCRT_R, SMCRT_K, false><<<blocks, kBlock, smem, s>>>(P, B);
    else transport_kernel<SMCRT_R, SMCRT_K, false, false, false, false><<<blocks, kBlock, smem, s>>>(P, B);
    return cudaGetLastError();
}

// Batch launches (pathlength and weight kernels): instances sharing the scene
// geometry; the per-instance tables are in device memory behind P.
cudaError_t SMCRT_CAT(launch_batch, SMCRT_TAG, SMCRT_K)(const Params<SMCRT_R>& P, const Buffers& B, int blocks,
                                                         cudaStream_t s) {
#if SMCRT_K == 2
    (void)P; (void)B; (void)blocks; (void)s;
    return cudaErrorNotSupported;
#else
    static const cudaError_t attr = cudaFuncSetAttribute(transport_kernel<SMCRT_R, SMCRT_K, false, true>,
                                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                         (int)slots_bytes<SMCRT_R>());
    static const cudaError_t attr0 =
        cudaFuncSetAttribute(transport_kernel<SMCRT_R, SMCRT_K, false, true, false, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)slots_bytes<SMCRT_R>());
    if (attr != cudaSuccess) return attr;
    if (attr0 != cudaSuccess) return attr0;
    if (P.sc.has_mods)
        transport_kernel<SMCRT_R, SMCRT_K, false, true><<<blocks, kBlock, slots_bytes<SMCRT_R>(), s>>>(P, B);
    else
        transport_kernel<SMCRT_R, SMCRT_K, false, true, false, false>
            <<<blocks, kBlock, slots_bytes<SMCRT_R>(), s>>>(P, B);
    return cudaGetLastError();
#endif
}

// Adjoint launches: FP32 pathlength transport only.
cudaError_t SMCRT_CAT(launch_adjoint, SMCRT_TAG, SMCRT_K)(const Params<SMCRT_R>& P, const Buffers& B, int blocks,
                                                           cudaStream_t s) {
#if SMCRT_K != 0
    (void)P; (void)B; (void)blocks; (void)s;
    return cudaErrorNotSupported;
#else
    if (sizeof(SMCRT_R) != 4) return cudaErrorNotSupported;
    static const cudaError_t attr = cudaFuncSetAttribute(transport_kernel<SMCRT_R, 0, false, false, true>,
                                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                         (int)slots_bytes<SMCRT_R>());
    static const cudaError_t attr0 =
        cudaFuncSetAttribute(transport_kernel<SMCRT_R, 0, false, false, true, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)slots_bytes<SMCRT_R>());
    if (attr != cudaSuccess) return attr;
    if (attr0 != cudaSuccess) return attr0;
    if (blocks == 0) return cudaSuccess;
    if (P.sc.has_mods)
        transport_kernel<SMCRT_R, 0, false, false, true><<<blocks, kBlock, slots_bytes<SMCRT_R>(), s>>>(P, B);
    else
        transport_kernel<SMCRT_R, 0, false, false, true, false><<<blocks, kBlock, slots_bytes<SMCRT_R>(), s>>>(P, B);
    return cudaGetLastError();
#endif
}

cudaError_t SMCRT_CAT(occupancy, SMCRT_TAG, SMCRT_K)(int block, size_t sbins_bytes, int* per_sm) {
    if (block != kBlock) return cudaErrorInvalidConfiguration;
    cudaError_t e = allow_smem<false>();
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, transport_kernel<SMCRT_R, SMCRT_K, false>, kBlock,
                                                         slots_bytes<SMCRT_R>() + sbins_bytes);
}

}  // namespace smcrt
