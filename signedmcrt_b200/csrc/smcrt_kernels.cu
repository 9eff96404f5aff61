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

// Dynamic shared memory of a launch: the CTA's packet slots and work-queue
// rings, then the privatized detector bins.  The kernel needs more than the
// default 48 KiB, an opt-in that is a property of the function on the CURRENT
// device, so it is set before every launch (a host-side call of a few
// microseconds against launches of milliseconds) rather than once per process:
// a process may launch on several GPUs.  Scenes whose primitives carry no
// modifiers run the instantiation compiled without the modifier code
// (MODS = false); replays always run the general one; scenes held in device
// memory run the BIG instantiation.
template <class K>
static cudaError_t allow_smem(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t SMCRT_CAT(launch, SMCRT_TAG, SMCRT_K)(const Params<SMCRT_R>& P, const Buffers& B, bool replay, int blocks,
                                                   int block, cudaStream_t s) {
    if (block != kBlock) return cudaErrorInvalidConfiguration;
    const size_t smem = slots_bytes<SMCRT_R>() + priv_offset(P.sbins) + 8 * (size_t)P.priv_n;
    const bool mods = P.sc.has_mods != 0;
    cudaError_t e;
    if (P.var_tab) {  // second-moment run: the instantiation with the voxel-score tables
        if (replay || P.gsc.prim) return cudaErrorNotSupported;
        auto k = transport_kernel<SMCRT_R, SMCRT_K, false, false, false, true, false, true>;
        if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
        k<<<blocks, kBlock, smem, s>>>(P, B);
    } else if (P.gsc.prim) {  // a scene in device memory (replays included)
        if (replay) {
            auto k = transport_kernel<SMCRT_R, SMCRT_K, true, false, false, true, true>;
            if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
            k<<<blocks, kBlock, smem, s>>>(P, B);
        } else {
            auto k = transport_kernel<SMCRT_R, SMCRT_K, false, false, false, true, true>;
            if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
            k<<<blocks, kBlock, smem, s>>>(P, B);
        }
    } else if (replay) {
        auto k = transport_kernel<SMCRT_R, SMCRT_K, true>;
        if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
        k<<<blocks, kBlock, smem, s>>>(P, B);
    } else if (mods) {
        auto k = transport_kernel<SMCRT_R, SMCRT_K, false>;
        if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
        k<<<blocks, kBlock, smem, s>>>(P, B);
    } else {
        auto k = transport_kernel<SMCRT_R, SMCRT_K, false, false, false, false>;
        if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
        k<<<blocks, kBlock, smem, s>>>(P, B);
    }
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
    const size_t smem = slots_bytes<SMCRT_R>();
    cudaError_t e;
    if (P.sc.has_mods) {
        auto k = transport_kernel<SMCRT_R, SMCRT_K, false, true>;
        if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
        k<<<blocks, kBlock, smem, s>>>(P, B);
    } else {
        auto k = transport_kernel<SMCRT_R, SMCRT_K, false, true, false, false>;
        if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
        k<<<blocks, kBlock, smem, s>>>(P, B);
    }
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
    if (blocks == 0) return cudaSuccess;
    const size_t smem = slots_bytes<SMCRT_R, true>();
    cudaError_t e;
    if (P.sc.has_mods) {
        auto k = transport_kernel<SMCRT_R, 0, false, false, true>;
        if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
        k<<<blocks, kBlock, smem, s>>>(P, B);
    } else {
        auto k = transport_kernel<SMCRT_R, 0, false, false, true, false>;
        if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
        k<<<blocks, kBlock, smem, s>>>(P, B);
    }
    return cudaGetLastError();
#endif
}

// Cells of a privatised fluence sub-box that fit beside the slots and `sbins`
// shared detector bins in one CTA of the plain kernel on the current device.
cudaError_t SMCRT_CAT(priv_cells, SMCRT_TAG, SMCRT_K)(int sbins, int* cells) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes a;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, transport_kernel<SMCRT_R, SMCRT_K, false, false, false, false>);
    if (e != cudaSuccess) return e;
    const long long room =
        (long long)optin - (long long)a.sharedSizeBytes - (long long)(slots_bytes<SMCRT_R>() + priv_offset(sbins));
    *cells = room > 0 ? (int)(room / 8) : 0;
    return cudaSuccess;
}

cudaError_t SMCRT_CAT(occupancy, SMCRT_TAG, SMCRT_K)(int block, size_t sbins_bytes, int* per_sm) {
    if (block != kBlock) return cudaErrorInvalidConfiguration;
    auto k = transport_kernel<SMCRT_R, SMCRT_K, false>;
    const size_t smem = slots_bytes<SMCRT_R>() + sbins_bytes;
    cudaError_t e = allow_smem(k, smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, kBlock, smem);
}

}  // namespace smcrt
