// smcrt_render.cu -- the SDF voxel render (render_sub, src/sdfs/sdf_base.f90:302-346):
// the minimum over all regions of the scene's signed distance at every voxel of a
// samples(1) x samples(2) x samples(3) grid, stored FP32 in Fortran order (i fastest).
//
// Compiled without FMA contraction, so the FP64 evaluation follows the CPU
// restatement operation for operation.  One thread per voxel, consecutive threads
// on consecutive i, so each warp writes 128 contiguous bytes of the image.
#include "smcrt_launch.h"

namespace smcrt {

namespace {

struct RenderGrid {
    long long n[3];
    double ns[3];  // nint(samples / 2), sdf_base.f90:320
    double w[3];   // extent / ns, sdf_base.f90:322
};

// Voxel (i, j, k), 1-based, sits at ((i - ns1) w1, (j - ns2) w2, (k - ns3) w3),
// sdf_base.f90:326-331.  The coordinates are formed in FP64 as the reference's
// real(wp) arithmetic does; an FP32 render rounds the point, then evaluates.
template <class R>
__global__ void __launch_bounds__(256) k_render(const __grid_constant__ SceneT<R> sc, const RenderGrid g,
                                                float* __restrict__ img) {
    const long long total = g.n[0] * g.n[1] * g.n[2];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < total; v += stride) {
        const long long i = v % g.n[0];
        const long long jk = v / g.n[0];
        const long long j = jk % g.n[1];
        const long long k = jk / g.n[1];
        const double x = ((double)(i + 1) - g.ns[0]) * g.w[0];
        const double y = ((double)(j + 1) - g.ns[1]) * g.w[1];
        const double z = ((double)(k + 1) - g.ns[2]) * g.w[2];
        const V3<R> p{(R)x, (R)y, (R)z};
        // minval(ds), sdf_base.f90:332-336
        R d = eval_region(sc, 0, p);
        for (int r = 1; r < sc.nregions; ++r) {
            const R e = eval_region(sc, r, p);
            d = e < d ? e : d;
        }
        img[v] = (float)d;
    }
}

template <class R>
cudaError_t render_t(const smcrt_scene* scene, const RenderGrid& g, float* d_img, int nsm, cudaStream_t s) {
    SceneT<R> sc;
    fill_scene(sc, scene);
    const long long total = g.n[0] * g.n[1] * g.n[2];
    const long long want = (total + 255) / 256;
    const long long cap = 16LL * nsm;  // a few resident CTAs per SM, grid-stride beyond
    const int blocks = (int)(want < cap ? want : cap);
    k_render<R><<<blocks, 256, 0, s>>>(sc, g, d_img);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_render(int precision, const smcrt_scene* scene, const int samples[3], const double extent[3],
                          float* d_img, int nsm, cudaStream_t s) {
    RenderGrid g;
    for (int a = 0; a < 3; ++a) {
        g.n[a] = samples[a];
        // nint rounds half away from zero: nint(n / 2) = (n + 1) / 2 for n >= 1
        g.ns[a] = (double)((samples[a] + 1) / 2);
        g.w[a] = extent[a] / g.ns[a];
    }
    if (g.n[0] * g.n[1] * g.n[2] == 0) return cudaSuccess;
    return precision == SMCRT_FP64 ? render_t<double>(scene, g, d_img, nsm, s)
                                   : render_t<float>(scene, g, d_img, nsm, s);
}

}  // namespace smcrt
