// smcrt_launch.h -- host-side entry points of the separately compiled kernel
// variants (one translation unit per transport precision x kernel kind, built
// from smcrt_kernels.cu with -DSMCRT_R/-DSMCRT_TAG/-DSMCRT_K).
#pragma once

#include <vector>

#include "smcrt_transport.cuh"

namespace smcrt {

#define SMCRT_DECL_VARIANT(R, TAG, K)                                                                       \
    cudaError_t launch_##TAG##_##K(const Params<R>& P, const Buffers& B, bool replay, int blocks, int block, \
                                   cudaStream_t s);                                                       \
    cudaError_t occupancy_##TAG##_##K(int block, size_t sbins_bytes, int* per_sm);                   \
    cudaError_t priv_cells_##TAG##_##K(int sbins, int* cells);                                            \
    cudaError_t launch_batch_##TAG##_##K(const Params<R>& P, const Buffers& B, int blocks, cudaStream_t s);   \
    cudaError_t launch_adjoint_##TAG##_##K(const Params<R>& P, const Buffers& B, int blocks, cudaStream_t s);

SMCRT_DECL_VARIANT(float, f32, 0)
SMCRT_DECL_VARIANT(float, f32, 1)
SMCRT_DECL_VARIANT(float, f32, 2)
SMCRT_DECL_VARIANT(double, f64, 0)
SMCRT_DECL_VARIANT(double, f64, 1)
SMCRT_DECL_VARIANT(double, f64, 2)
#undef SMCRT_DECL_VARIANT

// Sums `ncopies` fluence-grid copies into `out` and zeroes them (smcrt_api.cu).
cudaError_t reduce_tally_copies(double* out, double* copies, int ncopies, long long ncell, int nsm, cudaStream_t s);

// Device-function probes (smcrt_probes.cu).
cudaError_t probe_eval_sdf(int precision, const smcrt_scene* scene, const double* d_pts, long long n, double* d_out);
cudaError_t probe_normal(const smcrt_scene* scene, int region, double h, const double* d_pts, long long n,
                         double* d_out);
cudaError_t probe_fresnel(int precision, const double* I, const double* N, const double* n1, const double* n2,
                          const double* u, long long n, double* R_out, double* I_out, int* refl);
cudaError_t probe_scatter(int precision, const double* dir, const double* g, const double* u, long long n,
                          double* out);
cudaError_t probe_philox(const uint32_t* key, const uint32_t* ctr, long long n, uint32_t* out);
template <class R>
cudaError_t probe_emit(const Params<R>& P, long long first, long long n, double* pos, double* dir, int* layer);

// SDF voxel render into a device image of samples[0]*samples[1]*samples[2]
// floats, Fortran order (smcrt_render.cu).
cudaError_t launch_render(int precision, const smcrt_scene* scene, const int samples[3], const double extent[3],
                          float* d_img, int nsm, cudaStream_t s);

// Scene conversion shared by the API and the probes: the parameter-block tables
// (scenes of at most kMaxRegions regions / kMaxPrims primitives), and the
// device-memory tables of any scene with a bounding sphere per region and the
// cull margin.
template <class R>
void fill_scene(SceneT<R>& d, const smcrt_scene* s);
bool region_bound(const smcrt_scene* s, int r, double c[3], double* rad);
// Whether every region's SDF is an exact Euclidean distance under a rigid
// transform (the nearest-region cache needs 1-Lipschitz regions), and the
// margin covering the rounding of its test in precision `bytes` (4 or 8).
bool cache_policy(const smcrt_scene* s, const smcrt_grid* grid, int bytes, double* margin);
template <class R>
void scene_tables(const smcrt_scene* s, const smcrt_grid* grid, std::vector<DPrim<R>>& prims,
                  std::vector<DRegion<R>>& regions, std::vector<R>& bounds, R* margin);

}  // namespace smcrt
