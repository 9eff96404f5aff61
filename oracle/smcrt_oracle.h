/*
 * smcrt_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * C ABI of the CPU oracle: a C++17 restatement of signedMCRT's photon-packet
 * transport path, used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline as the checker.  Nothing in the product links or calls it.
 * Scene, grid, source and detector inputs reuse the product's flattened structs
 * from include/smcrt.h so both sides are fed identical data.
 */
#ifndef SMCRT_ORACLE_H
#define SMCRT_ORACLE_H

#include <stdint.h>
#include "../include/smcrt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_policy {
    int32_t precision;      /* SMCRT_FP32 / SMCRT_FP64 arithmetic of the transport */
    int32_t ref_dda;        /* 1: update_pos/update_voxels snapping DDA (inttau2.f90:213-441)
                               0: integer-stepping DDA (the GPU's) */
    int32_t crossing_f64;   /* 1: normal + Fresnel + reflect/refract in FP64 (the GPU's FP32 path) */
    int32_t tally_f32;      /* 1: accumulate jmean in FP32 like the reference (iarray.f90:12) */
    int32_t threads;        /* OpenMP threads; 0 = all */
    int32_t near_surface_f64;/* 1: the GPU's FP32 kernels' rule -- a sweep within 2 eps of a
                               surface, and every sweep after a crossing step, in FP64 */
    double eps;             /* surface epsilon (reference 1e-8) */
    double delta;           /* voxel snap (reference 1e-8, inttau2.f90:239) */
    double normal_h;        /* calcNormal step (reference 1e-6) */
    int64_t max_trace_steps;/* sphere-trace step cap per tauint2 (0 = 1,000,000) */
} oracle_policy;

int32_t oracle_run(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* src,
                   const smcrt_detector* dets, int32_t ndet, int32_t kernel, int32_t end_early,
                   const oracle_policy* pol, int64_t first, int64_t count, uint64_t seed,
                   uint32_t instance, const double* uniforms, const int64_t* offsets,
                   double* jmean, double* det_bins, smcrt_stats* stats,
                   smcrt_packet_state* states, double* jmean2);

/* jmean2 (nxg*nyg*nzg or NULL): per voxel, the sum over packets of the square of
 * the packet's own tally in that voxel (all its segments merged first): the
 * history-based second moment of the fluence tally. */
int64_t oracle_detector_bins(const smcrt_detector* dets, int32_t ndet);

/* Perturbation Monte Carlo (likelihood-ratio) reference gradient of
 * L = sum_v w[v] jmean[v] + sum_b h[b] bins[b] over packets [0, nphotons) of the
 * pathlength kernel (src/kernelsMod.f90:265-321) with respect to each region
 * group's (mua, mus, g): the sum over packets of C * d log p(path), C the packet's
 * contribution to L.  w: nxg*nyg*nzg voxel weights; h: detector bin weights or
 * NULL; region_group[r] in -1..ngroups-1 (ngroups <= 16).  grad: 3*ngroups + 1
 * doubles, [d/d mua..., d/d mus..., d/d g..., L]. */
int32_t oracle_adjoint(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* src,
                       const smcrt_detector* dets, int32_t ndet, const oracle_policy* pol,
                       int64_t nphotons, uint64_t seed, const double* w, const double* h,
                       const int32_t* region_group, int32_t ngroups, double* grad);

/* intersectPlane / intersectCircle (src/geometryMod.f90:217-270), the geometry of
 * the circle detector: 1 on a hit, 0 otherwise; *t the ray parameter. */
int32_t oracle_intersect_plane(const double* n, const double* p0, const double* l0, const double* l,
                               double* t);
int32_t oracle_intersect_circle(const double* n, const double* p0, double radius, const double* l0,
                                const double* l, double* t);

int32_t oracle_eval_sdf(const smcrt_scene* scene, int32_t precision, const double* pts,
                        int64_t npts, double* out);
/* render_sub (src/sdfs/sdf_base.f90:302-346): min over regions at every voxel,
 * FP32, Fortran order; samples[3] voxels, extent[3] half-widths. */
int32_t oracle_render(const smcrt_scene* scene, int32_t precision, const int32_t* samples,
                      const double* extent, float* image);
int32_t oracle_calc_normal(const smcrt_scene* scene, int32_t region0, double h,
                           const double* pts, int64_t npts, double* out_xyz);
int32_t oracle_fresnel(int32_t precision, const double* I, const double* N, const double* n1,
                       const double* n2, int64_t n, double* R);
int32_t oracle_reflect_refract(int32_t precision, const double* I, const double* N,
                               const double* n1, const double* n2, const double* u, int64_t n,
                               double* I_out, int32_t* reflected);
int32_t oracle_scatter_dir(int32_t precision, const double* dir_in, const double* g,
                           const double* u, int64_t n, double* dir_out);
int32_t oracle_philox(const uint32_t* key2, const uint32_t* ctr4, int64_t n, uint32_t* out4);
/* Emits npk packets (ids first..) and reports launch position/direction/layer (1-based). */
int32_t oracle_emit(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* src,
                    int32_t precision, int64_t first, int64_t npk, uint64_t seed,
                    double* pos, double* dir, int32_t* layer);
/* Detector hit test + bin of one hit (record_hit_1D/2D); returns global bin or -1. */
int64_t oracle_detector_bin(const smcrt_detector* dets, int32_t ndet, int32_t det,
                            const double* pos, const double* dir, double value, int32_t layer1);
int32_t oracle_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
