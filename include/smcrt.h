/*
 * smcrt.h -- C ABI of the B200 photon-packet transport library (libsmcrt_b200.so).
 *
 * This is the drop-in boundary for signedMCRT's per-packet transport loop.
 * signedMCRT (Fortran 2018) runs that loop inside
 *     subroutine pathlength_scatter(input_file)   src/kernelsMod.f90:165-333
 *     subroutine weight_scatter(input_file)       src/kernelsMod.f90:12-163
 *     subroutine test_kernel(input_file, end_early) src/kernelsMod.f90:335-448
 * between `setup(...)` (:236) and `finalise(...)` (:332).  The Fortran types on
 * that path (polymorphic class(sdf_base) allocatables, procedure pointers,
 * module-global state/jmean) are not C-interoperable, so the caller flattens them
 * into the plain structs below once per simulation and calls smcrt_create /
 * smcrt_run.  Every pointer is a plain host pointer unless the name says _dev.
 * No function exits or aborts the process: failures return a nonzero status and
 * smcrt_last_error() returns the message (thread-local).
 *
 * Conventions
 *  - Regions are the entries of the reference's `type(sdf) :: array(:)` in array
 *    order; array order sets priority at boundary crossings
 *    (src/inttau2.f90:131-136) and at launch (src/kernelsMod.f90:275-280).
 *    Region-valued fields here (detector.layer, packet layer) are 1-based, as in
 *    the reference (`packet%layer` is the array index).
 *  - Affine transforms use the reference's row-vector convention
 *    (src/vector_class.f90:292-304): p'_j = sum_i p_i*M[i][j] + M[3][j], i.e. the
 *    first three columns of the reference's 4x4 `transform`, stored row-major as
 *    M[4][3].  Build them exactly as the reference does (e.g. invert(translate(c))).
 *  - Fluence grids are nxg*nyg*nzg doubles in Fortran column-major order,
 *    idx = (i-1) + nxg*((j-1) + nyg*(k-1)), matching `jmean(nxg,nyg,nzg)`
 *    (src/iarray.f90:12).  Values are the raw path-length tally (not normalised;
 *    see normalise_fluence, src/writer.f90:25-50).
 */
#ifndef SMCRT_H
#define SMCRT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SMCRT_ABI_VERSION 5

/* ---- status codes -------------------------------------------------------- */
enum smcrt_status {
    SMCRT_OK = 0,
    SMCRT_ERR_ARG = 1,        /* bad argument (null pointer, size out of range) */
    SMCRT_ERR_SCENE = 2,      /* invalid scene (unknown kind, bad ranges, too large) */
    SMCRT_ERR_CUDA = 3,       /* a CUDA runtime call failed */
    SMCRT_ERR_DEVICE = 4,     /* the kernel raised a device status flag (see stats) */
    SMCRT_ERR_TIMEOUT = 5,    /* the host wait on the kernel ran out of time */
    SMCRT_ERR_NO_DEVICE = 6   /* no CUDA device visible */
};

/* ---- SDF primitives (src/sdfs/sdfs.f90:494-735) --------------------------- */
enum smcrt_prim_kind {
    SMCRT_SPHERE = 1,   /* params: [radius]                                 sdfs.f90:494-508 */
    SMCRT_BOX = 2,      /* params: [hx,hy,hz] half lengths (box_init halves) sdfs.f90:510-525 */
    SMCRT_TORUS = 3,    /* params: [oradius, iradius]                        sdfs.f90:527-542 */
    SMCRT_CYLINDER = 4, /* params: [ax,ay,az, bx,by,bz, radius]              sdfs.f90:544-581 */
    SMCRT_TRIPRISM = 5, /* params: [h1, h2]                                  sdfs.f90:583-597 */
    SMCRT_SEGMENT = 6,  /* params: [ax,ay,az, bx,by,bz] (radius fixed 0.1)   sdfs.f90:599-626 */
    SMCRT_CAPSULE = 7,  /* params: [ax,ay,az, bx,by,bz, r]                   sdfs.f90:628-648 */
    SMCRT_CONE = 8,     /* params: [ax,ay,az, bx,by,bz, ra, rb]              sdfs.f90:650-686 */
    SMCRT_EGG = 9,      /* params: [r1, r2, h]                               sdfs.f90:688-718 */
    SMCRT_PLANE = 10    /* params: [ax,ay,az] (normalised normal)            sdfs.f90:720-735 */
};

/* CSG fold of a model's children (src/sdfs/sdfModifiers.f90:412-475, eval_model
 * src/sdfs/sdf_base.f90:145-160): d = child0; d = op(d, child_i, k). */
enum smcrt_csg_op {
    SMCRT_OP_NONE = 0,
    SMCRT_OP_UNION = 1,
    SMCRT_OP_SMOOTH_UNION = 2,
    SMCRT_OP_SUBTRACTION = 3,
    SMCRT_OP_INTERSECTION = 4
};

/* SDF modifiers wrapping a primitive (src/sdfs/sdfModifiers.f90:273-375).  The
 * modifier has no transform of its own; the primitive keeps its transform.
 * (displacement takes a user function and repeat is not implemented in the
 * reference, so neither exists here.) */
enum smcrt_modifier {
    SMCRT_MOD_NONE = 0,
    SMCRT_MOD_ONION = 1,      /* [thickness]: |d| - t                 eval_onion :307-317 */
    SMCRT_MOD_REVOLUTION = 2, /* [o]: prim at (|(x,z)| - o, y, 0)      eval_revolution :290-305 */
    SMCRT_MOD_EXTRUDE = 3,    /* [h]: extrusion of the xy profile      eval_extrude :273-288 */
    SMCRT_MOD_ELONGATE = 4,   /* [sx, sy, sz]                          eval_elongate :319-335 */
    SMCRT_MOD_TWIST = 5,      /* [k]: rotation by k z about z          eval_twist :337-355 */
    SMCRT_MOD_BEND = 6        /* [k]: rotation by k x about z          eval_bend :357-375 */
};

typedef struct smcrt_prim {
    int32_t kind;          /* smcrt_prim_kind */
    int32_t nmods;         /* modifiers applied to this primitive, 0..2 */
    double transform[4][3];
    double params[8];
    int32_t mods[2];       /* smcrt_modifier, innermost first: onion(revolution(egg)) =
                              {REVOLUTION, ONION} */
    double mod_params[2][3];
} smcrt_prim;

/* One entry of the reference's sdf array: a single primitive (nprims == 1) or a
 * model (nprims > 1, folded with `op`), with its mono optical properties
 * (init_mono, src/opticalProps/opticalProperties.f90:107-125). */
typedef struct smcrt_region {
    int32_t first_prim;
    int32_t nprims;
    int32_t op;            /* smcrt_csg_op; ignored when nprims == 1 */
    int32_t layer_id;      /* the reference's sdf%layer (informational) */
    double k;              /* op parameter (smooth-union width) */
    double mus, mua, hgg, n;
} smcrt_region;

typedef struct smcrt_scene {
    int32_t nregions;
    int32_t nprims;
    const smcrt_region* regions;
    const smcrt_prim* prims;
} smcrt_scene;

/* cart_grid (src/grid.f90:14-25, init_grid :53-93): voxel counts and HALF sizes. */
typedef struct smcrt_grid {
    int32_t nxg, nyg, nzg, reserved;
    double xmax, ymax, zmax;
} smcrt_grid;

/* ---- sources (src/photon.f90) --------------------------------------------- */
enum smcrt_source_kind {
    SMCRT_SRC_POINT = 1,    /* photon.f90:290-338, 2 draws */
    SMCRT_SRC_PENCIL = 2,   /* photon.f90:464-505, 0 draws */
    SMCRT_SRC_UNIFORM = 3,  /* photon.f90:397-461, 2 draws */
    SMCRT_SRC_CIRCULAR = 4, /* photon.f90:214-287, 2 draws */
    SMCRT_SRC_ANNULUS = 5,  /* photon.f90:645-711, 2 draws (tophat) / 2 per trial (gaussian) */
    SMCRT_SRC_FOCUS = 6     /* photon.f90:340-394, 2 draws */
};
enum smcrt_annulus_type { SMCRT_ANNULUS_TOPHAT = 0, SMCRT_ANNULUS_GAUSSIAN = 1 };

typedef struct smcrt_source {
    int32_t kind;          /* smcrt_source_kind */
    int32_t annulus_type;  /* smcrt_annulus_type */
    double pos[3];         /* [source] position (photon_origin%pos) */
    double dir[3];         /* [source] direction (photon_origin%nxp..nzp) */
    double point1[3], point2[3], point3[3]; /* uniform source corners */
    double radius;         /* circular radius / annulus inner radius ("radius") */
    double radius_hi;      /* annulus outer radius ("radius_hi") */
    double beta;           /* annulus beam angle in degrees ("beta") */
    double z_inset;        /* annulus/focus start = grid zmax - z_inset; reference hard-codes 1e-8 */
} smcrt_source;

/* ---- detectors (src/detectors/detectors.f90) ------------------------------ */
enum smcrt_detector_kind {
    SMCRT_DET_CIRCLE = 1,   /* detectors.f90:74-127, nbins+1 bins, width maxval/(nbins-1) */
    SMCRT_DET_ANNULUS = 2,  /* detectors.f90:129-184, nbins+1 bins, width maxval/nbins */
    SMCRT_DET_CAMERA = 3    /* detectors.f90:186-253, (nbins+1)^2 bins, column-major */
};

typedef struct smcrt_detector {
    int32_t kind;          /* smcrt_detector_kind */
    int32_t layer;         /* 1-based region index the packet must end in */
    int32_t nbins;         /* as given in the TOML (the detector holds nbins+1 bins) */
    int32_t reserved;
    double pos[3];         /* centre (circle/annulus) or corner p1 (camera) */
    double dir[3];         /* normal (circle is normalised by the caller, as parse does) */
    double r1, r2;         /* circle: r1 = radius; annulus: r1..r2 */
    double maxval;
    double p2[3], p3[3];   /* camera corners */
} smcrt_detector;

/* ---- run options ---------------------------------------------------------- */
enum smcrt_kernel_kind {
    SMCRT_KERNEL_PATHLENGTH = 0, /* pathlength_scatter: analog absorption, path-length tally */
    SMCRT_KERNEL_WEIGHT = 1,     /* weight_scatter: implicit capture + roulette */
    SMCRT_KERNEL_TEST = 2        /* test_kernel: scatter-order position moments */
};
enum smcrt_precision { SMCRT_FP32 = 0, SMCRT_FP64 = 1 };
/* Order of the action groups in the transport kernel's per-round sorted packet
 * list (smcrt_options.group_order).  The FP64 near-surface sweeps come first and
 * the sweeps second in both; the warps take chunks of the list from its head, so
 * the last group's chunks end each round.  The order changes only the speed. */
enum smcrt_group_order {
    SMCRT_ORDER_WALK_LAST = 1,     /* ..., interactions, voxel walks, launches */
    SMCRT_ORDER_INTERACT_LAST = 2  /* ..., voxel walks, interactions, launches */
};

typedef struct smcrt_options {
    int32_t kernel;        /* smcrt_kernel_kind */
    int32_t precision;     /* transport arithmetic; tallies are always FP64 */
    int32_t end_early;     /* test kernel: kill after the 4th scatter (test_scat.f90:65) */
    int32_t block_size;    /* threads per CTA: 0 or 640 (a CTA holds 1280 FP32 / 640 FP64 packets) */
    int32_t blocks_per_sm; /* 0 = library default (persistent grid = SMs * this) */
    int32_t max_trace_steps; /* per tauint2 sphere-trace step cap; 0 = 1,000,000; at most 2,097,151 */
    double eps;            /* surface epsilon; <= 0 selects the reference's 1e-8
                              (inttau2.f90:44) in both precisions (FP32 transport
                              takes every decision against it in FP64) */
    double normal_h;       /* finite-difference step of the normal; <= 0 -> 1e-6
                              (sdf_base.f90:176); normals are evaluated in FP64 */
    uint32_t instance;     /* RNG stream id (second counter word) */
    int32_t timeout_ms;    /* time limit of one run in ms (device-side budget); 0 = 600000 */
    void* stream;          /* cudaStream_t to launch on; NULL = the default stream */
    int32_t private_stream;/* nonzero: the context creates and owns a non-blocking stream
                              and ignores `stream` */
    int32_t tally_copies;  /* copies of the fluence grid that the CTAs spread their
                              atomic adds over, summed after the launch (no
                              counterpart in the reference; the sum is the same
                              tally): 0 = library choice (as many as fit in
                              64 MiB, at most 8), 1 = a single grid, up to 16;
                              rounded down to a power of two */
    int32_t scene_memory;  /* where the kernel reads the scene: 0 = the launch's
                              parameter block when the scene fits (at most 16
                              regions and 32 primitives), device memory otherwise
                              (up to 255 regions and 4096 primitives, with a
                              bounding-sphere cull of the SDF sweep); 1 = device
                              memory always */
    int32_t variance;      /* nonzero: the context also keeps, per voxel, the FP64 sum over
                              packets of each packet's own score squared (the
                              history-based second moment of jmean; see
                              smcrt_run_moments).  Needs a scene in the parameter
                              block; allocates a voxel-score table per packet slot
                              (40 KiB each, ~7.8 GB for FP32 on 148 SMs) */
    int32_t nearest_cache; /* SDF sweeps of tracing steps skip the regions a per-packet
                              nearest-region bound rules out (results unchanged):
                              0 or 1 = on where the scene allows it (every region an
                              exact distance under a rigid transform), 2 = off */
    int32_t shared_fluence; /* FP32 transport with a pencil source: each CTA sums the
                              fluence of a sub-box along the beam (8 x 8 cells across it,
                              as far along it as shared memory allows) in shared memory
                              as 64-bit fixed point (2^-32 cm) and adds it to the FP64
                              grid once; 0 = library choice (off unless smcrt_autotune
                              picks it), 1 = on, 2 = off */
    int32_t group_order;   /* order of the action groups in each round's sorted list of
                              packets (the warps take its chunks from the head; no
                              counterpart in the reference, results unchanged):
                              0 = library choice (SMCRT_ORDER_WALK_LAST unless
                              smcrt_autotune picks the other), or one of smcrt_group_order */
    int32_t reserved[3];   /* zero */
} smcrt_options;

/* Event counters of one run (definitions identical in the CPU oracle). */
typedef struct smcrt_stats {
    double nscatt;               /* sum of scatters (kernelsMod.f90:292) */
    uint64_t packets;            /* packets launched */
    uint64_t sdf_evals;          /* primitive-region evaluations, packet%cnts semantics
                                    (inttau2.f90:55,90,108,121) + 4 per normal */
    uint64_t voxel_segments;     /* tally additions in update_grids */
    uint64_t trace_steps;        /* sphere-tracing steps */
    uint64_t scatters;           /* scatter calls */
    uint64_t fresnel_events;     /* reflect_refract calls */
    uint64_t reflections;        /* of which reflected */
    uint64_t kills_step_cap;     /* packets killed by the trace-step cap */
    uint64_t kills_error;        /* "should not be reached" states (inttau2.f90:156) */
    uint64_t rng_draws;          /* uniform draws consumed */
    double moments[24];          /* test kernel: sum pos (4x3) then sum pos^2 (4x3) */
    double kernel_ms;            /* device time of the transport kernel(s) */
    int32_t device_status;       /* 0 or a bitmask of device status flags */
    int32_t reserved;
    uint64_t h2d_bytes;          /* host-to-device bytes the call moved: the launch's kernel
                                    parameter block (scene, grid, source, detectors, run
                                    settings) and any uploaded tables */
    uint64_t d2h_bytes;          /* device-to-host bytes the call moved: tallies copied to
                                    host buffers and the event counters */
    uint64_t variance_overflows; /* second-moment runs: segments squared on their own because the
                                    packet's voxel-score table was crowded (their cross terms
                                    with the packet's other scores in that voxel are missing) */
    uint64_t reserved2[5];
} smcrt_stats;

/* Per-packet final state (history replay). */
typedef struct smcrt_packet_state {
    double pos[3];
    double dir[3];
    double weight;
    int32_t layer;         /* 1-based */
    int32_t nscatt;
    int32_t ndraws;        /* uniforms consumed */
    int32_t flags;         /* bit0 step cap, bit1 error state, bit2 stream exhausted */
} smcrt_packet_state;

typedef struct smcrt_ctx smcrt_ctx;

/* Library identity. */
int32_t smcrt_abi_version(void);
/* Message of the last failed call on this thread ("" if none). */
const char* smcrt_last_error(void);

/* Validates and uploads the flattened scene; replaces setup()'s geometry hand-off
 * (src/kernelsMod.f90:453-546 -> setup_simulation, src/setup.f90:14-54). */
int32_t smcrt_create(const smcrt_scene* scene, const smcrt_grid* grid,
                     const smcrt_source* source, const smcrt_detector* dets,
                     int32_t ndet, const smcrt_options* opts, smcrt_ctx** out);
void smcrt_destroy(smcrt_ctx* ctx);

/* Number of detector bins of the context (sum over detectors). */
int64_t smcrt_detector_bins(const smcrt_ctx* ctx);

/* Runs packets [0, nphotons) of stream `seed` -- the OpenMP packet loop
 * src/kernelsMod.f90:265-321 -- and copies the tallies to HOST buffers.
 * jmean (nxg*nyg*nzg) and det_bins (smcrt_detector_bins) are overwritten; either
 * may be NULL to skip it.  Blocks until done. */
int32_t smcrt_run(smcrt_ctx* ctx, int64_t nphotons, uint64_t seed,
                  double* jmean, double* det_bins, smcrt_stats* stats);

/* Adjoint of a pathlength run (no counterpart in the reference): the gradient of
 *     L = sum_v w[v] * jmean[v] + sum_b h[b] * det_bins[b]
 * (the raw tallies of smcrt_run(ctx, nphotons, seed)) with respect to every
 * region group's (mua, mus, g), by path replay: each packet is traced again from
 * its regenerated stream, twice (its total contribution, then the score terms of
 * its events), and nothing per packet is stored.  The expected value is exact;
 * the estimate is the perturbation Monte Carlo (score-function) gradient of the
 * same packets.  w_dev: FP32 DEVICE array (nxg*nyg*nzg), gbins_dev: FP64 DEVICE
 * array (smcrt_detector_bins) or NULL; region_group[r] in -1..ngroups-1 ties
 * region r's parameters to a group (-1: not differentiated), ngroups <= 5.
 * grad (HOST, 3*ngroups): [d/d mua of groups..., d/d mus..., d/d g...], sums
 * over packets (divide by nphotons for the per-packet loss).  Needs an FP32
 * pathlength context. */
int32_t smcrt_adjoint(smcrt_ctx* ctx, int64_t nphotons, uint64_t seed, const float* w_dev,
                      const double* gbins_dev, const int32_t* region_group, int32_t ngroups,
                      double* grad, smcrt_stats* stats);

/* Autotuning (no counterpart in the reference).  Times runs of trial_packets
 * packets of stream `seed` for each candidate launch configuration -- fluence-grid
 * copies 1, 2, 4, 8 (as many as fit in 256 MiB) x detector bins counted in
 * shared memory or in global memory -- and keeps the fastest for the context's
 * later runs.  The CTA shape (640 threads, 2 packet slots per thread) is fixed at
 * build time.  Overwrites the context's device tallies. */
typedef struct smcrt_tuning {
    int32_t tally_copies;  /* chosen fluence-grid copies */
    int32_t shared_bins;   /* 1: detector bins counted in shared memory */
    double packets_per_s;  /* measured rate of the chosen configuration */
    int32_t trials;        /* trial runs made */
    int32_t block_size;    /* threads per CTA of the transport kernel (fixed at build time) */
    int32_t slots_per_thread; /* packet slots per thread (2 in FP32, 1 in FP64 transport) */
    int32_t ctas_per_sm;   /* resident CTAs per SM of the persistent grid */
    int32_t nearest_cache; /* 1: sweeps skip regions the nearest-region cache rules out */
    int32_t shared_fluence; /* 1: each CTA sums a beam-axis sub-box of the fluence in shared memory */
    int32_t group_order;   /* chosen smcrt_group_order */
    int32_t reserved;      /* zero */
} smcrt_tuning;
int32_t smcrt_autotune(smcrt_ctx* ctx, int64_t trial_packets, uint64_t seed, smcrt_tuning* result);

/* Device-resident form: ADDS the tallies of packets [first, first+count) into
 * caller-owned DEVICE buffers, asynchronously on the context stream.  Used for
 * sharding packet ranges and for timing with data already in HBM.  stats may be
 * NULL; if not NULL the call synchronises to fill it. */
int32_t smcrt_run_device(smcrt_ctx* ctx, int64_t first, int64_t count, uint64_t seed,
                         double* jmean_dev, double* det_bins_dev, smcrt_stats* stats);

/* smcrt_run / smcrt_run_device of a context created with options.variance: the
 * same transport, plus the per-voxel second moment jmean2[v] = sum over packets
 * of (the packet's total path length in voxel v)^2, FP64, the layout of jmean.
 * With N packets the per-packet variance of voxel v is jmean2/N - (jmean/N)^2 and
 * the standard error of jmean/N is sqrt(that / N) (no counterpart in the
 * reference, which keeps no variance).  _moments copies to HOST buffers (each
 * may be NULL); _device_moments ADDS into DEVICE buffers on the context stream. */
int32_t smcrt_run_moments(smcrt_ctx* ctx, int64_t nphotons, uint64_t seed, double* jmean,
                          double* jmean2, double* det_bins, smcrt_stats* stats);
int32_t smcrt_run_device_moments(smcrt_ctx* ctx, int64_t first, int64_t count, uint64_t seed,
                                 double* jmean_dev, double* jmean2_dev, double* det_bins_dev,
                                 smcrt_stats* stats);

/* Replays packets from caller-supplied uniform streams instead of the counter
 * RNG: packet p consumes uniforms[offsets[p] .. offsets[p+1]) in the reference's
 * draw order -- emitter draws, tau (inttau2.f90:46), then per Fresnel crossing
 * the reflect test (surfaces.f90:33) and a new tau (inttau2.f90:168), per
 * interaction the albedo test (kernelsMod.f90:287), the bias test if g != 0
 * (photon.f90:739), the HG/isotropic draw, the phi draw, and the next tau.
 * Writes per-packet final states. */
int32_t smcrt_replay(smcrt_ctx* ctx, const double* uniforms, const int64_t* offsets,
                     int64_t npackets, double* jmean, double* det_bins,
                     smcrt_packet_state* states, smcrt_stats* stats);

/* ---- batches ----------------------------------------------------------------
 * Many instances of one scene -- the same geometry, grid, source, detectors and
 * options, each with its own region optics, packet count and seed -- transported
 * in ONE persistent launch (pathlength and weight kernels).  Instance i runs
 * packets [0, nphotons[i]) of stream seeds[i]: the packets smcrt_run would run
 * with that seed and those optics, so a batch equals its instances run one by one
 * (FP64: identical event counts).  No counterpart in the reference, which runs one
 * simulation per process. */
typedef struct smcrt_region_optics {
    double mus, mua, hgg, n;  /* as in smcrt_region */
} smcrt_region_optics;
typedef struct smcrt_batch smcrt_batch;

/* Creates a batch of ninst instances (1..262143), all with the scene's optics;
 * allocates the instances' FP64 tallies (ninst*ncell, instance-major) and
 * detector bins (ninst*nbins) on the device. */
int32_t smcrt_batch_create(const smcrt_scene* scene, const smcrt_grid* grid,
                           const smcrt_source* source, const smcrt_detector* dets,
                           int32_t ndet, const smcrt_options* opts, int32_t ninst,
                           smcrt_batch** out);
/* Sets every instance's region optics: optics[i*nregions + r] for instance i,
 * region r (scene order).  Waits for a launch in flight. */
int32_t smcrt_batch_set_optics(smcrt_batch* b, const smcrt_region_optics* optics);
/* Zeroes the batch tallies and launches all instances asynchronously on the
 * batch's stream.  use_graph != 0: the table upload, the zeroing and the kernel are
 * captured into a CUDA graph on the first such call and replayed after that
 * (packet counts and seeds are device data and may change between calls). */
int32_t smcrt_batch_launch(smcrt_batch* b, const int64_t* nphotons, const uint64_t* seeds,
                           int32_t use_graph);
/* Waits for the launch (bounded by the time limit) and copies to HOST buffers
 * (each may be NULL): jmean (ninst*ncell), det_bins (ninst*nbins),
 * per_instance[i] (packets, rng_draws and nscatt of instance i) and total (the
 * event counters of the whole launch). */
int32_t smcrt_batch_wait(smcrt_batch* b, double* jmean, double* det_bins,
                         smcrt_stats* per_instance, smcrt_stats* total);
/* Device addresses of the batch tallies (valid until smcrt_batch_destroy). */
int32_t smcrt_batch_device_tallies(smcrt_batch* b, double** jmean_dev, double** det_bins_dev);
/* The batch's cudaStream_t, for ordering caller work after a launch. */
int64_t smcrt_batch_stream(const smcrt_batch* b);
void smcrt_batch_destroy(smcrt_batch* b);

/* Batched run over contexts: ninst contexts whose scenes share their geometry
 * (region optics may differ) run as one batch launch; jmeans[i] / det_bins[i] are
 * host buffers (or NULL), stats[i] gets packets, rng_draws and nscatt.  Contexts
 * with different geometry, or test kernels, run one launch each. */
int32_t smcrt_run_batched(smcrt_ctx* const* ctxs, int32_t ninst, const int64_t* nphotons,
                          const uint64_t* seeds, double* const* jmeans,
                          double* const* det_bins, smcrt_stats* stats);

/* Allocation-free form of smcrt_run_device (no counterpart in the reference,
 * where signedMCRT allocates its tallies itself).  It is for callers that cannot
 * let a library allocate device memory: applications that hand out every byte of
 * device memory from their own pool allocator, or processes whose device memory
 * is reserved up front for a fixed budget.  It takes the same inputs as
 * smcrt_create plus caller-owned DEVICE tally buffers, creates no context and
 * calls no cudaMalloc/cudaFree: the kernel's scratch (work counter, event
 * counters, status word; about 300 bytes) lives in a static device array of
 * smcrt_static_scratch_bytes() bytes inside the library, present on every GPU
 * that loads it until the process exits.  Scenes that need device-resident scene
 * tables (more than 16 regions or 32 primitives) are refused with
 * SMCRT_ERR_SCENE.  ADDS the tallies of packets [first, first+count) into
 * jmean_dev/det_bins_dev on opts->stream (NULL = the default stream).  The first
 * call on a device looks up the array's device address for that device
 * (cudaGetSymbolAddress); make that first call before any stream capture.  Every
 * call shares the one array and clears it at its start: calls that overlap on
 * the GPU (other streams, other threads) race on it.  If stats is not NULL the
 * call waits for the kernel (with a host-side limit of the time budget plus
 * 30 s) and fills it; a run stopped by its time budget then returns
 * SMCRT_ERR_TIMEOUT.  If stats is NULL the call returns after the launch and such
 * a stop is NOT reported: pass stats to learn of it. */
int32_t smcrt_run_device_static(const smcrt_scene* scene, const smcrt_grid* grid,
                                const smcrt_source* source, const smcrt_detector* dets,
                                int32_t ndet, const smcrt_options* opts, int64_t first,
                                int64_t count, uint64_t seed, double* jmean_dev,
                                double* det_bins_dev, smcrt_stats* stats);
/* Size of the static scratch array used by smcrt_run_device_static. */
int64_t smcrt_static_scratch_bytes(void);

/* ---- SDF voxel render (render_sub, src/sdfs/sdf_base.f90:302-346) ---------- */
/* The minimum over all regions of the scene's signed distance at every voxel of a
 * samples[0] x samples[1] x samples[2] grid: voxel (i, j, k), 1-based, sits at
 * ((i - ns[0]) w[0], (j - ns[1]) w[1], (k - ns[2]) w[2]) with ns = nint(samples / 2)
 * and w = extent / ns.  Written FP32 in Fortran order (i fastest) to `image`, host
 * memory of samples[0]*samples[1]*samples[2] floats.  Replaces the OpenMP loop of
 * render_sub; the caller writes the file (write_data).  precision: SMCRT_FP64
 * evaluates in double as the reference's real(wp) does, SMCRT_FP32 in float.
 * Each samples[a] in [1, 65536]. */
int32_t smcrt_render(const smcrt_scene* scene, int32_t precision, const int32_t samples[3],
                     const double extent[3], float* image);
/* The same into caller DEVICE memory, asynchronously on `stream` (a cudaStream_t;
 * NULL = the default stream).  Allocates nothing. */
int32_t smcrt_render_device(const smcrt_scene* scene, int32_t precision, const int32_t samples[3],
                            const double extent[3], float* image_dev, void* stream);

/* ---- device-function probes (parity of the building blocks) --------------- */
/* Evaluates every region's SDF at npts points (xyz triples); out[p*nregions+r]. */
int32_t smcrt_eval_sdf(const smcrt_scene* scene, int32_t precision,
                       const double* pts, int64_t npts, double* out);
/* calcNormal (src/sdfs/sdf_base.f90:165-189) of one region at npts points. */
int32_t smcrt_calc_normal(const smcrt_scene* scene, int32_t region0, double h,
                          const double* pts, int64_t npts, double* out_xyz);
/* fresnel (src/surfaces.f90:86-120) per (I, N, n1, n2) tuple. */
int32_t smcrt_fresnel(int32_t precision, const double* I, const double* N,
                      const double* n1, const double* n2, int64_t n, double* R);
/* reflect_refract (src/surfaces.f90:14-40) with a given uniform u per tuple:
 * writes the new direction and reflect flag. */
int32_t smcrt_reflect_refract(int32_t precision, const double* I, const double* N,
                              const double* n1, const double* n2, const double* u,
                              int64_t n, double* I_out, int32_t* reflected);
/* scatter (src/photon.f90:713-779) with given uniforms (3 per call if g != 0,
 * else 2 (the bias-test draw is skipped when g == 0)). */
int32_t smcrt_scatter_dir(int32_t precision, const double* dir_in, const double* g,
                          const double* u, int64_t n, double* dir_out);
/* Launch state of packets [first, first+npk) of stream `seed` (instance 0): the
 * emitter of `source` (src/photon.f90: pencil :464-505, point :290-338, uniform
 * :397-461, circular :214-287, annulus :645-711, focus :340-394) and the launch
 * layer (src/kernelsMod.f90:275-280, 1-based) as the transport kernels take it.
 * pos/dir: 3 doubles per packet. */
int32_t smcrt_emit(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* source,
                   int32_t precision, int64_t first, int64_t npk, uint64_t seed, double* pos,
                   double* dir, int32_t* layer);
/* Philox4x32-10 block for (key, counter): 4 words per request. */
int32_t smcrt_philox(const uint32_t* key2, const uint32_t* ctr4, int64_t n, uint32_t* out4);

#ifdef __cplusplus
}
#endif
#endif /* SMCRT_H */
