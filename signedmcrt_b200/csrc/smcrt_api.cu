// smcrt_api.cu -- the C ABI of include/smcrt.h.
//
// The context owns device memory and a stream; a run zeroes the device tallies,
// launches the persistent transport kernel (one CTA set sized to the SM count x
// resident CTAs per SM), waits with a host-side time limit, and copies the FP64
// tallies out.  No call exits the process: errors return a status and a message.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "smcrt_launch.h"

using namespace smcrt;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CK(call)                                                                                         \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return fail(SMCRT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));             \
    } while (0)

// ---------------------------------------------------------------------------
// param_block: the caller needs the scene inside a launch's parameter block (at
// most kMaxRegions regions and kMaxPrims primitives: batches, the adjoint, the
// allocation-free run, the probes and the render); contexts also take larger
// scenes, up to kMaxRegionsDev / kMaxPrimsDev, kept in device memory.
int validate_scene(const smcrt_scene* s, bool param_block = true) {
    if (!s || !s->regions || !s->prims) return fail(SMCRT_ERR_ARG, "scene: null pointer");
    if (s->nregions <= 0 || s->nprims <= 0) return fail(SMCRT_ERR_SCENE, "scene: empty");
    const int maxr = param_block ? kMaxRegions : kMaxRegionsDev, maxp = param_block ? kMaxPrims : kMaxPrimsDev;
    if (s->nregions > maxr || s->nprims > maxp)
        return fail(SMCRT_ERR_SCENE, "scene: at most " + std::to_string(maxr) + " regions and " +
                                         std::to_string(maxp) + " primitives" +
                                         (param_block ? std::string(" here (larger scenes run through smcrt_create "
                                                                    "contexts)")
                                                      : std::string()));
    for (int i = 0; i < s->nprims; ++i) {
        const smcrt_prim& pr = s->prims[i];
        if (pr.kind < SMCRT_SPHERE || pr.kind > SMCRT_PLANE)
            return fail(SMCRT_ERR_SCENE, "scene: unknown primitive kind at " + std::to_string(i));
        if (pr.nmods < 0 || pr.nmods > 2)
            return fail(SMCRT_ERR_SCENE, "scene: primitive " + std::to_string(i) + " needs 0..2 modifiers");
        for (int j = 0; j < pr.nmods; ++j)
            if (pr.mods[j] < SMCRT_MOD_ONION || pr.mods[j] > SMCRT_MOD_BEND)
                return fail(SMCRT_ERR_SCENE, "scene: unknown modifier on primitive " + std::to_string(i));
    }
    for (int i = 0; i < s->nregions; ++i) {
        const smcrt_region& r = s->regions[i];
        if (r.nprims <= 0 || r.first_prim < 0 || r.first_prim + r.nprims > s->nprims)
            return fail(SMCRT_ERR_SCENE, "scene: region " + std::to_string(i) + " primitive range out of bounds");
        if (r.nprims > 1 && (r.op < SMCRT_OP_UNION || r.op > SMCRT_OP_INTERSECTION))
            return fail(SMCRT_ERR_SCENE, "scene: region " + std::to_string(i) + " has an unknown CSG op");
        if (r.nprims > 1 && r.op == SMCRT_OP_SMOOTH_UNION && !(r.k > 0))
            return fail(SMCRT_ERR_SCENE, "scene: smooth union needs k > 0");
    }
    return SMCRT_OK;
}

// Optical properties only matter to transport (the probes accept the
// reference's mono(0,0,0,0) test objects).
int validate_optics(const smcrt_scene* s) {
    for (int i = 0; i < s->nregions; ++i) {
        const smcrt_region& r = s->regions[i];
        if (!(r.mus >= 0) || !(r.mua >= 0) || !(r.n > 0) || !(r.mus + r.mua >= 0) || !std::isfinite(r.hgg) ||
            !(std::fabs(r.hgg) < 1.0))
            return fail(SMCRT_ERR_SCENE, "scene: region " + std::to_string(i) +
                                             " needs mus >= 0, mua >= 0, n > 0 and |g| < 1");
    }
    return SMCRT_OK;
}

template <class R>
void fill_grid(GridT<R>& g, const smcrt_grid& s) {
    g.nx = s.nxg;
    g.ny = s.nyg;
    g.nz = s.nzg;
    g.xmax = (R)s.xmax;
    g.ymax = (R)s.ymax;
    g.zmax = (R)s.zmax;
    g.vx = (R)2 * (R)s.xmax / (R)s.nxg;
    g.vy = (R)2 * (R)s.ymax / (R)s.nyg;
    g.vz = (R)2 * (R)s.zmax / (R)s.nzg;
    g.sx = (R)s.nxg / ((R)2 * (R)s.xmax);
    g.sy = (R)s.nyg / ((R)2 * (R)s.ymax);
    g.sz = (R)s.nzg / ((R)2 * (R)s.zmax);
    g.xmax_d = s.xmax;
    g.ymax_d = s.ymax;
    g.zmax_d = s.zmax;
    g.sx_d = (double)s.nxg / (2.0 * s.xmax);
    g.sy_d = (double)s.nyg / (2.0 * s.ymax);
    g.sz_d = (double)s.nzg / (2.0 * s.zmax);
    // the same expression as the walk's face positions had on the device (2.0 * max / n,
    // IEEE-rounded), computed once here instead of three FP64 divisions a step
    g.vx_d = 2.0 * s.xmax / (double)s.nxg;
    g.vy_d = 2.0 * s.ymax / (double)s.nyg;
    g.vz_d = 2.0 * s.zmax / (double)s.nzg;
}

template <class R>
void fill_source(SourceT<R>& d, const smcrt_source& s, const smcrt_grid& g) {
    std::memset(&d, 0, sizeof(d));
    d.kind = s.kind;
    d.annulus_type = s.annulus_type;
    for (int a = 0; a < 3; ++a) {
        d.pos[a] = (R)s.pos[a];
        d.dir[a] = (R)s.dir[a];
        d.p1[a] = (R)s.point1[a];
        d.p2[a] = (R)s.point2[a];
        d.p3[a] = (R)s.point3[a];
    }
    d.radius = (R)s.radius;
    d.radius_hi = (R)s.radius_hi;
    const double ang = s.beta * kPI / 180.0;
    d.sin_beta = (R)std::sin(ang);
    d.cos_beta = (R)std::cos(ang);
    d.zstart = (R)(g.zmax - s.z_inset);
    // circular source: rotationAlign(a, b) (src/sdfs/sdfHelpers.f90:114-140), a = x or z axis
    double bl = std::sqrt(s.dir[0] * s.dir[0] + s.dir[1] * s.dir[1] + s.dir[2] * s.dir[2]);
    double b[3] = {s.dir[0] / bl, s.dir[1] / bl, s.dir[2] / bl};
    double a[3] = {1, 0, 0};
    d.circ_swap = 0;
    if (std::fabs(b[0]) == 1.0 && b[1] == 0.0 && b[2] == 0.0) {
        a[0] = 0;
        a[2] = 1;
        d.circ_swap = 1;
    }
    double v[3] = {a[1] * b[2] - a[2] * b[1], -a[0] * b[2] + a[2] * b[0], a[0] * b[1] - a[1] * b[0]};
    double c = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    double k = 1.0 / (1.0 + c);
    double V[3][3] = {{0, v[2], -v[1]}, {-v[2], 0, v[0]}, {v[1], -v[0], 0}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s2 = 0;
            for (int q = 0; q < 3; ++q) s2 += V[i][q] * V[q][j];
            d.rot[3 * i + j] = (R)((i == j ? 1.0 : 0.0) + V[i][j] + s2 * k);
        }
}

int fill_dets(DetT* out, const smcrt_detector* dets, int ndet, int nregions, long long& total) {
    total = 0;
    for (int i = 0; i < ndet; ++i) {
        DetT& D = out[i];
        std::memset(&D, 0, sizeof(D));
        const smcrt_detector& s = dets[i];
        if (s.kind < SMCRT_DET_CIRCLE || s.kind > SMCRT_DET_CAMERA)
            return fail(SMCRT_ERR_ARG, "detector " + std::to_string(i) + ": unknown kind");
        if (s.nbins < 0) return fail(SMCRT_ERR_ARG, "detector " + std::to_string(i) + ": nbins < 0");
        if (s.layer < 1 || s.layer > nregions)
            return fail(SMCRT_ERR_ARG, "detector " + std::to_string(i) + ": layer outside 1..nregions");
        D.kind = s.kind;
        D.layer = s.layer;
        D.off = total;
        for (int a = 0; a < 3; ++a) {
            D.pos[a] = s.pos[a];
            D.dir[a] = s.dir[a];
        }
        D.r1 = s.r1;
        D.r2 = s.r2;
        D.nb = s.nbins + 1;
        if (s.kind == SMCRT_DET_CAMERA) {  // init_camera, detectors.f90:186-229
            D.bw = D.bwy = (s.nbins == 0) ? 1.0 : s.maxval / (double)D.nb;
            for (int a = 0; a < 3; ++a) {
                D.e1[a] = s.p2[a] - s.pos[a];
                D.e2[a] = s.p3[a] - s.pos[a];
            }
            D.width = std::sqrt(D.e1[0] * D.e1[0] + D.e1[1] * D.e1[1] + D.e1[2] * D.e1[2]);
            D.height = std::sqrt(D.e2[0] * D.e2[0] + D.e2[1] * D.e2[1] + D.e2[2] * D.e2[2]);
            double nx = D.e2[1] * D.e1[2] - D.e2[2] * D.e1[1];
            double ny = -D.e2[0] * D.e1[2] + D.e2[2] * D.e1[0];
            double nz = D.e2[0] * D.e1[1] - D.e2[1] * D.e1[0];
            double ln = std::sqrt(nx * nx + ny * ny + nz * nz);
            D.n[0] = nx / ln;
            D.n[1] = ny / ln;
            D.n[2] = nz / ln;
            total += (long long)D.nb * D.nb;
        } else {
            if (s.nbins == 0) D.bw = 1.0;
            else if (s.kind == SMCRT_DET_CIRCLE) D.bw = s.maxval / (double)(s.nbins - 1);  // :104
            else D.bw = s.maxval / (double)s.nbins;                                          // :163
            total += D.nb;
        }
    }
    return SMCRT_OK;
}

// Surface epsilon: the reference's 1e-8 (src/inttau2.f90:44) in both precisions.
// FP32 transport can keep it because every decision against it is taken in FP64
// (sweeps within near_band of a surface and crossing sweeps, see the kernel).
double default_eps(int, const smcrt_grid&) { return 1e-8; }

// FP32 transport: the distance below which a sweep is repeated in FP64 -- 16 FP32
// ulps of the largest grid half-size (FP32 coordinate rounding and the affine
// transform move a distance by a few ulps), and at least twice eps.
double near_band(double eps, const smcrt_grid& g) {
    const double L = std::fmax(g.xmax, std::fmax(g.ymax, g.zmax));
    int e;
    std::frexp(L, &e);                     // L in [2^(e-1), 2^e)
    const double ulp = std::ldexp(1.0, e - 24);  // FP32 spacing at L
    return std::fmax(2.0 * eps, 16.0 * ulp);
}

// The per-flight sphere-trace step count shares its slot word with the
// nearest-region cache: 21 bits.
constexpr int kMaxTraceSteps = (1 << 21) - 1;
// Option checks shared by contexts, batches and the allocation-free run.
int check_steps(const smcrt_options* o) {
    if (o && o->max_trace_steps > kMaxTraceSteps)
        return fail(SMCRT_ERR_ARG, "options: max_trace_steps must be at most " + std::to_string(kMaxTraceSteps));
    if (o && (o->group_order < 0 || o->group_order > SMCRT_ORDER_INTERACT_LAST))
        return fail(SMCRT_ERR_ARG, "options: group_order must be 0, 1 or 2");
    return SMCRT_OK;
}

// The kernel's nibble table for an smcrt_group_order (0: the library's choice).
unsigned group_order_table(int order) {
    return order == SMCRT_ORDER_INTERACT_LAST ? kOrderInteractLast : kOrderWalkLast;
}

int pick_device(int& dev, int& nsm) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(SMCRT_ERR_NO_DEVICE, "no CUDA device visible");
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    return SMCRT_OK;
}

// Sums the fluence-grid copies into the output grid and zeroes them for the
// next launch: cells are independent, one coalesced grid-stride pass.
__global__ void __launch_bounds__(256) reduce_copies_kernel(double* __restrict__ out, double* __restrict__ copies,
                                                            int ncopies, long long ncell) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ncell; i += stride) {
        double sum = 0.0;
        for (int k = 0; k < ncopies; ++k) {
            double* q = copies + (long long)k * ncell + i;
            sum += *q;
            *q = 0.0;
        }
        if (sum != 0.0) out[i] += sum;
    }
}

}  // namespace

cudaError_t smcrt::reduce_tally_copies(double* out, double* copies, int ncopies, long long ncell, int nsm,
                                       cudaStream_t s) {
    const long long need = (ncell + 255) / 256;
    const int blocks = (int)std::min<long long>(need, (long long)nsm * 8);
    reduce_copies_kernel<<<blocks, 256, 0, s>>>(out, copies, ncopies, ncell);
    return cudaGetLastError();
}

// ===========================================================================
struct smcrt_ctx {
    int device = 0, nsm = 0;
    int precision = SMCRT_FP32, kernel = SMCRT_KERNEL_PATHLENGTH;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Params<float>* pf = nullptr;
    Params<double>* pd = nullptr;
    long long ncell = 0, nbins = 0;
    int tcopies = 1;                          // fluence-grid copies (1 = the output grid only)
    int copies_alloc = 1;                     // copies d_copies holds (+1 for the output grid)
    bool shared_bins_on = true;               // detector bins counted in shared memory when they fit
    double* d_jmean = nullptr;
    double* d_copies = nullptr;               // tcopies - 1 zeroed copies
    double* d_bins = nullptr;
    unsigned long long* d_work = nullptr;     // [0] work, [1..C_NUM] counters
    double* d_mom = nullptr;                  // 25
    int* d_status = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int block = 256, grid_blocks = 0;
    int timeout_ms = 600000;
    bool big = false;                         // scene tables in device memory (d_scene)
    void* d_scene = nullptr;
    bool variance = false;                    // second-moment runs available
    unsigned char* d_vartab = nullptr;        // voxel-score table of every packet slot
    size_t vartab_bytes = 0;
    bool vartab_clean = false;                // every table seen empty after the last moments run
    bool cache_allowed = false;               // every region 1-Lipschitz: the nearest-region cache may run
    // shared-memory fluence privatisation (FP32, sources with a start point): the
    // sub-box around the source's cell, its extent along the beam fitted per launch
    bool priv_allowed = false, priv_on = false;
    int priv_o[3] = {0, 0, 0}, priv_d[3] = {0, 0, 0}, priv_axis = 2, priv_sign = -1;
    double* d_jmean2 = nullptr;               // second moment of smcrt_run_moments
};

namespace {

// Detector bins counted per CTA in shared memory: all of them when they fit,
// else none.  A CTA's count of one bin is at most the packets of the launch, so
// launches of 2^32 packets or more use the global bins.
int shared_bins(long long nbins, long long count) {
    return (nbins > 0 && nbins <= kMaxSharedBins && count < (1ll << 32)) ? (int)nbins : 0;
}

// Resident CTAs per SM of the transport kernel with `smem` bytes of dynamic
// shared memory, capped by the caller's blocks_per_sm.
int resident_per_sm(int precision, int kernel, int block, size_t smem, int blocks_per_sm, int* out) {
    int per_sm = 0;
    cudaError_t e;
    if (precision == SMCRT_FP64) {
        e = kernel == SMCRT_KERNEL_WEIGHT ? occupancy_f64_1(block, smem, &per_sm)
            : kernel == SMCRT_KERNEL_TEST ? occupancy_f64_2(block, smem, &per_sm)
                                          : occupancy_f64_0(block, smem, &per_sm);
    } else {
        e = kernel == SMCRT_KERNEL_WEIGHT ? occupancy_f32_1(block, smem, &per_sm)
            : kernel == SMCRT_KERNEL_TEST ? occupancy_f32_2(block, smem, &per_sm)
                                          : occupancy_f32_0(block, smem, &per_sm);
    }
    if (e != cudaSuccess) return fail(SMCRT_ERR_CUDA, std::string("occupancy: ") + cudaGetErrorString(e));
    if (per_sm < 1) per_sm = 1;
    if (blocks_per_sm > 0 && blocks_per_sm < per_sm) per_sm = blocks_per_sm;
    *out = per_sm;
    return SMCRT_OK;
}

int occupancy_grid(smcrt_ctx* c, int precision, int kernel, int blocks_per_sm) {
    int per_sm = 0;
    const size_t smem = sizeof(unsigned) * (size_t)shared_bins(c->nbins, 0);
    int rc = resident_per_sm(precision, kernel, c->block, smem, blocks_per_sm, &per_sm);
    if (rc) return rc;
    c->grid_blocks = c->nsm * per_sm;
    return SMCRT_OK;
}

// Fluence-grid copies: the requested number, or as many as fit in 64 MiB (at
// most 8), rounded down to a power of two.  Copies spread the atomic adds of
// packets that share voxels (a pencil beam's axis) over several addresses.
int tally_copies(const smcrt_options* o, long long ncell, int* out) {
    const int req = o ? o->tally_copies : 0;
    if (req < 0 || req > kMaxTallyCopies)
        return fail(SMCRT_ERR_ARG, "options: tally_copies must be 0.." + std::to_string(kMaxTallyCopies));
    const long long budget = 64ll << 20;
    const long long want = req > 0 ? req : std::max(1ll, std::min(8ll, budget / (8ll * ncell)));
    int tc = 1;  // rounded down to a power of two (the kernel picks a copy by a mask)
    while (tc * 2 <= want) tc *= 2;
    *out = tc;
    return SMCRT_OK;
}

template <class R>
void fill_params(Params<R>* P, const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* src,
                 const DetT* dets, int ndet, const smcrt_options* o) {
    std::memset(P, 0, sizeof(*P));
    fill_scene(P->sc, scene);
    fill_scene(P->sc64, scene);
    fill_grid(P->grid, *grid);
    fill_source(P->src, *src, *grid);
    for (int i = 0; i < ndet; ++i) P->det[i] = dets[i];
    P->ndet = ndet;
    P->kernel = o ? o->kernel : SMCRT_KERNEL_PATHLENGTH;
    P->end_early = o ? o->end_early : 0;
    P->max_steps = (o && o->max_trace_steps > 0) ? o->max_trace_steps : 1000000;
    const int prec = (sizeof(R) == 4) ? SMCRT_FP32 : SMCRT_FP64;
    P->eps = (R)((o && o->eps > 0) ? o->eps : default_eps(prec, *grid));
    P->near_band = (R)near_band((double)P->eps, *grid);
    // the nearest-region cache: on wherever every region is 1-Lipschitz, unless
    // switched off (smcrt_autotune times both)
    const bool allowed = cache_policy(scene, grid, (int)sizeof(R), &P->cache_margin);
    const int want = o ? o->nearest_cache : 0;
    P->cache_ok = allowed && want != 2 ? 1 : 0;
    P->group_order = group_order_table(o ? o->group_order : 0);
    P->normal_h = (o && o->normal_h > 0) ? o->normal_h : 1e-6;
    P->instance = o ? o->instance : 0u;
    P->tcopies = 1;
    P->tmask = 0;
    P->ncell = (long long)grid->nxg * grid->nyg * grid->nzg;
    P->budget_ns = (unsigned long long)((o && o->timeout_ms > 0) ? o->timeout_ms : 600000) * 1000000ull;
}

template <class R>
Params<R>* make_params(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* src,
                       const DetT* dets, int ndet, const smcrt_options* o) {
    Params<R>* P = new Params<R>;
    fill_params(P, scene, grid, src, dets, ndet, o);
    return P;
}

Buffers make_buffers(smcrt_ctx* c, double* jm, double* bins) {
    Buffers B;
    B.jmean = jm;
    B.bins = bins;
    B.work = c->d_work;
    B.counters = c->d_work + 1;
    B.moments = c->d_mom;
    B.status = c->d_status;
    B.uniforms = nullptr;
    B.offsets = nullptr;
    B.states = nullptr;
    return B;
}

int launch_f32(smcrt_ctx* c, const Params<float>& P, const Buffers& B, bool replay, int blocks) {
    cudaError_t e = P.kernel == SMCRT_KERNEL_WEIGHT ? launch_f32_1(P, B, replay, blocks, c->block, c->stream)
                    : P.kernel == SMCRT_KERNEL_TEST ? launch_f32_2(P, B, replay, blocks, c->block, c->stream)
                                                    : launch_f32_0(P, B, replay, blocks, c->block, c->stream);
    if (e != cudaSuccess) return fail(SMCRT_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return SMCRT_OK;
}
int launch_f64(smcrt_ctx* c, const Params<double>& P, const Buffers& B, bool replay, int blocks) {
    cudaError_t e = P.kernel == SMCRT_KERNEL_WEIGHT ? launch_f64_1(P, B, replay, blocks, c->block, c->stream)
                    : P.kernel == SMCRT_KERNEL_TEST ? launch_f64_2(P, B, replay, blocks, c->block, c->stream)
                                                    : launch_f64_0(P, B, replay, blocks, c->block, c->stream);
    if (e != cudaSuccess) return fail(SMCRT_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return SMCRT_OK;
}

template <class R>
void set_tally_table(Params<R>* P, double* jm, double* copies, int tc, long long ncell) {
    P->tcopies = tc;
    P->tmask = (unsigned)(tc - 1);
    for (int k = 0; k < kMaxTallyCopies; ++k)
        P->jtab[k] = (k == 0) ? jm : (k < tc ? copies + (long long)(k - 1) * ncell : nullptr);
}

// The privatised sub-box of a launch with `sb` shared detector bins: the context's
// box, its extent along the beam cut to the shared memory left beside the slots
// and the bins (no box when fewer than 64 cells fit).
int set_priv(smcrt_ctx* c, Params<float>& P, int sb) {
    P.priv_n = 0;
    if (!c->priv_on) return SMCRT_OK;
    int cells = 0;
    cudaError_t e = c->kernel == SMCRT_KERNEL_WEIGHT ? priv_cells_f32_1(sb, &cells)
                  : c->kernel == SMCRT_KERNEL_TEST ? priv_cells_f32_2(sb, &cells)
                                                   : priv_cells_f32_0(sb, &cells);
    if (e != cudaSuccess) return fail(SMCRT_ERR_CUDA, std::string("shared fluence: ") + cudaGetErrorString(e));
    int d[3] = {c->priv_d[0], c->priv_d[1], c->priv_d[2]};
    const int a = c->priv_axis, across = d[(a + 1) % 3] * d[(a + 2) % 3];
    d[a] = std::min(d[a], cells / std::max(1, across));
    if (d[a] < 1 || d[0] * d[1] * d[2] < 64) return SMCRT_OK;
    int o[3] = {c->priv_o[0], c->priv_o[1], c->priv_o[2]};
    if (c->priv_sign < 0) o[a] = c->priv_o[a] + c->priv_d[a] - d[a];  // keep the cells next to the source
    for (int k = 0; k < 3; ++k) {
        P.priv_o[k] = o[k];
        P.priv_d[k] = d[k];
    }
    P.priv_n = d[0] * d[1] * d[2];
    return SMCRT_OK;
}

// Enqueues: reset work/counters/status, then the kernel for [first, first+count).
// jm2: the second-moment grid of a moments run (nullptr otherwise).  Retiring
// packets empty their voxel-score tables, so the tables are filled with the empty
// key only before the first moments run and after one that was not seen to finish
// (stopped by its time budget, or launched without a wait on its stats).
int enqueue(smcrt_ctx* c, long long first, long long count, uint64_t seed, double* jm, double* bins, bool replay,
            const double* d_u, const long long* d_off, smcrt_packet_state* d_states, double* jm2 = nullptr) {
    CK(cudaMemsetAsync(c->d_work, 0, sizeof(unsigned long long) * (1 + C_NUM), c->stream));
    if (jm2 && !c->vartab_clean) CK(cudaMemsetAsync(c->d_vartab, 0xFF, c->vartab_bytes, c->stream));
    if (jm2) c->vartab_clean = false;
    CK(cudaMemsetAsync(c->d_mom, 0, sizeof(double) * 25, c->stream));
    CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
    Buffers B = make_buffers(c, jm, bins);
    B.uniforms = d_u;
    B.offsets = d_off;
    B.states = d_states;
    long long need = (count + c->block - 1) / c->block;
    int blocks = (int)std::min<long long>(c->grid_blocks, std::max<long long>(need, 1));
    const int sb = c->shared_bins_on ? shared_bins(c->nbins, count) : 0;
    int tc = 1;  // a power of two, at most one copy per CTA
    while (tc * 2 <= std::min(c->tcopies, blocks)) tc *= 2;
    int rc;
    if (c->precision == SMCRT_FP64) {
        c->pd->first = first;
        c->pd->count = count;
        c->pd->seed = seed;
        c->pd->sbins = sb;
        c->pd->var_tab = jm2 ? c->d_vartab : nullptr;
        c->pd->jmean2 = jm2;
        set_tally_table(c->pd, jm, c->d_copies, tc, c->ncell);
        rc = launch_f64(c, *c->pd, B, replay, blocks);
    } else {
        c->pf->first = first;
        c->pf->count = count;
        c->pf->seed = seed;
        c->pf->sbins = sb;
        c->pf->var_tab = jm2 ? c->d_vartab : nullptr;
        c->pf->jmean2 = jm2;
        rc = set_priv(c, *c->pf, sb);
        if (rc) return rc;
        set_tally_table(c->pf, jm, c->d_copies, tc, c->ncell);
        rc = launch_f32(c, *c->pf, B, replay, blocks);
    }
    if (rc) return rc;
    if (tc > 1) CK(reduce_tally_copies(jm, c->d_copies, tc - 1, c->ncell, c->nsm, c->stream));
    return SMCRT_OK;
}

// Waits for ev1.  The kernel enforces the context's time limit itself (a
// %globaltimer budget, after which threads stop between flights and raise
// STATUS_ABORTED); the host waits that long plus a grace period.
// Sleep between two polls of a running launch, about 1% of the time waited so far
// (20 us to 500 us): a short launch is not held up by a long sleep, and a long one
// costs few polls.
void poll_sleep(double waited_ms) {
    std::this_thread::sleep_for(std::chrono::microseconds((long)std::min(500.0, std::max(20.0, waited_ms * 10.0))));
}

int wait_bounded(smcrt_ctx* c) {
    auto t0 = std::chrono::steady_clock::now();
    const double limit = (double)c->timeout_ms + 30000.0;
    for (;;) {
        cudaError_t e = cudaEventQuery(c->ev1);
        if (e == cudaSuccess) return SMCRT_OK;
        if (e != cudaErrorNotReady) return fail(SMCRT_ERR_CUDA, std::string("kernel: ") + cudaGetErrorString(e));
        double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms > limit) return fail(SMCRT_ERR_TIMEOUT, "transport kernel did not finish within its time limit");
        poll_sleep(ms);
    }
}

// Bytes of one launch's kernel parameter block (the scene and run settings
// travel as kernel parameters) and of the counter read-back.
size_t param_bytes(const smcrt_ctx* c) {
    return c->precision == SMCRT_FP64 ? sizeof(Params<double>) : sizeof(Params<float>);
}
constexpr size_t kCounterBytes = sizeof(unsigned long long) * (1 + C_NUM) + sizeof(double) * 25 + sizeof(int);

int read_stats(smcrt_ctx* c, smcrt_stats* st) {
    unsigned long long cnt[1 + C_NUM];
    double mom[25];
    int status = 0;
    CK(cudaMemcpy(cnt, c->d_work, sizeof(cnt), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(mom, c->d_mom, sizeof(mom), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&status, c->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    if (st) {
        std::memset(st, 0, sizeof(*st));
        const unsigned long long* k = cnt + 1;
        st->packets = k[C_PACKETS];
        st->sdf_evals = k[C_SDF];
        st->voxel_segments = k[C_VOX];
        st->trace_steps = k[C_STEPS];
        st->scatters = k[C_SCAT];
        st->fresnel_events = k[C_FRES];
        st->reflections = k[C_REFL];
        st->kills_step_cap = k[C_STEPCAP];
        st->kills_error = k[C_ERR];
        st->rng_draws = k[C_DRAWS];
        st->variance_overflows = k[C_VAROVF];
        for (int i = 0; i < 24; ++i) st->moments[i] = mom[i];
        st->nscatt = mom[24];
        st->kernel_ms = ms;
        st->device_status = status;
        st->h2d_bytes = param_bytes(c);
        st->d2h_bytes = kCounterBytes;
    }
    if (status & STATUS_ABORTED)
        return fail(SMCRT_ERR_TIMEOUT, "transport kernel reached its time limit and stopped early");
    if (status & (STATUS_STREAM_EXHAUSTED | STATUS_BAD_INDEX))
        return fail(SMCRT_ERR_DEVICE, "device status flag " + std::to_string(status));
    return SMCRT_OK;
}

// Uploads a scene too large for the parameter block (or placed in device memory
// on request): the tables of the transport precision R and the FP64 tables
// (boundary events), bounding spheres included, in one device allocation owned
// by the context.
template <class R>
int upload_scene(smcrt_ctx* c, const smcrt_scene* scene, const smcrt_grid* grid, SceneG<R>& g, SceneG<double>& g64,
                 size_t* total) {
    std::vector<DPrim<R>> pr;
    std::vector<DRegion<R>> rg;
    std::vector<R> bd;
    R margin = 0;
    scene_tables(scene, grid, pr, rg, bd, &margin);
    std::vector<DPrim<double>> pr64;
    std::vector<DRegion<double>> rg64;
    std::vector<double> bd64;
    double margin64 = 0;
    scene_tables(scene, grid, pr64, rg64, bd64, &margin64);
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t o1 = al(sizeof(DPrim<R>) * pr.size()), o2 = o1 + al(sizeof(DRegion<R>) * rg.size()),
                 o3 = o2 + al(sizeof(R) * bd.size()), o4 = o3 + al(sizeof(DPrim<double>) * pr64.size()),
                 o5 = o4 + al(sizeof(DRegion<double>) * rg64.size()), o6 = o5 + al(sizeof(double) * bd64.size());
    std::vector<unsigned char> host(o6, 0);
    std::memcpy(host.data(), pr.data(), sizeof(DPrim<R>) * pr.size());
    std::memcpy(host.data() + o1, rg.data(), sizeof(DRegion<R>) * rg.size());
    std::memcpy(host.data() + o2, bd.data(), sizeof(R) * bd.size());
    std::memcpy(host.data() + o3, pr64.data(), sizeof(DPrim<double>) * pr64.size());
    std::memcpy(host.data() + o4, rg64.data(), sizeof(DRegion<double>) * rg64.size());
    std::memcpy(host.data() + o5, bd64.data(), sizeof(double) * bd64.size());
    CK(cudaMalloc(&c->d_scene, o6));
    CK(cudaMemcpy(c->d_scene, host.data(), o6, cudaMemcpyHostToDevice));
    unsigned char* d = (unsigned char*)c->d_scene;
    int has_mods = 0;
    for (int i = 0; i < scene->nprims; ++i) has_mods |= scene->prims[i].nmods > 0;
    g.nregions = g64.nregions = scene->nregions;
    g.nprims = g64.nprims = scene->nprims;
    g.has_mods = g64.has_mods = has_mods;
    g.prim = (const DPrim<R>*)d;
    g.region = (const DRegion<R>*)(d + o1);
    g.bound = (const R*)(d + o2);
    g.cull_margin = margin;
    g64.prim = (const DPrim<double>*)(d + o3);
    g64.region = (const DRegion<double>*)(d + o4);
    g64.bound = (const double*)(d + o5);
    g64.cull_margin = margin64;
    *total = o6;
    return SMCRT_OK;
}

// RAII device buffer for the probes.
struct DBuf {
    void* p = nullptr;
    ~DBuf() {
        if (p) cudaFree(p);
    }
};

int upload(DBuf& b, const void* h, size_t bytes) {
    CK(cudaMalloc(&b.p, bytes ? bytes : 8));
    if (h && bytes) CK(cudaMemcpy(b.p, h, bytes, cudaMemcpyHostToDevice));
    return SMCRT_OK;
}

#define UP(buf, ptr, bytes)                          \
    do {                                             \
        int rc_ = upload(buf, ptr, bytes);           \
        if (rc_) return rc_;                         \
    } while (0)

}  // namespace

// ===========================================================================
extern "C" {

int32_t smcrt_abi_version(void) { return SMCRT_ABI_VERSION; }

const char* smcrt_last_error(void) { return g_err.c_str(); }

int32_t smcrt_create(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* source,
                     const smcrt_detector* dets, int32_t ndet, const smcrt_options* opts, smcrt_ctx** out) {
    g_err.clear();
    if (!out) return fail(SMCRT_ERR_ARG, "out is null");
    *out = nullptr;
    int rc = validate_scene(scene, false);
    if (rc) return rc;
    rc = validate_optics(scene);
    if (rc) return rc;
    if (!grid || grid->nxg <= 0 || grid->nyg <= 0 || grid->nzg <= 0 || !(grid->xmax > 0) || !(grid->ymax > 0) ||
        !(grid->zmax > 0))
        return fail(SMCRT_ERR_ARG, "grid: need positive voxel counts and half sizes");
    if ((long long)grid->nxg * grid->nyg * grid->nzg > (1ll << 31))
        return fail(SMCRT_ERR_ARG, "grid: more than 2^31 voxels");
    if (!source || source->kind < SMCRT_SRC_POINT || source->kind > SMCRT_SRC_FOCUS)
        return fail(SMCRT_ERR_ARG, "source: unknown kind");
    if (ndet < 0 || ndet > kMaxDetectors || (ndet > 0 && !dets))
        return fail(SMCRT_ERR_ARG, "detectors: 0.." + std::to_string(kMaxDetectors) + " supported");
    if (opts && (opts->scene_memory < 0 || opts->scene_memory > 1))
        return fail(SMCRT_ERR_ARG, "options: scene_memory must be 0 or 1");
    if (opts && (opts->nearest_cache < 0 || opts->nearest_cache > 2))
        return fail(SMCRT_ERR_ARG, "options: nearest_cache must be 0, 1 or 2");
    if (opts && (opts->shared_fluence < 0 || opts->shared_fluence > 2))
        return fail(SMCRT_ERR_ARG, "options: shared_fluence must be 0, 1 or 2");
    const bool big = scene->nregions > kMaxRegions || scene->nprims > kMaxPrims || (opts && opts->scene_memory == 1);
    const int prec = opts ? opts->precision : SMCRT_FP32;
    const int kern = opts ? opts->kernel : SMCRT_KERNEL_PATHLENGTH;
    if (prec != SMCRT_FP32 && prec != SMCRT_FP64) return fail(SMCRT_ERR_ARG, "options: unknown precision");
    if (kern < SMCRT_KERNEL_PATHLENGTH || kern > SMCRT_KERNEL_TEST) return fail(SMCRT_ERR_ARG, "options: unknown kernel");
    if (check_steps(opts)) return SMCRT_ERR_ARG;
    DetT dtab[kMaxDetectors];
    long long nbins = 0;
    rc = fill_dets(dtab, dets, ndet, scene->nregions, nbins);
    if (rc) return rc;

    smcrt_ctx* c = new smcrt_ctx;
    rc = pick_device(c->device, c->nsm);
    if (rc) {
        delete c;
        return rc;
    }
    c->precision = prec;
    c->kernel = kern;
    c->ncell = (long long)grid->nxg * grid->nyg * grid->nzg;
    c->nbins = nbins;
    c->block = (opts && opts->block_size > 0) ? opts->block_size : kBlock;
    if (c->block != kBlock) {
        delete c;
        return fail(SMCRT_ERR_ARG, "options: block_size must be 0 or " + std::to_string(kBlock));
    }
    c->timeout_ms = (opts && opts->timeout_ms > 0) ? opts->timeout_ms : 600000;
    if (prec == SMCRT_FP64) c->pd = make_params<double>(scene, grid, source, dtab, ndet, opts);
    else c->pf = make_params<float>(scene, grid, source, dtab, ndet, opts);
    {
        double margin;
        c->cache_allowed = cache_policy(scene, grid, prec == SMCRT_FP64 ? 8 : 4, &margin);
    }
    // the privatised fluence sub-box of a pencil beam: 8 x 8 cells around the
    // entry cell across the beam, along it from the entry through the grid
    if (prec == SMCRT_FP32 && source->kind == SMCRT_SRC_PENCIL) {
        const double mx[3] = {grid->xmax, grid->ymax, grid->zmax};
        const int n[3] = {grid->nxg, grid->nyg, grid->nzg};
        int cell[3], axis = 0;
        for (int a = 0; a < 3; ++a) {
            const int ca = (int)std::floor((source->pos[a] + mx[a]) * n[a] / (2.0 * mx[a]));
            cell[a] = std::min(std::max(ca, 0), n[a] - 1);
            if (std::fabs(source->dir[a]) > std::fabs(source->dir[axis])) axis = a;
        }
        c->priv_axis = axis;
        c->priv_sign = source->dir[axis] > 0 ? 1 : -1;
        for (int a = 0; a < 3; ++a) {
            if (a == axis) {
                c->priv_o[a] = c->priv_sign > 0 ? cell[a] : 0;
                c->priv_d[a] = c->priv_sign > 0 ? n[a] - cell[a] : cell[a] + 1;
            } else {
                c->priv_d[a] = std::min(8, n[a]);
                c->priv_o[a] = std::min(std::max(cell[a] - c->priv_d[a] / 2, 0), n[a] - c->priv_d[a]);
            }
        }
        c->priv_allowed = true;
        c->priv_on = opts && opts->shared_fluence == 1;
    }

    auto bail = [&](int code) {
        smcrt_destroy(c);
        return code;
    };
#define CKC(call)                                                                                      \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return bail(fail(SMCRT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_))); \
    } while (0)
    if (opts && opts->private_stream) {
        CKC(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    } else {
        c->stream = opts ? (cudaStream_t)opts->stream : (cudaStream_t)0;
    }
    CKC(cudaMalloc(&c->d_jmean, sizeof(double) * c->ncell));
    rc = tally_copies(opts, c->ncell, &c->tcopies);
    if (rc) return bail(rc);
    if (c->tcopies > 1) {
        const size_t bytes = sizeof(double) * (size_t)(c->tcopies - 1) * (size_t)c->ncell;
        CKC(cudaMalloc(&c->d_copies, bytes));
        CKC(cudaMemset(c->d_copies, 0, bytes));  // the reduce kernel re-zeroes after each launch
    }
    c->copies_alloc = c->tcopies;
    CKC(cudaMalloc(&c->d_bins, sizeof(double) * std::max(1ll, nbins)));
    CKC(cudaMalloc(&c->d_work, sizeof(unsigned long long) * (1 + C_NUM)));
    CKC(cudaMalloc(&c->d_mom, sizeof(double) * 25));
    CKC(cudaMalloc(&c->d_status, sizeof(int)));
    CKC(cudaEventCreate(&c->ev0));
    CKC(cudaEventCreate(&c->ev1));
    if (big) {
        // the scene in device memory: transport-precision tables, then FP64 tables
        c->big = true;
        size_t bytes = 0;
        if (prec == SMCRT_FP64) rc = upload_scene<double>(c, scene, grid, c->pd->gsc, c->pd->gsc64, &bytes);
        else rc = upload_scene<float>(c, scene, grid, c->pf->gsc, c->pf->gsc64, &bytes);
        if (rc) return bail(rc);
    }
#undef CKC
    rc = occupancy_grid(c, prec, kern, opts ? opts->blocks_per_sm : 0);
    if (rc) return bail(rc);
    if (opts && opts->variance) {
        if (c->big)
            return bail(fail(SMCRT_ERR_ARG, "options: variance needs a scene in the parameter block (at most " +
                                                std::to_string(kMaxRegions) + " regions and " +
                                                std::to_string(kMaxPrims) + " primitives)"));
        c->variance = true;
        const size_t slots = (size_t)(prec == SMCRT_FP64 ? SlotCount<double>::n : SlotCount<float>::n);
        c->vartab_bytes = kVarSlotBytes * slots * (size_t)c->grid_blocks;
        if (cudaMalloc(&c->d_vartab, c->vartab_bytes) != cudaSuccess)
            return bail(fail(SMCRT_ERR_CUDA, "variance: cannot allocate " + std::to_string(c->vartab_bytes >> 20) +
                                                 " MiB of voxel-score tables"));
        if (cudaMalloc(&c->d_jmean2, sizeof(double) * c->ncell) != cudaSuccess)
            return bail(fail(SMCRT_ERR_CUDA, "variance: cannot allocate the second-moment grid"));
    }
    *out = c;
    return SMCRT_OK;
}

void smcrt_destroy(smcrt_ctx* c) {
    if (!c) return;
    cudaStreamSynchronize(c->stream);
    if (c->d_jmean) cudaFree(c->d_jmean);
    if (c->d_copies) cudaFree(c->d_copies);
    if (c->d_bins) cudaFree(c->d_bins);
    if (c->d_work) cudaFree(c->d_work);
    if (c->d_mom) cudaFree(c->d_mom);
    if (c->d_status) cudaFree(c->d_status);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    if (c->d_scene) cudaFree(c->d_scene);
    if (c->d_vartab) cudaFree(c->d_vartab);
    if (c->d_jmean2) cudaFree(c->d_jmean2);
    delete c->pf;
    delete c->pd;
    delete c;
}

int64_t smcrt_detector_bins(const smcrt_ctx* c) { return c ? c->nbins : -1; }

int32_t smcrt_run_device(smcrt_ctx* c, int64_t first, int64_t count, uint64_t seed, double* jmean_dev,
                         double* det_bins_dev, smcrt_stats* stats) {
    g_err.clear();
    if (!c) return fail(SMCRT_ERR_ARG, "ctx is null");
    if (first < 0 || count < 0) return fail(SMCRT_ERR_ARG, "negative packet range");
    if (!jmean_dev || (c->nbins > 0 && !det_bins_dev)) return fail(SMCRT_ERR_ARG, "device buffers are null");
    CK(cudaEventRecord(c->ev0, c->stream));
    int rc = enqueue(c, first, count, seed, jmean_dev, det_bins_dev ? det_bins_dev : c->d_bins, false, nullptr,
                     nullptr, nullptr);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    if (!stats) return SMCRT_OK;
    rc = wait_bounded(c);
    if (rc) return rc;
    return read_stats(c, stats);
}

int32_t smcrt_adjoint(smcrt_ctx* c, int64_t nphotons, uint64_t seed, const float* w_dev, const double* gbins_dev,
                      const int32_t* region_group, int32_t ngroups, double* grad, smcrt_stats* stats) {
    g_err.clear();
    if (!c || nphotons < 0 || !w_dev || !region_group || !grad) return fail(SMCRT_ERR_ARG, "adjoint: bad arguments");
    if (c->precision != SMCRT_FP32 || c->kernel != SMCRT_KERNEL_PATHLENGTH)
        return fail(SMCRT_ERR_ARG, "adjoint: needs an FP32 pathlength context");
    if (c->big)
        return fail(SMCRT_ERR_SCENE, "adjoint: needs a scene of at most " + std::to_string(kMaxRegions) +
                                         " regions and " + std::to_string(kMaxPrims) + " primitives in the "
                                         "parameter block");
    if (ngroups < 1 || ngroups > kMaxAdjGroups)
        return fail(SMCRT_ERR_ARG, "adjoint: 1.." + std::to_string(kMaxAdjGroups) + " parameter groups");
    Params<float>& P = *c->pf;
    for (int r = 0; r < P.sc.nregions; ++r) {
        const int g = region_group[r];
        if (g < -1 || g >= ngroups) return fail(SMCRT_ERR_ARG, "adjoint: region group out of range");
        P.adj_group[r] = g < 0 ? 255 : (unsigned char)g;
    }
    double* d_out = nullptr;
    CK(cudaMalloc(&d_out, sizeof(double) * 3 * (size_t)ngroups));
    auto done = [&](int rc) {
        cudaFree(d_out);
        P.adj_w = nullptr;
        P.adj_gbins = nullptr;
        P.adj_out = nullptr;
        P.adj_ngroups = 0;
        return rc;
    };
    if (cudaMemsetAsync(d_out, 0, sizeof(double) * 3 * (size_t)ngroups, c->stream) != cudaSuccess)
        return done(fail(SMCRT_ERR_CUDA, "adjoint: memset failed"));
    P.adj_w = w_dev;
    P.adj_gbins = gbins_dev;
    P.adj_out = d_out;
    P.adj_ngroups = ngroups;
    P.first = 0;
    P.count = nphotons;
    P.seed = seed;
    P.sbins = 0;
    P.priv_n = 0;  // the adjoint keeps no fluence tally
    set_tally_table(&P, c->d_jmean, c->d_copies, 1, c->ncell);
    if (cudaMemsetAsync(c->d_work, 0, sizeof(unsigned long long) * (1 + C_NUM), c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->d_mom, 0, sizeof(double) * 25, c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream) != cudaSuccess)
        return done(fail(SMCRT_ERR_CUDA, "adjoint: memset failed"));
    Buffers B = make_buffers(c, c->d_jmean, c->d_bins);
    const long long need = (nphotons + kBlock - 1) / kBlock;
    const int blocks = (int)std::min<long long>(c->grid_blocks, std::max<long long>(need, 1));
    if (cudaEventRecord(c->ev0, c->stream) != cudaSuccess) return done(fail(SMCRT_ERR_CUDA, "adjoint: event"));
    cudaError_t e = launch_adjoint_f32_0(P, B, blocks, c->stream);
    if (e != cudaSuccess) return done(fail(SMCRT_ERR_CUDA, std::string("adjoint launch: ") + cudaGetErrorString(e)));
    if (cudaEventRecord(c->ev1, c->stream) != cudaSuccess) return done(fail(SMCRT_ERR_CUDA, "adjoint: event"));
    int rc = wait_bounded(c);
    if (rc) return done(rc);
    if (cudaMemcpy(grad, d_out, sizeof(double) * 3 * (size_t)ngroups, cudaMemcpyDeviceToHost) != cudaSuccess)
        return done(fail(SMCRT_ERR_CUDA, "adjoint: copy failed"));
    rc = read_stats(c, stats);
    return done(rc);
}

int32_t smcrt_autotune(smcrt_ctx* c, int64_t trial_packets, uint64_t seed, smcrt_tuning* result) {
    g_err.clear();
    if (!c || trial_packets < 1) return fail(SMCRT_ERR_ARG, "autotune: bad arguments");
    // candidates: fluence-grid copies 1, 2, 4, 8 (as many as fit in 256 MiB), detector bins
    // in shared memory or not (only when there are bins that fit), the nearest-region
    // cache and the shared fluence sub-box where allowed, and both group orders
    std::vector<int> copies;
    for (int k = 1; k <= 8; k *= 2)
        if (k == 1 || (long long)k * c->ncell * 8 <= (256ll << 20)) copies.push_back(k);
    const int maxc = copies.back();
    if (maxc > c->copies_alloc) {
        CK(cudaStreamSynchronize(c->stream));
        if (c->d_copies) CK(cudaFree(c->d_copies));
        c->d_copies = nullptr;
        const size_t bytes = sizeof(double) * (size_t)(maxc - 1) * (size_t)c->ncell;
        CK(cudaMalloc(&c->d_copies, bytes));
        CK(cudaMemset(c->d_copies, 0, bytes));
        c->copies_alloc = maxc;
    }
    std::vector<int> sbins = {1};
    if (c->nbins > 0 && c->nbins <= kMaxSharedBins) sbins.push_back(0);
    std::vector<int> caches = {0};
    if (c->cache_allowed) caches.push_back(1);
    std::vector<int> privs = {0};
    if (c->priv_allowed) privs.push_back(1);
    const std::vector<int> orders = {SMCRT_ORDER_WALK_LAST, SMCRT_ORDER_INTERACT_LAST};
    auto set_order = [&](int order) {
        if (c->pf) c->pf->group_order = group_order_table(order);
        if (c->pd) c->pd->group_order = group_order_table(order);
    };
    const int keep_tc = c->tcopies;
    const bool keep_sb = c->shared_bins_on;
    auto set_cache = [&](int on) {
        if (c->pf) c->pf->cache_ok = on;
        if (c->pd) c->pd->cache_ok = on;
    };
    double best = -1.0;
    int best_tc = keep_tc, best_sb = keep_sb, best_cache = c->pf ? c->pf->cache_ok : c->pd->cache_ok, trials = 0;
    int best_priv = c->priv_on;
    const unsigned keep_order = c->pf ? c->pf->group_order : c->pd->group_order;
    int best_order = keep_order == kOrderInteractLast ? SMCRT_ORDER_INTERACT_LAST : SMCRT_ORDER_WALK_LAST;
    for (int tc : copies)
        for (int sb : sbins)
          for (int ca : caches)
            for (int pv : privs)
              for (int go : orders) {
            c->tcopies = tc;
            c->shared_bins_on = sb != 0;
            set_cache(ca);
            c->priv_on = pv != 0;
            set_order(go);
            double best_here = 0.0;
            for (int rep = 0; rep < 2; ++rep) {  // best of two: the first may pay cold caches
                CK(cudaMemsetAsync(c->d_jmean, 0, sizeof(double) * c->ncell, c->stream));
                CK(cudaMemsetAsync(c->d_bins, 0, sizeof(double) * std::max(1ll, c->nbins), c->stream));
                CK(cudaEventRecord(c->ev0, c->stream));
                int rc = enqueue(c, 0, trial_packets, seed, c->d_jmean, c->d_bins, false, nullptr, nullptr, nullptr);
                if (rc) return rc;
                CK(cudaEventRecord(c->ev1, c->stream));
                rc = wait_bounded(c);
                if (rc) return rc;
                float ms = 0;
                CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
                best_here = std::max(best_here, (double)trial_packets / (ms * 1e-3));
                ++trials;
            }
            if (best_here > best) {
                best = best_here;
                best_tc = tc;
                best_sb = sb;
                best_cache = ca;
                best_priv = pv;
                best_order = go;
            }
        }
    c->tcopies = best_tc;
    c->shared_bins_on = best_sb != 0;
    set_cache(best_cache);
    c->priv_on = best_priv != 0;
    set_order(best_order);
    if (result) {
        result->tally_copies = best_tc;
        result->shared_bins = best_sb;
        result->packets_per_s = best;
        result->trials = trials;
        result->block_size = c->block;
        result->slots_per_thread =
            c->precision == SMCRT_FP64 ? SlotCount<double>::per_thread : SlotCount<float>::per_thread;
        result->ctas_per_sm = c->grid_blocks / std::max(1, c->nsm);
        result->nearest_cache = best_cache;
        result->shared_fluence = best_priv;
        result->group_order = best_order;
        result->reserved = 0;
    }
    return SMCRT_OK;
}

int32_t smcrt_run(smcrt_ctx* c, int64_t nphotons, uint64_t seed, double* jmean, double* det_bins,
                  smcrt_stats* stats) {
    g_err.clear();
    if (!c) return fail(SMCRT_ERR_ARG, "ctx is null");
    if (nphotons < 0) return fail(SMCRT_ERR_ARG, "nphotons < 0");
    CK(cudaMemsetAsync(c->d_jmean, 0, sizeof(double) * c->ncell, c->stream));
    CK(cudaMemsetAsync(c->d_bins, 0, sizeof(double) * std::max(1ll, c->nbins), c->stream));
    CK(cudaEventRecord(c->ev0, c->stream));
    int rc = enqueue(c, 0, nphotons, seed, c->d_jmean, c->d_bins, false, nullptr, nullptr, nullptr);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    rc = wait_bounded(c);
    if (rc) return rc;
    if (jmean) CK(cudaMemcpyAsync(jmean, c->d_jmean, sizeof(double) * c->ncell, cudaMemcpyDeviceToHost, c->stream));
    if (det_bins && c->nbins > 0)
        CK(cudaMemcpyAsync(det_bins, c->d_bins, sizeof(double) * c->nbins, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    rc = read_stats(c, stats);
    if (stats)
        stats->d2h_bytes += (jmean ? sizeof(double) * (size_t)c->ncell : 0) +
                            (det_bins && c->nbins > 0 ? sizeof(double) * (size_t)c->nbins : 0);
    return rc;
}

int32_t smcrt_run_moments(smcrt_ctx* c, int64_t nphotons, uint64_t seed, double* jmean, double* jmean2,
                          double* det_bins, smcrt_stats* stats) {
    g_err.clear();
    if (!c) return fail(SMCRT_ERR_ARG, "ctx is null");
    if (!c->variance) return fail(SMCRT_ERR_ARG, "moments: the context was created without options.variance");
    if (nphotons < 0) return fail(SMCRT_ERR_ARG, "nphotons < 0");
    CK(cudaMemsetAsync(c->d_jmean, 0, sizeof(double) * c->ncell, c->stream));
    CK(cudaMemsetAsync(c->d_jmean2, 0, sizeof(double) * c->ncell, c->stream));
    CK(cudaMemsetAsync(c->d_bins, 0, sizeof(double) * std::max(1ll, c->nbins), c->stream));
    CK(cudaEventRecord(c->ev0, c->stream));
    int rc = enqueue(c, 0, nphotons, seed, c->d_jmean, c->d_bins, false, nullptr, nullptr, nullptr, c->d_jmean2);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    rc = wait_bounded(c);
    if (rc) return rc;
    if (jmean) CK(cudaMemcpyAsync(jmean, c->d_jmean, sizeof(double) * c->ncell, cudaMemcpyDeviceToHost, c->stream));
    if (jmean2)
        CK(cudaMemcpyAsync(jmean2, c->d_jmean2, sizeof(double) * c->ncell, cudaMemcpyDeviceToHost, c->stream));
    if (det_bins && c->nbins > 0)
        CK(cudaMemcpyAsync(det_bins, c->d_bins, sizeof(double) * c->nbins, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    rc = read_stats(c, stats);
    if (rc == SMCRT_OK) c->vartab_clean = true;
    if (stats)
        stats->d2h_bytes += (jmean ? sizeof(double) * (size_t)c->ncell : 0) +
                            (jmean2 ? sizeof(double) * (size_t)c->ncell : 0) +
                            (det_bins && c->nbins > 0 ? sizeof(double) * (size_t)c->nbins : 0);
    return rc;
}

int32_t smcrt_run_device_moments(smcrt_ctx* c, int64_t first, int64_t count, uint64_t seed, double* jmean_dev,
                                 double* jmean2_dev, double* det_bins_dev, smcrt_stats* stats) {
    g_err.clear();
    if (!c) return fail(SMCRT_ERR_ARG, "ctx is null");
    if (!c->variance) return fail(SMCRT_ERR_ARG, "moments: the context was created without options.variance");
    if (first < 0 || count < 0) return fail(SMCRT_ERR_ARG, "negative packet range");
    if (!jmean_dev || !jmean2_dev || (c->nbins > 0 && !det_bins_dev))
        return fail(SMCRT_ERR_ARG, "device buffers are null");
    CK(cudaEventRecord(c->ev0, c->stream));
    int rc = enqueue(c, first, count, seed, jmean_dev, det_bins_dev ? det_bins_dev : c->d_bins, false, nullptr,
                     nullptr, nullptr, jmean2_dev);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    if (!stats) return SMCRT_OK;
    rc = wait_bounded(c);
    if (rc) return rc;
    rc = read_stats(c, stats);
    if (rc == SMCRT_OK) c->vartab_clean = true;
    return rc;
}

int32_t smcrt_replay(smcrt_ctx* c, const double* uniforms, const int64_t* offsets, int64_t npackets, double* jmean,
                     double* det_bins, smcrt_packet_state* states, smcrt_stats* stats) {
    g_err.clear();
    if (!c || !uniforms || !offsets || npackets < 0) return fail(SMCRT_ERR_ARG, "replay: bad arguments");
    for (int64_t p = 0; p < npackets; ++p)
        if (offsets[p + 1] < offsets[p]) return fail(SMCRT_ERR_ARG, "replay: offsets must be non-decreasing");
    const size_t nu = (size_t)offsets[npackets];
    DBuf du, doff, dst;
    UP(du, uniforms, sizeof(double) * nu);
    UP(doff, offsets, sizeof(int64_t) * (npackets + 1));
    UP(dst, nullptr, sizeof(smcrt_packet_state) * std::max<int64_t>(npackets, 1));
    CK(cudaMemsetAsync(c->d_jmean, 0, sizeof(double) * c->ncell, c->stream));
    CK(cudaMemsetAsync(c->d_bins, 0, sizeof(double) * std::max(1ll, c->nbins), c->stream));
    CK(cudaEventRecord(c->ev0, c->stream));
    int rc = enqueue(c, 0, npackets, 0, c->d_jmean, c->d_bins, true, (const double*)du.p, (const long long*)doff.p,
                     (smcrt_packet_state*)dst.p);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    rc = wait_bounded(c);
    if (rc) return rc;
    if (jmean) CK(cudaMemcpy(jmean, c->d_jmean, sizeof(double) * c->ncell, cudaMemcpyDeviceToHost));
    if (det_bins && c->nbins > 0) CK(cudaMemcpy(det_bins, c->d_bins, sizeof(double) * c->nbins, cudaMemcpyDeviceToHost));
    if (states) CK(cudaMemcpy(states, dst.p, sizeof(smcrt_packet_state) * npackets, cudaMemcpyDeviceToHost));
    rc = read_stats(c, stats);
    if (stats) {
        stats->h2d_bytes += sizeof(double) * nu + sizeof(int64_t) * (npackets + 1);
        stats->d2h_bytes += (jmean ? sizeof(double) * (size_t)c->ncell : 0) +
                            (det_bins && c->nbins > 0 ? sizeof(double) * (size_t)c->nbins : 0) +
                            (states ? sizeof(smcrt_packet_state) * (size_t)npackets : 0);
    }
    return rc;
}

}  // extern "C"

// ===========================================================================
// Batches: instances of one scene geometry, each with its own region optics,
// packet count and seed, transported in ONE persistent launch.  The kernel maps
// a launch packet id to (instance, instance packet id) through a prefix table
// in device memory, so packet counts and seeds are data: a captured CUDA graph
// stays valid when they change.
struct smcrt_batch {
    int device = 0, nsm = 0, precision = SMCRT_FP32, kernel = SMCRT_KERNEL_PATHLENGTH;
    int ninst = 0, grid_blocks = 0, timeout_ms = 600000;
    long long ncell = 0, nbins = 0;
    cudaStream_t stream = nullptr;
    Params<float>* pf = nullptr;
    Params<double>* pd = nullptr;
    std::vector<smcrt_region> regions;  // the base scene, for smcrt_batch_set_optics
    std::vector<smcrt_prim> prims;
    double* d_jm = nullptr;
    double* d_bins = nullptr;
    void* d_opt = nullptr;
    long long* d_prefix = nullptr;
    unsigned long long* d_seed = nullptr;
    unsigned long long* d_bstats = nullptr;
    unsigned long long* d_work = nullptr;  // [0] work, [1..C_NUM] counters
    double* d_mom = nullptr;
    int* d_status = nullptr;
    long long* h_prefix = nullptr;          // pinned staging of the tables
    unsigned long long* h_seed = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool pending = false;
};

namespace {

template <class R>
void optics_of(const SceneT<R>& sc, const SceneT<double>& sc64, InstOptics<R>& o) {
    std::memset(&o, 0, sizeof(o));
    for (int r = 0; r < sc.nregions; ++r) {
        o.kappa[r] = sc.region[r].kappa;
        o.albedo[r] = sc.region[r].albedo;
        o.hgg[r] = sc.region[r].hgg;
        o.g2[r] = sc.region[r].g2;
        o.nidx[r] = sc.region[r].nidx;
        o.nidx64[r] = sc64.region[r].nidx;
    }
}

template <class R>
Params<R>* batch_params(smcrt_batch* b);
template <>
Params<float>* batch_params<float>(smcrt_batch* b) { return b->pf; }
template <>
Params<double>* batch_params<double>(smcrt_batch* b) { return b->pd; }

// Device buffers and tables of a batch whose parameters (b->pf or b->pd) are set.
template <class R>
int batch_alloc(smcrt_batch* b) {
    CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CK(cudaMalloc(&b->d_jm, sizeof(double) * (size_t)b->ninst * (size_t)b->ncell));
    CK(cudaMalloc(&b->d_bins, sizeof(double) * (size_t)std::max(1ll, b->ninst * b->nbins)));
    CK(cudaMalloc(&b->d_opt, sizeof(InstOptics<R>) * (size_t)b->ninst));
    CK(cudaMalloc(&b->d_prefix, sizeof(long long) * (size_t)(b->ninst + 1)));
    CK(cudaMalloc(&b->d_seed, sizeof(unsigned long long) * (size_t)b->ninst));
    CK(cudaMalloc(&b->d_bstats, sizeof(unsigned long long) * 3 * (size_t)b->ninst));
    CK(cudaMalloc(&b->d_work, sizeof(unsigned long long) * (1 + C_NUM)));
    CK(cudaMalloc(&b->d_mom, sizeof(double) * 25));
    CK(cudaMalloc(&b->d_status, sizeof(int)));
    CK(cudaMallocHost(&b->h_prefix, sizeof(long long) * (size_t)(b->ninst + 1)));
    CK(cudaMallocHost(&b->h_seed, sizeof(unsigned long long) * (size_t)b->ninst));
    CK(cudaEventCreate(&b->ev0));
    CK(cudaEventCreate(&b->ev1));
    Params<R>* P = batch_params<R>(b);
    P->bopt = (const InstOptics<R>*)b->d_opt;
    P->bprefix = b->d_prefix;
    P->bseed = b->d_seed;
    P->bstats = b->d_bstats;
    P->ninst = b->ninst;
    P->nbins = b->nbins;
    P->sbins = 0;
    P->tcopies = 1;
    P->tmask = 0;
    P->ncell = b->ncell;
    for (int k = 0; k < kMaxTallyCopies; ++k) P->jtab[k] = k == 0 ? b->d_jm : nullptr;
    P->first = 0;
    P->count = 0;
    int per_sm = 0;
    int rc = resident_per_sm(b->precision, b->kernel, kBlock, 0, 0, &per_sm);
    if (rc) return rc;
    b->grid_blocks = b->nsm * per_sm;
    // set the kernel's shared-memory limit now, outside any stream capture
    cudaError_t e = b->precision == SMCRT_FP64
                        ? (b->kernel == SMCRT_KERNEL_WEIGHT ? launch_batch_f64_1(*b->pd, Buffers{}, 0, b->stream)
                                                            : launch_batch_f64_0(*b->pd, Buffers{}, 0, b->stream))
                        : (b->kernel == SMCRT_KERNEL_WEIGHT ? launch_batch_f32_1(*b->pf, Buffers{}, 0, b->stream)
                                                            : launch_batch_f32_0(*b->pf, Buffers{}, 0, b->stream));
    if (e != cudaSuccess && e != cudaErrorInvalidConfiguration)
        return fail(SMCRT_ERR_CUDA, std::string("batch kernel set-up: ") + cudaGetErrorString(e));
    cudaGetLastError();
    return SMCRT_OK;
}

template <class R>
int batch_upload_optics(smcrt_batch* b, const std::vector<InstOptics<R>>& o) {
    CK(cudaMemcpyAsync(b->d_opt, o.data(), sizeof(InstOptics<R>) * o.size(), cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    return SMCRT_OK;
}

// The launch sequence: tables in, tallies and counters zeroed, the kernel.
int batch_enqueue(smcrt_batch* b) {
    cudaStream_t s = b->stream;
    CK(cudaMemcpyAsync(b->d_prefix, b->h_prefix, sizeof(long long) * (size_t)(b->ninst + 1), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(b->d_seed, b->h_seed, sizeof(unsigned long long) * (size_t)b->ninst, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(b->d_jm, 0, sizeof(double) * (size_t)b->ninst * (size_t)b->ncell, s));
    CK(cudaMemsetAsync(b->d_bins, 0, sizeof(double) * (size_t)std::max(1ll, b->ninst * b->nbins), s));
    CK(cudaMemsetAsync(b->d_bstats, 0, sizeof(unsigned long long) * 3 * (size_t)b->ninst, s));
    CK(cudaMemsetAsync(b->d_work, 0, sizeof(unsigned long long) * (1 + C_NUM), s));
    CK(cudaMemsetAsync(b->d_mom, 0, sizeof(double) * 25, s));
    CK(cudaMemsetAsync(b->d_status, 0, sizeof(int), s));
    Buffers B{};
    B.jmean = b->d_jm;
    B.bins = b->d_bins;
    B.work = b->d_work;
    B.counters = b->d_work + 1;
    B.moments = b->d_mom;
    B.status = b->d_status;
    cudaError_t e;
    if (b->precision == SMCRT_FP64)
        e = b->kernel == SMCRT_KERNEL_WEIGHT ? launch_batch_f64_1(*b->pd, B, b->grid_blocks, s)
                                             : launch_batch_f64_0(*b->pd, B, b->grid_blocks, s);
    else
        e = b->kernel == SMCRT_KERNEL_WEIGHT ? launch_batch_f32_1(*b->pf, B, b->grid_blocks, s)
                                             : launch_batch_f32_0(*b->pf, B, b->grid_blocks, s);
    if (e != cudaSuccess) return fail(SMCRT_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    return SMCRT_OK;
}

int batch_wait(smcrt_batch* b) {
    auto t0 = std::chrono::steady_clock::now();
    const double limit = (double)b->timeout_ms + 30000.0;
    for (;;) {
        cudaError_t e = cudaEventQuery(b->ev1);
        if (e == cudaSuccess) return SMCRT_OK;
        if (e != cudaErrorNotReady) return fail(SMCRT_ERR_CUDA, std::string("batch kernel: ") + cudaGetErrorString(e));
        double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms > limit) return fail(SMCRT_ERR_TIMEOUT, "batch kernel did not finish within its time limit");
        poll_sleep(ms);
    }
}

void batch_free(smcrt_batch* b) {
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_jm);
    cudaFree(b->d_bins);
    cudaFree(b->d_opt);
    cudaFree(b->d_prefix);
    cudaFree(b->d_seed);
    cudaFree(b->d_bstats);
    cudaFree(b->d_work);
    cudaFree(b->d_mom);
    cudaFree(b->d_status);
    if (b->h_prefix) cudaFreeHost(b->h_prefix);
    if (b->h_seed) cudaFreeHost(b->h_seed);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b->pf;
    delete b->pd;
    delete b;
}

// Per-instance optics of a batch from `ninst` scenes that differ from the base
// scene only in their region optics (converted as smcrt_create converts them).
template <class R>
int batch_optics_from_regions(smcrt_batch* b, const smcrt_region_optics* optics) {
    const int nr = (int)b->regions.size();
    std::vector<InstOptics<R>> o((size_t)b->ninst);
    std::vector<smcrt_region> regs(b->regions);
    smcrt_scene sc{nr, (int32_t)b->prims.size(), regs.data(), b->prims.data()};
    SceneT<R>* s1 = new SceneT<R>;
    SceneT<double>* s2 = new SceneT<double>;
    for (int i = 0; i < b->ninst; ++i) {
        for (int r = 0; r < nr; ++r) {
            if (optics) {
                const smcrt_region_optics& q = optics[(size_t)i * nr + r];
                regs[r].mus = q.mus;
                regs[r].mua = q.mua;
                regs[r].hgg = q.hgg;
                regs[r].n = q.n;
            }
        }
        int rc = validate_optics(&sc);
        if (rc) {
            delete s1;
            delete s2;
            return fail(rc, "batch instance " + std::to_string(i) + ": " + g_err);
        }
        fill_scene(*s1, &sc);
        fill_scene(*s2, &sc);
        optics_of(*s1, *s2, o[(size_t)i]);
    }
    delete s1;
    delete s2;
    return batch_upload_optics<R>(b, o);
}

int batch_set_counts(smcrt_batch* b, const int64_t* nphotons, const uint64_t* seeds) {
    if (!nphotons || !seeds) return fail(SMCRT_ERR_ARG, "batch: nphotons and seeds are required");
    long long acc = 0;
    b->h_prefix[0] = 0;
    for (int i = 0; i < b->ninst; ++i) {
        if (nphotons[i] < 0) return fail(SMCRT_ERR_ARG, "batch: negative packet count");
        acc += nphotons[i];
        b->h_prefix[i + 1] = acc;
        b->h_seed[i] = seeds[i];
    }
    return SMCRT_OK;
}

}  // namespace

extern "C" {

int32_t smcrt_batch_create(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* source,
                           const smcrt_detector* dets, int32_t ndet, const smcrt_options* opts, int32_t ninst,
                           smcrt_batch** out) {
    g_err.clear();
    if (!out) return fail(SMCRT_ERR_ARG, "out is null");
    *out = nullptr;
    if (ninst < 1 || ninst > (1 << 18) - 1) return fail(SMCRT_ERR_ARG, "batch: ninst must be 1..262143");
    int rc = validate_scene(scene);
    if (rc) return rc;
    rc = validate_optics(scene);
    if (rc) return rc;
    if (!grid || grid->nxg <= 0 || grid->nyg <= 0 || grid->nzg <= 0 || !(grid->xmax > 0) || !(grid->ymax > 0) ||
        !(grid->zmax > 0))
        return fail(SMCRT_ERR_ARG, "grid: need positive voxel counts and half sizes");
    if (!source || source->kind < SMCRT_SRC_POINT || source->kind > SMCRT_SRC_FOCUS)
        return fail(SMCRT_ERR_ARG, "source: unknown kind");
    if (ndet < 0 || ndet > kMaxDetectors || (ndet > 0 && !dets))
        return fail(SMCRT_ERR_ARG, "detectors: 0.." + std::to_string(kMaxDetectors) + " supported");
    const int prec = opts ? opts->precision : SMCRT_FP32;
    const int kern = opts ? opts->kernel : SMCRT_KERNEL_PATHLENGTH;
    if (prec != SMCRT_FP32 && prec != SMCRT_FP64) return fail(SMCRT_ERR_ARG, "options: unknown precision");
    if (kern != SMCRT_KERNEL_PATHLENGTH && kern != SMCRT_KERNEL_WEIGHT)
        return fail(SMCRT_ERR_ARG, "batch: pathlength and weight kernels only");
    if (opts && opts->block_size > 0 && opts->block_size != kBlock)
        return fail(SMCRT_ERR_ARG, "options: block_size must be 0 or " + std::to_string(kBlock));
    if (check_steps(opts)) return SMCRT_ERR_ARG;
    DetT dtab[kMaxDetectors];
    long long nbins = 0;
    rc = fill_dets(dtab, dets, ndet, scene->nregions, nbins);
    if (rc) return rc;
    smcrt_batch* b = new smcrt_batch;
    rc = pick_device(b->device, b->nsm);
    if (rc) {
        delete b;
        return rc;
    }
    b->precision = prec;
    b->kernel = kern;
    b->ninst = ninst;
    b->ncell = (long long)grid->nxg * grid->nyg * grid->nzg;
    b->nbins = nbins;
    b->timeout_ms = (opts && opts->timeout_ms > 0) ? opts->timeout_ms : 600000;
    b->regions.assign(scene->regions, scene->regions + scene->nregions);
    b->prims.assign(scene->prims, scene->prims + scene->nprims);
    if (prec == SMCRT_FP64) b->pd = make_params<double>(scene, grid, source, dtab, ndet, opts);
    else b->pf = make_params<float>(scene, grid, source, dtab, ndet, opts);
    rc = prec == SMCRT_FP64 ? batch_alloc<double>(b) : batch_alloc<float>(b);
    if (!rc) rc = prec == SMCRT_FP64 ? batch_optics_from_regions<double>(b, nullptr)
                                     : batch_optics_from_regions<float>(b, nullptr);
    if (rc) {
        batch_free(b);
        return rc;
    }
    *out = b;
    return SMCRT_OK;
}

int32_t smcrt_batch_set_optics(smcrt_batch* b, const smcrt_region_optics* optics) {
    g_err.clear();
    if (!b || !optics) return fail(SMCRT_ERR_ARG, "batch_set_optics: null argument");
    if (b->pending) {
        int rc = batch_wait(b);
        if (rc) return rc;
    }
    return b->precision == SMCRT_FP64 ? batch_optics_from_regions<double>(b, optics)
                                      : batch_optics_from_regions<float>(b, optics);
}

int32_t smcrt_batch_launch(smcrt_batch* b, const int64_t* nphotons, const uint64_t* seeds, int32_t use_graph) {
    g_err.clear();
    if (!b) return fail(SMCRT_ERR_ARG, "batch is null");
    if (b->pending) {  // the staging buffers feed the previous launch until it ends
        int rc = batch_wait(b);
        if (rc) return rc;
    }
    int rc = batch_set_counts(b, nphotons, seeds);
    if (rc) return rc;
    CK(cudaEventRecord(b->ev0, b->stream));
    if (use_graph) {
        if (!b->exec) {
            CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            rc = batch_enqueue(b);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(b->stream, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return fail(SMCRT_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(e));
            b->graph = g;
            CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
        }
        CK(cudaGraphLaunch(b->exec, b->stream));
    } else {
        rc = batch_enqueue(b);
        if (rc) return rc;
    }
    CK(cudaEventRecord(b->ev1, b->stream));
    b->pending = true;
    return SMCRT_OK;
}

int32_t smcrt_batch_wait(smcrt_batch* b, double* jmean, double* det_bins, smcrt_stats* per_instance,
                         smcrt_stats* total) {
    g_err.clear();
    if (!b) return fail(SMCRT_ERR_ARG, "batch is null");
    if (!b->pending) return fail(SMCRT_ERR_ARG, "batch_wait: nothing launched");
    int rc = batch_wait(b);
    if (rc) return rc;
    b->pending = false;
    if (jmean)
        CK(cudaMemcpy(jmean, b->d_jm, sizeof(double) * (size_t)b->ninst * (size_t)b->ncell, cudaMemcpyDeviceToHost));
    if (det_bins && b->nbins > 0)
        CK(cudaMemcpy(det_bins, b->d_bins, sizeof(double) * (size_t)b->ninst * (size_t)b->nbins,
                      cudaMemcpyDeviceToHost));
    unsigned long long cnt[1 + C_NUM];
    double mom[25];
    int status = 0;
    CK(cudaMemcpy(cnt, b->d_work, sizeof(cnt), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(mom, b->d_mom, sizeof(mom), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&status, b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    if (per_instance) {
        std::vector<unsigned long long> bs(3 * (size_t)b->ninst);
        CK(cudaMemcpy(bs.data(), b->d_bstats, sizeof(unsigned long long) * bs.size(), cudaMemcpyDeviceToHost));
        for (int i = 0; i < b->ninst; ++i) {
            smcrt_stats& st = per_instance[i];
            std::memset(&st, 0, sizeof(st));
            st.packets = bs[3 * (size_t)i];
            st.rng_draws = bs[3 * (size_t)i + 1];
            st.nscatt = (double)bs[3 * (size_t)i + 2];
            st.kernel_ms = ms;
            st.device_status = status;
        }
    }
    if (total) {
        std::memset(total, 0, sizeof(*total));
        const unsigned long long* k = cnt + 1;
        total->packets = k[C_PACKETS];
        total->sdf_evals = k[C_SDF];
        total->voxel_segments = k[C_VOX];
        total->trace_steps = k[C_STEPS];
        total->scatters = k[C_SCAT];
        total->fresnel_events = k[C_FRES];
        total->reflections = k[C_REFL];
        total->kills_step_cap = k[C_STEPCAP];
        total->kills_error = k[C_ERR];
        total->rng_draws = k[C_DRAWS];
        total->nscatt = mom[24];
        total->kernel_ms = ms;
        total->device_status = status;
    }
    if (status & STATUS_ABORTED) return fail(SMCRT_ERR_TIMEOUT, "batch kernel reached its time limit and stopped early");
    if (status & (STATUS_STREAM_EXHAUSTED | STATUS_BAD_INDEX))
        return fail(SMCRT_ERR_DEVICE, "device status flag " + std::to_string(status));
    return SMCRT_OK;
}

int32_t smcrt_batch_device_tallies(smcrt_batch* b, double** jmean_dev, double** det_bins_dev) {
    g_err.clear();
    if (!b) return fail(SMCRT_ERR_ARG, "batch is null");
    if (jmean_dev) *jmean_dev = b->d_jm;
    if (det_bins_dev) *det_bins_dev = b->d_bins;
    return SMCRT_OK;
}

int64_t smcrt_batch_stream(const smcrt_batch* b) { return b ? (int64_t)(intptr_t)b->stream : 0; }

void smcrt_batch_destroy(smcrt_batch* b) {
    if (b) batch_free(b);
}

}  // extern "C"

namespace {

// The scene geometry, grid, source, detectors and run options of two contexts'
// parameter blocks are equal (region optics may differ).
template <class R>
bool same_geometry(const Params<R>& a, const Params<R>& b) {
    if (a.sc.nregions != b.sc.nregions || a.sc.nprims != b.sc.nprims) return false;
    if (std::memcmp(a.sc.prim, b.sc.prim, sizeof(a.sc.prim[0]) * (size_t)a.sc.nprims)) return false;
    for (int r = 0; r < a.sc.nregions; ++r) {
        const DRegion<R>&x = a.sc.region[r], &y = b.sc.region[r];
        if (x.first != y.first || x.n != y.n || x.op != y.op || x.k != y.k) return false;
    }
    return !std::memcmp(&a.grid, &b.grid, sizeof(a.grid)) && !std::memcmp(&a.src, &b.src, sizeof(a.src)) &&
           a.ndet == b.ndet && !std::memcmp(a.det, b.det, sizeof(a.det[0]) * (size_t)a.ndet) &&
           a.kernel == b.kernel && a.end_early == b.end_early && a.max_steps == b.max_steps && a.eps == b.eps &&
           a.normal_h == b.normal_h && a.instance == b.instance;
}

template <class R>
const Params<R>* ctx_params(const smcrt_ctx* c);
template <>
const Params<float>* ctx_params<float>(const smcrt_ctx* c) { return c->pf; }
template <>
const Params<double>* ctx_params<double>(const smcrt_ctx* c) { return c->pd; }

// One batch launch over contexts that share their geometry; done = false when
// they do not (the caller then runs them one by one).
template <class R>
int run_batched_t(smcrt_ctx* const* ctxs, int32_t ninst, const int64_t* nphotons, const uint64_t* seeds,
                  double* const* jmeans, double* const* det_bins, smcrt_stats* stats, bool& done) {
    done = false;
    const Params<R>* P0 = ctx_params<R>(ctxs[0]);
    if (ctxs[0]->kernel == SMCRT_KERNEL_TEST) return SMCRT_OK;
    for (int i = 0; i < ninst; ++i)
        if (ctxs[i]->big) return SMCRT_OK;  // batches hold their scene in the parameter block
    for (int i = 1; i < ninst; ++i)
        if (ctxs[i]->precision != ctxs[0]->precision || ctxs[i]->device != ctxs[0]->device ||
            !same_geometry(*P0, *ctx_params<R>(ctxs[i])))
            return SMCRT_OK;
    smcrt_batch* b = new smcrt_batch;
    b->device = ctxs[0]->device;
    b->nsm = ctxs[0]->nsm;
    b->precision = ctxs[0]->precision;
    b->kernel = ctxs[0]->kernel;
    b->ninst = ninst;
    b->ncell = ctxs[0]->ncell;
    b->nbins = ctxs[0]->nbins;
    b->timeout_ms = ctxs[0]->timeout_ms;
    if (sizeof(R) == 8) b->pd = new Params<double>(*ctxs[0]->pd);
    else b->pf = new Params<float>(*ctxs[0]->pf);
    int rc = batch_alloc<R>(b);
    if (!rc) {
        std::vector<InstOptics<R>> o((size_t)ninst);
        for (int i = 0; i < ninst; ++i) {
            const Params<R>* Pi = ctx_params<R>(ctxs[i]);
            optics_of(Pi->sc, Pi->sc64, o[(size_t)i]);
        }
        rc = batch_upload_optics<R>(b, o);
    }
    if (!rc) rc = smcrt_batch_launch(b, nphotons, seeds, 0);
    std::vector<smcrt_stats> per((size_t)ninst);
    if (!rc) rc = smcrt_batch_wait(b, nullptr, nullptr, per.data(), nullptr);
    for (int i = 0; !rc && i < ninst; ++i) {
        if (jmeans && jmeans[i])
            if (cudaMemcpy(jmeans[i], b->d_jm + (size_t)i * b->ncell, sizeof(double) * (size_t)b->ncell,
                           cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = fail(SMCRT_ERR_CUDA, "batched: tally copy failed");
        if (!rc && det_bins && det_bins[i] && b->nbins > 0)
            if (cudaMemcpy(det_bins[i], b->d_bins + (size_t)i * b->nbins, sizeof(double) * (size_t)b->nbins,
                           cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = fail(SMCRT_ERR_CUDA, "batched: bin copy failed");
        if (stats) stats[i] = per[(size_t)i];
    }
    batch_free(b);
    done = rc == SMCRT_OK;
    return rc;
}

}  // namespace

extern "C" {

int32_t smcrt_run_batched(smcrt_ctx* const* ctxs, int32_t ninst, const int64_t* nphotons, const uint64_t* seeds,
                          double* const* jmeans, double* const* det_bins, smcrt_stats* stats) {
    g_err.clear();
    if (!ctxs || ninst < 1 || !nphotons || !seeds) return fail(SMCRT_ERR_ARG, "run_batched: bad arguments");
    for (int i = 0; i < ninst; ++i)
        if (!ctxs[i]) return fail(SMCRT_ERR_ARG, "run_batched: null context");
    bool done = false;
    int rc = ctxs[0]->precision == SMCRT_FP64
                 ? run_batched_t<double>(ctxs, ninst, nphotons, seeds, jmeans, det_bins, stats, done)
                 : run_batched_t<float>(ctxs, ninst, nphotons, seeds, jmeans, det_bins, stats, done);
    if (rc || done) return rc;
    // contexts with different geometry (or test kernels): one launch each
    for (int i = 0; i < ninst; ++i) {
        rc = smcrt_run(ctxs[i], nphotons[i], seeds[i], jmeans ? jmeans[i] : nullptr,
                       det_bins ? det_bins[i] : nullptr, stats ? &stats[i] : nullptr);
        if (rc) return rc;
    }
    return SMCRT_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free run.  Some callers cannot allocate device memory at all: host
// applications that own every byte of device memory through their own pool
// allocator, or processes whose device memory is reserved up front for a fixed
// budget, where a library's own cudaMalloc would fail or break the accounting.
// smcrt_run_device_static serves them: it creates no context and calls no
// cudaMalloc/cudaFree.  The transport kernel's scratch (the
// packet-work counter, the event counters, the device status word) lives in the
// file-scope array below, loaded with the library on every GPU that uses it and
// held until the process exits.  Every call shares this one array, so calls that
// overlap on the GPU (different streams or threads) race on it.
}  // extern "C"

namespace {

constexpr size_t kStaticScratchBytes = 4096;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Scratch layout: [work u64][C_NUM counters u64][25 moments f64][status i32].
constexpr size_t kScratchCounters = sizeof(unsigned long long) * (1 + C_NUM);
constexpr size_t kScratchMoments = sizeof(double) * 25;
constexpr size_t kScratchNeeded = kScratchCounters + kScratchMoments + sizeof(int);

constexpr int kMaxDevices = 64;
unsigned char* g_scratch_dev[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of the static scratch on the current device, resolved once per
// device (the host-side name g_static_scratch is not a device address).
int static_scratch(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(SMCRT_ERR_ARG, "static run: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
            return fail(SMCRT_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
        g_scratch_dev[dev] = (unsigned char*)p;
    }
    *out = g_scratch_dev[dev];
    return SMCRT_OK;
}

template <class R>
int run_static_t(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* source,
                 const smcrt_detector* dets, int32_t ndet, const smcrt_options* opts, long long first,
                 long long count, uint64_t seed, double* jmean_dev, double* bins_dev, smcrt_stats* stats) {
    DetT dtab[kMaxDetectors];
    long long nbins = 0;
    int rc = fill_dets(dtab, dets, ndet, scene->nregions, nbins);
    if (rc) return rc;
    if (nbins > 0 && !bins_dev) return fail(SMCRT_ERR_ARG, "static run: detector bins buffer is null");
    int dev = 0, nsm = 0;
    rc = pick_device(dev, nsm);
    if (rc) return rc;
    unsigned char* scratch = nullptr;
    rc = static_scratch(dev, &scratch);
    if (rc) return rc;
    const int kern = opts ? opts->kernel : SMCRT_KERNEL_PATHLENGTH;
    const int block = (opts && opts->block_size > 0) ? opts->block_size : kBlock;
    if (block != kBlock) return fail(SMCRT_ERR_ARG, "options: block_size must be 0 or " + std::to_string(kBlock));
    // the launch parameters live on this host stack (no heap, no device memory)
    Params<R> P;
    fill_params(&P, scene, grid, source, dtab, ndet, opts);
    P.first = first;
    P.count = count;
    P.seed = seed;
    P.sbins = shared_bins(nbins, count);
    P.jtab[0] = jmean_dev;  // one fluence grid: no copies without allocation
    int per_sm = 0;
    cudaError_t e;
    rc = resident_per_sm(sizeof(R) == 8 ? SMCRT_FP64 : SMCRT_FP32, kern, block, sizeof(unsigned) * (size_t)P.sbins,
                         opts ? opts->blocks_per_sm : 0, &per_sm);
    if (rc) return rc;
    const long long need = (count + block - 1) / block;
    const int blocks = (int)std::min<long long>((long long)nsm * per_sm, std::max<long long>(need, 1));
    cudaStream_t s = opts ? (cudaStream_t)opts->stream : (cudaStream_t)0;
    // the scratch keeps the previous call's values: clear what must start at zero
    CK(cudaMemsetAsync(scratch, 0, kScratchNeeded, s));
    Buffers B;
    B.jmean = jmean_dev;
    B.bins = bins_dev;
    B.work = (unsigned long long*)scratch;
    B.counters = (unsigned long long*)scratch + 1;
    B.moments = (double*)(scratch + kScratchCounters);
    B.status = (int*)(scratch + kScratchCounters + kScratchMoments);
    B.uniforms = nullptr;
    B.offsets = nullptr;
    B.states = nullptr;
    if constexpr (sizeof(R) == 8)
        e = kern == SMCRT_KERNEL_WEIGHT ? launch_f64_1(P, B, false, blocks, block, s)
          : kern == SMCRT_KERNEL_TEST   ? launch_f64_2(P, B, false, blocks, block, s)
                                        : launch_f64_0(P, B, false, blocks, block, s);
    else
        e = kern == SMCRT_KERNEL_WEIGHT ? launch_f32_1(P, B, false, blocks, block, s)
          : kern == SMCRT_KERNEL_TEST   ? launch_f32_2(P, B, false, blocks, block, s)
                                        : launch_f32_0(P, B, false, blocks, block, s);
    if (e != cudaSuccess) return fail(SMCRT_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    if (!stats) return SMCRT_OK;
    // wait with a host-side limit: the kernel's own time budget plus a grace period
    // (a stream query needs no event, so nothing is created)
    {
        const double limit = (double)((opts && opts->timeout_ms > 0) ? opts->timeout_ms : 600000) + 30000.0;
        const auto w0 = std::chrono::steady_clock::now();
        for (;;) {
            const cudaError_t q = cudaStreamQuery(s);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) return fail(SMCRT_ERR_CUDA, std::string("kernel: ") + cudaGetErrorString(q));
            const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
            if (ms > limit) return fail(SMCRT_ERR_TIMEOUT, "transport kernel did not finish within its time limit");
            poll_sleep(ms);
        }
    }
    unsigned long long cnt[1 + C_NUM];
    double mom[25];
    int status = 0;
    CK(cudaMemcpy(cnt, scratch, sizeof(cnt), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(mom, scratch + kScratchCounters, sizeof(mom), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&status, scratch + kScratchCounters + kScratchMoments, sizeof(int), cudaMemcpyDeviceToHost));
    std::memset(stats, 0, sizeof(*stats));
    const unsigned long long* k = cnt + 1;
    stats->packets = k[C_PACKETS];
    stats->sdf_evals = k[C_SDF];
    stats->voxel_segments = k[C_VOX];
    stats->trace_steps = k[C_STEPS];
    stats->scatters = k[C_SCAT];
    stats->fresnel_events = k[C_FRES];
    stats->reflections = k[C_REFL];
    stats->kills_step_cap = k[C_STEPCAP];
    stats->kills_error = k[C_ERR];
    stats->rng_draws = k[C_DRAWS];
    for (int i = 0; i < 24; ++i) stats->moments[i] = mom[i];
    stats->nscatt = mom[24];
    stats->device_status = status;
    if (status & STATUS_ABORTED) return fail(SMCRT_ERR_TIMEOUT, "transport kernel reached its time limit and stopped early");
    return SMCRT_OK;
}

}  // namespace

extern "C" {

int64_t smcrt_static_scratch_bytes(void) { return (int64_t)kStaticScratchBytes; }

int32_t smcrt_run_device_static(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* source,
                                const smcrt_detector* dets, int32_t ndet, const smcrt_options* opts, int64_t first,
                                int64_t count, uint64_t seed, double* jmean_dev, double* det_bins_dev,
                                smcrt_stats* stats) {
    g_err.clear();
    // one run needs the work counter, the event counters, the moments and the
    // status word; the array is sized for that and a larger need is refused
    if (kScratchNeeded > kStaticScratchBytes)
        return fail(SMCRT_ERR_ARG, "static run: the kernel needs " + std::to_string(kScratchNeeded) +
                                       " bytes of scratch, the library's static array holds " +
                                       std::to_string(kStaticScratchBytes));
    int rc = validate_scene(scene);
    if (rc) return rc;
    rc = validate_optics(scene);
    if (rc) return rc;
    if (!grid || grid->nxg <= 0 || grid->nyg <= 0 || grid->nzg <= 0 || !(grid->xmax > 0) || !(grid->ymax > 0) ||
        !(grid->zmax > 0))
        return fail(SMCRT_ERR_ARG, "grid: need positive voxel counts and half sizes");
    if ((long long)grid->nxg * grid->nyg * grid->nzg > (1ll << 31))
        return fail(SMCRT_ERR_ARG, "grid: more than 2^31 voxels");
    if (!source || source->kind < SMCRT_SRC_POINT || source->kind > SMCRT_SRC_FOCUS)
        return fail(SMCRT_ERR_ARG, "source: unknown kind");
    if (ndet < 0 || ndet > kMaxDetectors || (ndet > 0 && !dets))
        return fail(SMCRT_ERR_ARG, "detectors: 0.." + std::to_string(kMaxDetectors) + " supported");
    if (!jmean_dev) return fail(SMCRT_ERR_ARG, "static run: fluence buffer is null");
    if (first < 0 || count < 0) return fail(SMCRT_ERR_ARG, "negative packet range");
    if (opts && opts->kernel != SMCRT_KERNEL_PATHLENGTH && opts->kernel != SMCRT_KERNEL_WEIGHT &&
        opts->kernel != SMCRT_KERNEL_TEST)
        return fail(SMCRT_ERR_ARG, "options: unknown kernel");
    if (check_steps(opts)) return SMCRT_ERR_ARG;
    const int prec = opts ? opts->precision : SMCRT_FP32;
    if (prec == SMCRT_FP64)
        return run_static_t<double>(scene, grid, source, dets, ndet, opts, first, count, seed, jmean_dev, det_bins_dev,
                                    stats);
    if (prec != SMCRT_FP32) return fail(SMCRT_ERR_ARG, "options: unknown precision");
    return run_static_t<float>(scene, grid, source, dets, ndet, opts, first, count, seed, jmean_dev, det_bins_dev,
                               stats);
}

int32_t smcrt_eval_sdf(const smcrt_scene* scene, int32_t precision, const double* pts, int64_t npts, double* out) {
    g_err.clear();
    int rc = validate_scene(scene);
    if (rc) return rc;
    if (!pts || !out || npts < 0) return fail(SMCRT_ERR_ARG, "eval_sdf: bad arguments");
    if (npts == 0) return SMCRT_OK;
    int dev, nsm;
    rc = pick_device(dev, nsm);
    if (rc) return rc;
    DBuf dp, dout;
    UP(dp, pts, sizeof(double) * 3 * npts);
    UP(dout, nullptr, sizeof(double) * npts * scene->nregions);
    CK(probe_eval_sdf(precision, scene, (const double*)dp.p, npts, (double*)dout.p));
    CK(cudaMemcpy(out, dout.p, sizeof(double) * npts * scene->nregions, cudaMemcpyDeviceToHost));
    return SMCRT_OK;
}

int32_t smcrt_calc_normal(const smcrt_scene* scene, int32_t region0, double h, const double* pts, int64_t npts,
                          double* out) {
    g_err.clear();
    int rc = validate_scene(scene);
    if (rc) return rc;
    if (region0 < 0 || region0 >= scene->nregions || !pts || !out || npts < 0)
        return fail(SMCRT_ERR_ARG, "calc_normal: bad arguments");
    if (npts == 0) return SMCRT_OK;
    int dev, nsm;
    rc = pick_device(dev, nsm);
    if (rc) return rc;
    DBuf dp, dout;
    UP(dp, pts, sizeof(double) * 3 * npts);
    UP(dout, nullptr, sizeof(double) * 3 * npts);
    CK(probe_normal(scene, region0, h > 0 ? h : 1e-6, (const double*)dp.p, npts, (double*)dout.p));
    CK(cudaMemcpy(out, dout.p, sizeof(double) * 3 * npts, cudaMemcpyDeviceToHost));
    return SMCRT_OK;
}

static int render_args(const smcrt_scene* scene, int32_t precision, const int32_t* samples, const double* extent,
                       const void* image, long long& total) {
    int rc = validate_scene(scene);
    if (rc) return rc;
    if (!samples || !extent || !image) return fail(SMCRT_ERR_ARG, "render: null pointer");
    if (precision != SMCRT_FP32 && precision != SMCRT_FP64) return fail(SMCRT_ERR_ARG, "render: bad precision");
    total = 1;
    for (int a = 0; a < 3; ++a) {
        if (samples[a] < 1 || samples[a] > 65536) return fail(SMCRT_ERR_ARG, "render: samples out of [1, 65536]");
        if (!std::isfinite(extent[a])) return fail(SMCRT_ERR_ARG, "render: extent not finite");
        total *= samples[a];
    }
    return SMCRT_OK;
}

int32_t smcrt_render(const smcrt_scene* scene, int32_t precision, const int32_t samples[3], const double extent[3],
                     float* image) {
    g_err.clear();
    long long total = 0;
    int rc = render_args(scene, precision, samples, extent, image, total);
    if (rc) return rc;
    int dev, nsm;
    rc = pick_device(dev, nsm);
    if (rc) return rc;
    DBuf dimg;
    UP(dimg, nullptr, sizeof(float) * total);
    CK(launch_render(precision, scene, samples, extent, (float*)dimg.p, nsm, 0));
    CK(cudaMemcpy(image, dimg.p, sizeof(float) * total, cudaMemcpyDeviceToHost));
    return SMCRT_OK;
}

int32_t smcrt_render_device(const smcrt_scene* scene, int32_t precision, const int32_t samples[3],
                            const double extent[3], float* image_dev, void* stream) {
    g_err.clear();
    long long total = 0;
    int rc = render_args(scene, precision, samples, extent, image_dev, total);
    if (rc) return rc;
    int dev, nsm;
    rc = pick_device(dev, nsm);
    if (rc) return rc;
    CK(launch_render(precision, scene, samples, extent, image_dev, nsm, (cudaStream_t)stream));
    return SMCRT_OK;
}

static int fresnel_common(int32_t precision, const double* I, const double* N, const double* n1, const double* n2,
                          const double* u, int64_t n, double* R, double* Iout, int32_t* refl) {
    if (!I || !N || !n1 || !n2 || n < 0) return fail(SMCRT_ERR_ARG, "fresnel: bad arguments");
    if (n == 0) return SMCRT_OK;
    int dev, nsm;
    int rc = pick_device(dev, nsm);
    if (rc) return rc;
    DBuf dI, dN, d1, d2, du, dR, dIo, dr;
    UP(dI, I, sizeof(double) * 3 * n);
    UP(dN, N, sizeof(double) * 3 * n);
    UP(d1, n1, sizeof(double) * n);
    UP(d2, n2, sizeof(double) * n);
    if (u) {
        UP(du, u, sizeof(double) * n);
        UP(dIo, nullptr, sizeof(double) * 3 * n);
        UP(dr, nullptr, sizeof(int) * n);
    }
    if (R) UP(dR, nullptr, sizeof(double) * n);
    CK(probe_fresnel(precision, (const double*)dI.p, (const double*)dN.p, (const double*)d1.p, (const double*)d2.p,
                     (const double*)du.p, n, (double*)dR.p, (double*)dIo.p, (int*)dr.p));
    if (R) CK(cudaMemcpy(R, dR.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (u) {
        CK(cudaMemcpy(Iout, dIo.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(refl, dr.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    }
    return SMCRT_OK;
}

int32_t smcrt_fresnel(int32_t precision, const double* I, const double* N, const double* n1, const double* n2,
                      int64_t n, double* R) {
    g_err.clear();
    if (!R) return fail(SMCRT_ERR_ARG, "fresnel: R is null");
    return fresnel_common(precision, I, N, n1, n2, nullptr, n, R, nullptr, nullptr);
}

int32_t smcrt_reflect_refract(int32_t precision, const double* I, const double* N, const double* n1,
                              const double* n2, const double* u, int64_t n, double* I_out, int32_t* reflected) {
    g_err.clear();
    if (!u || !I_out || !reflected) return fail(SMCRT_ERR_ARG, "reflect_refract: bad arguments");
    return fresnel_common(precision, I, N, n1, n2, u, n, nullptr, I_out, reflected);
}

int32_t smcrt_scatter_dir(int32_t precision, const double* dir_in, const double* g, const double* u, int64_t n,
                          double* dir_out) {
    g_err.clear();
    if (!dir_in || !g || !u || !dir_out || n < 0) return fail(SMCRT_ERR_ARG, "scatter_dir: bad arguments");
    if (n == 0) return SMCRT_OK;
    int dev, nsm;
    int rc = pick_device(dev, nsm);
    if (rc) return rc;
    DBuf dd, dg, du, dout;
    UP(dd, dir_in, sizeof(double) * 3 * n);
    UP(dg, g, sizeof(double) * n);
    UP(du, u, sizeof(double) * 3 * n);
    UP(dout, nullptr, sizeof(double) * 3 * n);
    CK(probe_scatter(precision, (const double*)dd.p, (const double*)dg.p, (const double*)du.p, n, (double*)dout.p));
    CK(cudaMemcpy(dir_out, dout.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
    return SMCRT_OK;
}

int32_t smcrt_emit(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* source, int32_t precision,
                   int64_t first, int64_t npk, uint64_t seed, double* pos, double* dir, int32_t* layer) {
    g_err.clear();
    int rc = validate_scene(scene);
    if (rc) return rc;
    if (!grid || grid->nxg <= 0 || grid->nyg <= 0 || grid->nzg <= 0 || !(grid->xmax > 0) || !(grid->ymax > 0) ||
        !(grid->zmax > 0))
        return fail(SMCRT_ERR_ARG, "grid: need positive voxel counts and half sizes");
    if (!source || source->kind < SMCRT_SRC_POINT || source->kind > SMCRT_SRC_FOCUS)
        return fail(SMCRT_ERR_ARG, "source: unknown kind");
    if (precision != SMCRT_FP32 && precision != SMCRT_FP64) return fail(SMCRT_ERR_ARG, "emit: bad precision");
    if (first < 0 || npk < 0 || !pos || !dir || !layer) return fail(SMCRT_ERR_ARG, "emit: bad arguments");
    if (npk == 0) return SMCRT_OK;
    int dev, nsm;
    rc = pick_device(dev, nsm);
    if (rc) return rc;
    DBuf dp, dd, dl;
    UP(dp, nullptr, sizeof(double) * 3 * npk);
    UP(dd, nullptr, sizeof(double) * 3 * npk);
    UP(dl, nullptr, sizeof(int32_t) * npk);
    if (precision == SMCRT_FP64) {
        std::unique_ptr<Params<double>> P(new Params<double>);
        fill_params(P.get(), scene, grid, source, nullptr, 0, nullptr);
        P->seed = seed;
        CK(probe_emit<double>(*P, first, npk, (double*)dp.p, (double*)dd.p, (int*)dl.p));
    } else {
        std::unique_ptr<Params<float>> P(new Params<float>);
        fill_params(P.get(), scene, grid, source, nullptr, 0, nullptr);
        P->seed = seed;
        CK(probe_emit<float>(*P, first, npk, (double*)dp.p, (double*)dd.p, (int*)dl.p));
    }
    CK(cudaMemcpy(pos, dp.p, sizeof(double) * 3 * npk, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dir, dd.p, sizeof(double) * 3 * npk, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(layer, dl.p, sizeof(int32_t) * npk, cudaMemcpyDeviceToHost));
    return SMCRT_OK;
}

int32_t smcrt_philox(const uint32_t* key2, const uint32_t* ctr4, int64_t n, uint32_t* out4) {
    g_err.clear();
    if (!key2 || !ctr4 || !out4 || n < 0) return fail(SMCRT_ERR_ARG, "philox: bad arguments");
    if (n == 0) return SMCRT_OK;
    int dev, nsm;
    int rc = pick_device(dev, nsm);
    if (rc) return rc;
    DBuf dk, dc, dout;
    UP(dk, key2, sizeof(uint32_t) * 2 * n);
    UP(dc, ctr4, sizeof(uint32_t) * 4 * n);
    UP(dout, nullptr, sizeof(uint32_t) * 4 * n);
    CK(probe_philox((const uint32_t*)dk.p, (const uint32_t*)dc.p, n, (uint32_t*)dout.p));
    CK(cudaMemcpy(out4, dout.p, sizeof(uint32_t) * 4 * n, cudaMemcpyDeviceToHost));
    return SMCRT_OK;
}

}  // extern "C"
