// smcrt_probes.cu -- element-wise kernels that expose the transport's device
// building blocks (SDF evaluation, calcNormal, Fresnel, HG scatter, Philox) for
// parity checks, plus the host-side scene conversion shared with the API.
#include <cmath>
#include <cstring>
#include <vector>

#include "smcrt_launch.h"

namespace smcrt {

template <class R>
void fill_prim(DPrim<R>& d, const smcrt_prim& s) {
    std::memset(&d, 0, sizeof(d));
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 3; ++b) d.m[3 * a + b] = (R)s.transform[a][b];
    for (int a = 0; a < 8; ++a) d.q[a] = (R)s.params[a];
    d.kind = s.kind;
    d.nmods = s.nmods;
    for (int j = 0; j < 2; ++j) {
        d.mod[j] = s.mods[j];
        for (int a = 0; a < 3; ++a) d.mp[j][a] = (R)s.mod_params[j][a];
    }
}

template <class R>
void fill_region(DRegion<R>& r, const smcrt_region& g) {
    std::memset(&r, 0, sizeof(r));
    r.first = g.first_prim;
    r.n = g.nprims;
    r.op = g.op;
    r.k = (R)g.k;
    // init_mono, src/opticalProps/opticalProperties.f90:107-125
    const double kappa = g.mus + g.mua;
    const double albedo = (g.mua < 1e-9) ? 1.0 : g.mus / kappa;
    r.kappa = (R)kappa;
    r.albedo = (R)albedo;
    r.hgg = (R)g.hgg;
    r.g2 = (R)(g.hgg * g.hgg);
    r.nidx = (R)g.n;
    r.mus = (R)g.mus;
    r.mua = (R)g.mua;
}

// A scene larger than the parameter block leaves the block's tables empty (no
// region): such scenes are read from device memory (SceneG) instead.
template <class R>
void fill_scene(SceneT<R>& d, const smcrt_scene* s) {
    std::memset(&d, 0, sizeof(d));
    d.has_mods = 0;
    for (int i = 0; i < s->nprims; ++i) d.has_mods |= s->prims[i].nmods > 0;
    if (s->nregions > kMaxRegions || s->nprims > kMaxPrims) return;
    d.nregions = s->nregions;
    d.nprims = s->nprims;
    for (int i = 0; i < s->nprims; ++i) fill_prim(d.prim[i], s->prims[i]);
    for (int i = 0; i < s->nregions; ++i) fill_region(d.region[i], s->regions[i]);
}

// Bounding sphere of region r in world coordinates, for the sweep's cull
// (sweep_regions): only single primitives without modifiers whose SDF is the
// exact Euclidean distance, under a rigid transform.  Returns false otherwise.
bool region_bound(const smcrt_scene* s, int r, double c[3], double* rad) {
    const smcrt_region& g = s->regions[r];
    if (g.nprims != 1) return false;
    const smcrt_prim& pr = s->prims[g.first_prim];
    if (pr.nmods != 0) return false;
    const double* q = pr.params;
    double cl[3] = {0, 0, 0}, rl = 0;
    auto seg = [&](double extra) {
        const double h[3] = {0.5 * (q[3] - q[0]), 0.5 * (q[4] - q[1]), 0.5 * (q[5] - q[2])};
        for (int a = 0; a < 3; ++a) cl[a] = 0.5 * (q[a] + q[a + 3]);
        return std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]) + extra;
    };
    switch (pr.kind) {
        case SMCRT_SPHERE: rl = q[0]; break;
        case SMCRT_BOX: rl = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]); break;
        case SMCRT_TORUS: rl = std::fabs(q[0]) + std::fabs(q[1]); break;
        case SMCRT_CAPSULE: rl = seg(q[6]); break;
        case SMCRT_SEGMENT: rl = seg(0.1); break;
        case SMCRT_CYLINDER: {
            const double hl = seg(0.0);
            rl = std::sqrt(hl * hl + q[6] * q[6]);
            break;
        }
        default: return false;
    }
    if (!(rl >= 0) || !std::isfinite(rl)) return false;
    // p_local = p_world . M3 + t (row vector); rigid M3 => p_world = (p_local - t) . M3^T
    const double(*M)[3] = pr.transform;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const double dot = M[i][0] * M[j][0] + M[i][1] * M[j][1] + M[i][2] * M[j][2];
            if (std::fabs(dot - (i == j ? 1.0 : 0.0)) > 1e-9) return false;
        }
    for (int i = 0; i < 3; ++i) {
        double v = 0;
        for (int j = 0; j < 3; ++j) v += (cl[j] - M[3][j]) * M[i][j];
        c[i] = v;
    }
    *rad = rl;
    return std::isfinite(c[0]) && std::isfinite(c[1]) && std::isfinite(c[2]);
}

bool cache_policy(const smcrt_scene* s, const smcrt_grid* grid, int bytes, double* margin) {
    double scale = 1.0;
    if (grid) scale = std::fmax(scale, std::fmax(grid->xmax, std::fmax(grid->ymax, grid->zmax)));
    for (int i = 0; i < s->nregions; ++i) {
        double c[3], rad;
        if (!region_bound(s, i, c, &rad)) {
            *margin = 0;
            return false;
        }
        scale = std::fmax(scale, std::fabs(c[0]) + std::fabs(c[1]) + std::fabs(c[2]) + rad);
    }
    // 64 ulps of the coordinates' magnitude: the transform and the primitive's
    // few operations round a region's value by a handful of ulps
    int e;
    std::frexp(scale, &e);
    *margin = std::ldexp(64.0, e - (bytes == 4 ? 24 : 53));
    return true;
}

template <class R>
void scene_tables(const smcrt_scene* s, const smcrt_grid* grid, std::vector<DPrim<R>>& prims,
                  std::vector<DRegion<R>>& regions, std::vector<R>& bounds, R* margin) {
    prims.resize(s->nprims);
    regions.resize(s->nregions);
    bounds.assign(4 * (size_t)s->nregions, (R)0);
    for (int i = 0; i < s->nprims; ++i) fill_prim(prims[i], s->prims[i]);
    double scale = 1.0;
    if (grid) scale = std::fmax(scale, std::fmax(grid->xmax, std::fmax(grid->ymax, grid->zmax)));
    for (int i = 0; i < s->nregions; ++i) {
        fill_region(regions[i], s->regions[i]);
        double c[3], rad;
        if (region_bound(s, i, c, &rad)) {
            for (int a = 0; a < 3; ++a) bounds[4 * i + a] = (R)c[a];
            bounds[4 * i + 3] = (R)rad;
            scale = std::fmax(scale, std::fabs(c[0]) + std::fabs(c[1]) + std::fabs(c[2]) + rad);
        } else {
            bounds[4 * i + 3] = (R)(-1);
        }
    }
    // the test's rounding (and the evaluation's) is a few ulps of the coordinates;
    // the margin is far above it
    *margin = (R)((sizeof(R) == 4 ? 1e-4 : 1e-11) * 4.0 * scale);
}
template void scene_tables<float>(const smcrt_scene*, const smcrt_grid*, std::vector<DPrim<float>>&,
                                  std::vector<DRegion<float>>&, std::vector<float>&, float*);
template void scene_tables<double>(const smcrt_scene*, const smcrt_grid*, std::vector<DPrim<double>>&,
                                   std::vector<DRegion<double>>&, std::vector<double>&, double*);
template void fill_scene<float>(SceneT<float>&, const smcrt_scene*);
template void fill_scene<double>(SceneT<double>&, const smcrt_scene*);

namespace {

template <class R>
__global__ void k_eval_sdf(const __grid_constant__ SceneT<R> sc, const double* pts, long long n, double* out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<R> p{(R)pts[3 * i], (R)pts[3 * i + 1], (R)pts[3 * i + 2]};
    for (int r = 0; r < sc.nregions; ++r) out[i * sc.nregions + r] = (double)eval_region(sc, r, p);
}

__global__ void k_normal(const __grid_constant__ SceneT<double> sc, int region, double h, const double* pts,
                         long long n, double* out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<double> nn = calc_normal(sc, region, V3<double>{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]}, h);
    out[3 * i] = nn.x;
    out[3 * i + 1] = nn.y;
    out[3 * i + 2] = nn.z;
}

template <class R>
__global__ void k_fresnel(const double* I, const double* N, const double* n1, const double* n2, const double* u,
                          long long n, double* R_out, double* I_out, int* refl) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<R> d{(R)I[3 * i], (R)I[3 * i + 1], (R)I[3 * i + 2]}, nn{(R)N[3 * i], (R)N[3 * i + 1], (R)N[3 * i + 2]};
    const R Rf = fresnel(d, nn, (R)n1[i], (R)n2[i]);
    if (R_out) R_out[i] = (double)Rf;
    if (I_out) {
        const bool r = (R)u[i] <= Rf;
        d = r ? reflect(d, nn) : refract(d, nn, (R)n1[i] / (R)n2[i]);
        I_out[3 * i] = d.x;
        I_out[3 * i + 1] = d.y;
        I_out[3 * i + 2] = d.z;
        refl[i] = r;
    }
}

template <class R>
__global__ void k_scatter(const double* dir, const double* g, const double* u, long long n, double* out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stream<R, true> s;
    s.init(0, 0, 0, u + 3 * i, 3);
    V3<R> d{(R)dir[3 * i], (R)dir[3 * i + 1], (R)dir[3 * i + 2]};
    d = hg_scatter(d, (R)g[i], (R)(g[i] * g[i]), s);
    out[3 * i] = d.x;
    out[3 * i + 1] = d.y;
    out[3 * i + 2] = d.z;
}

__global__ void k_philox(const uint32_t* key, const uint32_t* ctr, long long n, uint32_t* out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t o[4];
    philox4x32_10(key[2 * i], key[2 * i + 1], ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3], o);
    for (int a = 0; a < 4; ++a) out[4 * i + a] = o[a];
}

// Launch state of packets [first, first + n) of stream P.seed: the emitter
// (src/photon.f90) and the launch layer (src/kernelsMod.f90:275-280, 1-based).
template <class R>
__global__ void k_emit(const __grid_constant__ Params<R> P, long long first, long long n, double* pos, double* dir,
                       int* layer) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Pk<R> pk;
    Stream<R, false> rng;
    rng.init(P.seed, P.instance, (uint64_t)(first + i), nullptr, 0);
    emit(P, pk, rng);
    // the launch sweep as the transport kernel takes it: within near_band of a
    // surface, FP32 transport decides on the FP64 position with the FP64 scene
    const SweepOut<R> o = sweep_regions<R, true>(P.sc, cv<R>(pk.pos), 0);
    int lay = o.lay;
    if (sizeof(R) == 4 && o.mna <= P.near_band) lay = sweep_regions<double, true>(P.sc64, pk.pos, 0).lay;
    layer[i] = lay + 1;
    pos[3 * i] = pk.pos.x;
    pos[3 * i + 1] = pk.pos.y;
    pos[3 * i + 2] = pk.pos.z;
    dir[3 * i] = (double)pk.dir.x;
    dir[3 * i + 1] = (double)pk.dir.y;
    dir[3 * i + 2] = (double)pk.dir.z;
}

inline int nblk(long long n) { return (int)((n + 127) / 128); }

}  // namespace

cudaError_t probe_eval_sdf(int precision, const smcrt_scene* scene, const double* d_pts, long long n, double* d_out) {
    if (precision == SMCRT_FP64) {
        SceneT<double>* sc = new SceneT<double>;
        fill_scene(*sc, scene);
        k_eval_sdf<double><<<nblk(n), 128>>>(*sc, d_pts, n, d_out);
        delete sc;
    } else {
        SceneT<float>* sc = new SceneT<float>;
        fill_scene(*sc, scene);
        k_eval_sdf<float><<<nblk(n), 128>>>(*sc, d_pts, n, d_out);
        delete sc;
    }
    return cudaGetLastError();
}

cudaError_t probe_normal(const smcrt_scene* scene, int region, double h, const double* d_pts, long long n,
                         double* d_out) {
    SceneT<double>* sc = new SceneT<double>;
    fill_scene(*sc, scene);
    k_normal<<<nblk(n), 128>>>(*sc, region, h, d_pts, n, d_out);
    delete sc;
    return cudaGetLastError();
}

cudaError_t probe_fresnel(int precision, const double* I, const double* N, const double* n1, const double* n2,
                          const double* u, long long n, double* R_out, double* I_out, int* refl) {
    if (precision == SMCRT_FP64) k_fresnel<double><<<nblk(n), 128>>>(I, N, n1, n2, u, n, R_out, I_out, refl);
    else k_fresnel<float><<<nblk(n), 128>>>(I, N, n1, n2, u, n, R_out, I_out, refl);
    return cudaGetLastError();
}

cudaError_t probe_scatter(int precision, const double* dir, const double* g, const double* u, long long n,
                          double* out) {
    if (precision == SMCRT_FP64) k_scatter<double><<<nblk(n), 128>>>(dir, g, u, n, out);
    else k_scatter<float><<<nblk(n), 128>>>(dir, g, u, n, out);
    return cudaGetLastError();
}

cudaError_t probe_philox(const uint32_t* key, const uint32_t* ctr, long long n, uint32_t* out) {
    k_philox<<<nblk(n), 128>>>(key, ctr, n, out);
    return cudaGetLastError();
}

template <class R>
cudaError_t probe_emit(const Params<R>& P, long long first, long long n, double* pos, double* dir, int* layer) {
    k_emit<R><<<nblk(n), 128>>>(P, first, n, pos, dir, layer);
    return cudaGetLastError();
}
template cudaError_t probe_emit<float>(const Params<float>&, long long, long long, double*, double*, int*);
template cudaError_t probe_emit<double>(const Params<double>&, long long, long long, double*, double*, int*);

}  // namespace smcrt
