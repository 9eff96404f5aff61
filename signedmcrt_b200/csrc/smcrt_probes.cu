// smcrt_probes.cu -- element-wise kernels that expose the transport's device
// building blocks (SDF evaluation, calcNormal, Fresnel, HG scatter, Philox) for
// parity checks, plus the host-side scene conversion shared with the API.
#include <cstring>

#include "smcrt_launch.h"

namespace smcrt {

template <class R>
void fill_scene(SceneT<R>& d, const smcrt_scene* s) {
    std::memset(&d, 0, sizeof(d));
    d.nregions = s->nregions;
    d.nprims = s->nprims;
    d.has_mods = 0;
    for (int i = 0; i < s->nprims; ++i) d.has_mods |= s->prims[i].nmods > 0;
    for (int i = 0; i < s->nprims; ++i) {
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 3; ++b) d.prim[i].m[3 * a + b] = (R)s->prims[i].transform[a][b];
        for (int a = 0; a < 8; ++a) d.prim[i].q[a] = (R)s->prims[i].params[a];
        d.prim[i].kind = s->prims[i].kind;
        d.prim[i].nmods = s->prims[i].nmods;
        for (int j = 0; j < 2; ++j) {
            d.prim[i].mod[j] = s->prims[i].mods[j];
            for (int a = 0; a < 3; ++a) d.prim[i].mp[j][a] = (R)s->prims[i].mod_params[j][a];
        }
    }
    for (int i = 0; i < s->nregions; ++i) {
        const smcrt_region& g = s->regions[i];
        DRegion<R>& r = d.region[i];
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
}
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

}  // namespace smcrt
