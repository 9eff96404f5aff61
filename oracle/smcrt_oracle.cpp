// smcrt_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A CPU restatement of signedMCRT's photon-packet transport path, written from
// the reference's Fortran sources.  Each function names the reference lines it
// follows (paths relative to the signedMCRT project root).  It runs in two
// semantics, selected by oracle_policy:
//   * reference semantics: FP64, eps = 1e-8, the snapping voxel walk of
//     update_grids/update_pos/update_voxels, optional FP32 tally -- the
//     reference algorithm as written, used as the CPU baseline and as the
//     statistical reference;
//   * device semantics: FP32 or FP64 transport, scale-relative epsilon,
//     integer-stepping voxel walk and FP64 boundary events -- the algorithm the
//     CUDA kernel implements, used for per-packet replay parity.
// Randomness is either the counter-based Philox4x32-10 stream keyed by
// (seed, instance, packet id) or a caller-injected uniform stream in the
// reference's draw order.
#include "smcrt_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPI = 3.14159265358979323846264338327950288;  // 4*atan(1), constants.f90:22

// ---------------------------------------------------------------------------
// vec3 (src/vector_class.f90)
template <class R>
struct V3 {
    R x, y, z;
};
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }  // :292
template <class R> inline R length(V3<R> a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }  // :405-411
template <class R> inline V3<R> magnitude(V3<R> a) { R t = length(a); return {a.x / t, a.y / t, a.z / t}; }  // :392-402
template <class R> inline V3<R> vabs(V3<R> a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
template <class R> inline V3<R> vmax(V3<R> a, R v) { return {std::max(a.x, v), std::max(a.y, v), std::max(a.z, v)}; }
template <class R> inline R clamp(R x, R lo, R hi) { return std::min(std::max(x, lo), hi); }  // utils.clamp
template <class R> inline R fsign(R a, R b) { return std::signbit(b) ? -std::fabs(a) : std::fabs(a); }  // Fortran sign(a,b)

// ---------------------------------------------------------------------------
// Scene in working precision.
template <class R>
struct Prim {
    int kind;
    R m[4][3];
    R p[8];
    int nmods;
    int mod[2];
    R mp[2][3];
};
template <class R>
struct Region {
    int first, n, op;
    R k, mus, mua, hgg, g2, n_idx, kappa, albedo;
};

template <class R>
struct Scene {
    std::vector<Prim<R>> prims;
    std::vector<Region<R>> regions;
};

// init_mono, src/opticalProps/opticalProperties.f90:107-125 (computed in FP64, then rounded).
template <class R>
Scene<R> make_scene(const smcrt_scene* s) {
    Scene<R> out;
    for (int i = 0; i < s->nprims; ++i) {
        Prim<R> p{};
        p.kind = s->prims[i].kind;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 3; ++b) p.m[a][b] = (R)s->prims[i].transform[a][b];
        for (int a = 0; a < 8; ++a) p.p[a] = (R)s->prims[i].params[a];
        p.nmods = s->prims[i].nmods;
        for (int j = 0; j < 2; ++j) {
            p.mod[j] = s->prims[i].mods[j];
            for (int a = 0; a < 3; ++a) p.mp[j][a] = (R)s->prims[i].mod_params[j][a];
        }
        out.prims.push_back(p);
    }
    for (int i = 0; i < s->nregions; ++i) {
        const smcrt_region& g = s->regions[i];
        Region<R> r{};
        r.first = g.first_prim;
        r.n = g.nprims;
        r.op = g.op;
        r.k = (R)g.k;
        double kappa = g.mus + g.mua;
        double albedo = (g.mua < 1e-9) ? 1.0 : g.mus / kappa;
        r.mus = (R)g.mus;
        r.mua = (R)g.mua;
        r.hgg = (R)g.hgg;
        r.g2 = (R)(g.hgg * g.hgg);
        r.n_idx = (R)g.n;
        r.kappa = (R)kappa;
        r.albedo = (R)albedo;
        out.regions.push_back(r);
    }
    return out;
}

int validate_scene(const smcrt_scene* s) {
    if (!s || s->nregions <= 0 || s->nprims <= 0 || !s->regions || !s->prims) return 1;
    for (int i = 0; i < s->nprims; ++i) {
        if (s->prims[i].kind < SMCRT_SPHERE || s->prims[i].kind > SMCRT_PLANE) return 1;
        if (s->prims[i].nmods < 0 || s->prims[i].nmods > 2) return 1;
        for (int j = 0; j < s->prims[i].nmods; ++j)
            if (s->prims[i].mods[j] < SMCRT_MOD_ONION || s->prims[i].mods[j] > SMCRT_MOD_BEND) return 1;
    }
    for (int i = 0; i < s->nregions; ++i) {
        const smcrt_region& r = s->regions[i];
        if (r.nprims <= 0 || r.first_prim < 0 || r.first_prim + r.nprims > s->nprims) return 1;
        if (r.nprims > 1 && (r.op < SMCRT_OP_UNION || r.op > SMCRT_OP_INTERSECTION)) return 1;
    }
    return 0;
}

// pos .dot. transform, src/vector_class.f90:292-304
template <class R>
inline V3<R> xform(const R m[4][3], V3<R> a) {
    V3<R> d;
    d.x = m[0][0] * a.x + m[1][0] * a.y + m[2][0] * a.z + m[3][0];
    d.y = m[0][1] * a.x + m[1][1] * a.y + m[2][1] * a.z + m[3][1];
    d.z = m[0][2] * a.x + m[1][2] * a.y + m[2][2] * a.z + m[3][2];
    return d;
}

// Primitive SDFs, src/sdfs/sdfs.f90:494-735
template <class R>
R eval_prim_base(const Prim<R>& pr, V3<R> pos) {
    V3<R> p = xform(pr.m, pos);
    const R* q = pr.p;
    const R zero = 0, one = 1, half = (R)0.5;
    switch (pr.kind) {
        case SMCRT_SPHERE:  // :494-508
            return std::sqrt(p.x * p.x + p.y * p.y + p.z * p.z) - q[0];
        case SMCRT_BOX: {  // :510-525
            V3<R> d = vabs(p) - V3<R>{q[0], q[1], q[2]};
            return length(vmax(d, zero)) + std::min(std::max(d.x, std::max(d.y, d.z)), zero);
        }
        case SMCRT_TORUS: {  // :527-542
            V3<R> t{length(V3<R>{p.x, zero, p.z}) - q[0], p.y, zero};
            return length(t) - q[1];
        }
        case SMCRT_CYLINDER: {  // :544-581
            V3<R> a{q[0], q[1], q[2]}, b{q[3], q[4], q[5]};
            V3<R> ba = b - a, pa = p - a;
            R baba = dot(ba, ba), paba = dot(pa, ba);
            R x = length(pa * baba - ba * paba) - q[6] * baba;
            R y = std::fabs(paba - baba * half) - baba * half;
            R x2 = x * x, y2 = (y * y) * baba, d;
            if (std::max(x, y) < zero) {
                d = -std::min(x2, y2);
            } else {
                if (x > zero && y > zero) d = x2 + y2;
                else if (x > zero) d = x2;
                else if (y > zero) d = y2;
                else d = zero;
            }
            return fsign(std::sqrt(std::fabs(d)) / baba, d);
        }
        case SMCRT_TRIPRISM: {  // :583-597
            V3<R> a = vabs(p);
            return std::max(a.z - q[1], std::max(a.x * (R)0.866025 + p.y * half, -p.y) - q[0] * half);
        }
        case SMCRT_SEGMENT:  // :599-626
        case SMCRT_CAPSULE: {  // :628-648
            V3<R> a{q[0], q[1], q[2]}, b{q[3], q[4], q[5]};
            V3<R> pa = p - a, ba = b - a;
            R h = clamp(dot(pa, ba) / dot(ba, ba), zero, one);
            R r = (pr.kind == SMCRT_SEGMENT) ? (R)0.1 : q[6];
            return length(pa - ba * h) - r;
        }
        case SMCRT_CONE: {  // :650-686
            V3<R> a{q[0], q[1], q[2]}, b{q[3], q[4], q[5]};
            R ra = q[6], rb = q[7];
            R rba = rb - ra;
            R baba = dot(b - a, b - a);
            R papa = dot(p - a, p - a);
            R paba = dot(p - a, b - a) / baba;
            // sqrt of a negative rounding residue (points on the axis) is taken as 0
            R x = std::sqrt(std::max(papa - baba * paba * paba, zero));
            R cax = (paba < half) ? std::max(zero, x - ra) : std::max(zero, x - rb);
            R cay = std::fabs(paba - half) - half;
            R k = rba * rba + baba;
            R f = clamp((rba * (x - ra) + paba * baba) / k, zero, one);
            R cbx = x - ra - f * rba;
            R cby = paba - f;
            R s = (cbx < zero && cay < zero) ? -one : one;
            return s * std::sqrt(std::min(cax * cax + baba * cay * cay, cbx * cbx + baba * cby * cby));
        }
        case SMCRT_EGG: {  // :688-718
            V3<R> pin{std::fabs(p.x), p.y, p.z};
            R r = q[0] - q[1];
            R hin = q[2] + r;
            R l = (hin * hin - r * r) / ((R)2 * r);
            if (pin.y <= zero) return length(pin) - q[0];
            if ((pin.y - hin) * l > pin.x * hin)
                return length(pin - V3<R>{zero, hin, zero}) - ((q[0] + l) - length(V3<R>{hin, l, zero}));
            return length(pin + V3<R>{l, zero, zero}) - (q[0] + l);
        }
        case SMCRT_PLANE:  // :720-735
            return dot(p, V3<R>{q[0], q[1], q[2]});
    }
    return zero;
}

// Modifiers, src/sdfs/sdfModifiers.f90:273-375: eval_revolution (:290-305),
// eval_elongate (:319-335), eval_twist (:337-355), eval_bend (:357-375) change the
// point the wrapped SDF is evaluated at; eval_onion (:307-317), eval_extrude
// (:273-288) and eval_elongate change its value.  The wrapped primitive applies
// its own transform; a modifier has none.
template <class R>
V3<R> mod_point(int kind, const R* q, V3<R> p) {
    const R zero = 0;
    if (kind == SMCRT_MOD_REVOLUTION) return V3<R>{length(V3<R>{p.x, p.z, zero}) - q[0], p.y, zero};
    if (kind == SMCRT_MOD_ELONGATE)
        return V3<R>{std::max(std::fabs(p.x) - q[0], zero), std::max(std::fabs(p.y) - q[1], zero),
                     std::max(std::fabs(p.z) - q[2], zero)};
    if (kind == SMCRT_MOD_TWIST || kind == SMCRT_MOD_BEND) {
        const R a = q[0] * (kind == SMCRT_MOD_TWIST ? p.z : p.x);
        const R c = std::cos(a), s = std::sin(a);
        return V3<R>{c * p.x - s * p.y, s * p.x + c * p.y, p.z};
    }
    return p;
}
template <class R>
R mod_value(int kind, const R* q, R d, V3<R> p) {
    const R zero = 0;
    if (kind == SMCRT_MOD_ONION) return std::fabs(d) - q[0];
    if (kind == SMCRT_MOD_EXTRUDE) {
        const V3<R> w{d, std::fabs(p.z) - q[0], zero};
        return std::min(std::max(w.x, w.y), zero) + length(vmax(w, zero));
    }
    if (kind == SMCRT_MOD_ELONGATE) {
        const V3<R> e = vabs(p) - V3<R>{q[0], q[1], q[2]};
        return d + std::min(std::max(e.x, std::max(e.y, e.z)), zero);
    }
    return d;
}
// onion(revolution(egg)): the outer modifier's point map first, the inner's value
// map first -- the nested evaluate calls of the reference.
template <class R>
R eval_prim(const Prim<R>& pr, V3<R> pos) {
    if (pr.nmods == 0) return eval_prim_base(pr, pos);
    const V3<R> p1 = pr.nmods == 2 ? mod_point(pr.mod[1], pr.mp[1], pos) : pos;
    const V3<R> p2 = mod_point(pr.mod[0], pr.mp[0], p1);
    R d = mod_value(pr.mod[0], pr.mp[0], eval_prim_base(pr, p2), p1);
    if (pr.nmods == 2) d = mod_value(pr.mod[1], pr.mp[1], d, pos);
    return d;
}

// eval_model (src/sdfs/sdf_base.f90:145-160) with the CSG ops of
// src/sdfs/sdfModifiers.f90:412-475.
template <class R>
R eval_region(const Scene<R>& sc, int r, V3<R> pos) {
    const Region<R>& g = sc.regions[r];
    R d = eval_prim(sc.prims[g.first], pos);
    for (int i = 1; i < g.n; ++i) {
        R d2 = eval_prim(sc.prims[g.first + i], pos);
        switch (g.op) {
            case SMCRT_OP_UNION: d = std::min(d, d2); break;
            case SMCRT_OP_SMOOTH_UNION: {
                R h = std::max(g.k - std::fabs(d - d2), (R)0) / g.k;
                d = std::min(d, d2) - h * h * h * g.k * ((R)1 / (R)6);
                break;
            }
            case SMCRT_OP_SUBTRACTION: d = std::max(-d, d2); break;
            case SMCRT_OP_INTERSECTION: d = std::max(d, d2); break;
        }
    }
    return d;
}

// calcNormal, src/sdfs/sdf_base.f90:165-189
template <class R>
V3<R> calc_normal(const Scene<R>& sc, int r, V3<R> p, R h) {
    const V3<R> xyy{1, -1, -1}, yyx{-1, -1, 1}, yxy{-1, 1, -1}, xxx{1, 1, 1};
    V3<R> n = xyy * eval_region(sc, r, p + xyy * h) + yyx * eval_region(sc, r, p + yyx * h) +
              yxy * eval_region(sc, r, p + yxy * h) + xxx * eval_region(sc, r, p + xxx * h);
    return magnitude(n);
}

// ---------------------------------------------------------------------------
// Fresnel, src/surfaces.f90:14-120
template <class R>
R fresnel(V3<R> I, V3<R> N, R n1, R n2) {
    R costt = std::fabs(dot(I, N));
    R sintt = std::sqrt((R)1 - costt * costt);
    R sint2 = n1 / n2 * sintt;
    if (sint2 > (R)1) return (R)1;
    if (costt == (R)1) return (R)0;
    sint2 = (n1 / n2) * sintt;
    R cost2 = std::sqrt((R)1 - sint2 * sint2);
    R f1 = std::fabs((n1 * costt - n2 * cost2) / (n1 * costt + n2 * cost2));
    R f2 = std::fabs((n1 * cost2 - n2 * costt) / (n1 * cost2 + n2 * costt));
    f1 = f1 * f1;
    f2 = f2 * f2;
    return (R)0.5 * (f1 + f2);
}
template <class R>
V3<R> reflect(V3<R> I, V3<R> N) {  // :42-55
    return I - (R)2 * dot(N, I) * N;
}
template <class R>
V3<R> refract(V3<R> I, V3<R> N, R eta) {  // :57-84
    V3<R> Nt = N;
    R c1 = dot(Nt, I);
    if (c1 < (R)0) c1 = -c1;
    else Nt = (R)(-1) * N;
    R c2 = std::sqrt((R)1 - (eta * eta) * ((R)1 - c1 * c1));
    return eta * I + (eta * c1 - c2) * Nt;
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): 10 rounds of the 4x32 S-box with multipliers
// 0xD2511F53 / 0xCD9E8D57 and Weyl key increments 0x9E3779B9 / 0xBB67AE85.
inline void philox(const uint32_t key_in[2], const uint32_t ctr[4], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Uniform in (0,1): FP32 from 23 bits of one word, FP64 from 52 bits of two.
template <class R> struct U01;
template <> struct U01<float> {
    static float from(const uint32_t* w) { return (float)(w[0] >> 9) * 0x1p-23f + 0x1p-24f; }
    static constexpr int words = 1;
};
template <> struct U01<double> {
    static double from(const uint32_t* w) {
        uint64_t m = ((uint64_t)w[0] << 20) | (uint64_t)(w[1] >> 12);
        return (double)m * 0x1p-52 + 0x1p-53;
    }
    static constexpr int words = 2;
};

template <class R>
struct PhiloxStream {
    uint32_t key[2];
    uint32_t ctr[4];
    uint32_t buf[4];
    int used = 4;
    int64_t ndraws = 0;
    int flags = 0;
    PhiloxStream(uint64_t seed, uint32_t instance, uint64_t pid) {
        key[0] = (uint32_t)seed;
        key[1] = (uint32_t)(seed >> 32);
        ctr[0] = 0;
        ctr[1] = instance;
        ctr[2] = (uint32_t)pid;
        ctr[3] = (uint32_t)(pid >> 32);
    }
    R next() {
        if (used + U01<R>::words > 4) {
            philox(key, ctr, buf);
            ctr[0] += 1;
            used = 0;
        }
        R u = U01<R>::from(buf + used);
        used += U01<R>::words;
        ++ndraws;
        return u;
    }
};

template <class R>
struct InjectedStream {
    const double* u;
    int64_t n;
    int64_t ndraws = 0;
    int flags = 0;
    R next() {
        if (ndraws >= n) {
            flags |= 4;
            ++ndraws;
            return (R)0.5;
        }
        return (R)u[ndraws++];
    }
};

// ---------------------------------------------------------------------------
// Grid (src/grid.f90:53-93) and tallies.
struct GridD {
    int nx, ny, nz;
    double xmax, ymax, zmax;
    std::vector<double> xf, yf, zf;
    explicit GridD(const smcrt_grid& g) : nx(g.nxg), ny(g.nyg), nz(g.nzg), xmax(g.xmax), ymax(g.ymax), zmax(g.zmax) {
        xf.resize(nx + 1);
        yf.resize(ny + 1);
        zf.resize(nz + 2);
        for (int i = 1; i <= nx + 1; ++i) xf[i - 1] = ((double)(i - 1) * 2.0) * xmax / nx;
        for (int i = 1; i <= ny + 1; ++i) yf[i - 1] = ((double)(i - 1) * 2.0) * ymax / ny;
        for (int i = 1; i <= nz + 2; ++i) zf[i - 1] = ((double)(i - 1) * 2.0) * zmax / nz;
    }
};

struct Tally {
    double* j64 = nullptr;
    float* j32 = nullptr;
    const double* w = nullptr;  // perturbation MC: voxel weights of the loss
    double* csum = nullptr;     // and the packet's weighted path length
    // second moment: the packet's own score per voxel, squared into j2 when the
    // packet ends (history-based variance)
    std::unordered_map<int64_t, double>* packet = nullptr;
    void add(int64_t idx, double v) {
        if (csum) *csum += w[idx] * v;
        if (packet) (*packet)[idx] += v;
        if (j32) {
            float* a = j32 + idx;
#pragma omp atomic
            *a += (float)v;
        } else if (j64) {
            double* a = j64 + idx;
#pragma omp atomic
            *a += v;
        }
    }
};

constexpr int kAdjGroups = 16;
struct Counters {
    uint64_t sdf = 0, vox = 0, steps = 0, scat = 0, fres = 0, refl = 0, stepcap = 0, err = 0, draws = 0;
    double nscatt = 0;
    double mom[24] = {0};
    double adj[3 * kAdjGroups] = {0};  // perturbation MC: sum over packets of C * score
    double loss = 0;                   // and of C
};

template <class R>
struct Packet {
    V3<double> pos;  // FP64 position accumulator in every mode (the GPU's FP32 path keeps it too)
    V3<R> dir;
    R weight;
    int layer;  // 0-based
    int bounces;
    bool tflag;
    int flags;  // bit0 step cap, bit1 error state
    int nscatt;
};

struct Pol {
    double eps, delta, h;
    bool ref_dda, crossing_f64;
    bool kill_le;  // device semantics: d <= eps at the start of a flight counts as on the surface
    bool near_f64; // device FP32 semantics: near-surface and crossing sweeps in FP64 (see sweep)
    double near_band = 0;  // ... closer than this to a surface
    int64_t max_steps;
};

// update_voxels, src/inttau2.f90:414-441 (and the index formula in working precision)
template <class R>
inline void voxel_of(const GridD& g, V3<R> p, int& ci, int& cj, int& ck) {
    ci = (int)std::floor((R)g.nx * p.x / ((R)2 * (R)g.xmax)) + 1;
    cj = (int)std::floor((R)g.ny * p.y / ((R)2 * (R)g.ymax)) + 1;
    ck = (int)std::floor((R)g.nz * p.z / ((R)2 * (R)g.zmax)) + 1;
    if (ci > g.nx || ci < 1) ci = -1;
    if (cj > g.ny || cj < 1) cj = -1;
    if (ck > g.nz || ck < 1) ck = -1;
}
// The device semantics' cell of an FP64 grid-coordinate point: FP64 transport
// divides as update_voxels does; FP32 transport multiplies by the FP64 n / (2 max).
template <class R>
inline void cell_of(const GridD& g, V3<double> p, int& ci, int& cj, int& ck) {
    if (sizeof(R) == 8) {
        voxel_of(g, p, ci, cj, ck);
        return;
    }
    ci = (int)std::floor(p.x * ((double)g.nx / (2.0 * g.xmax))) + 1;
    cj = (int)std::floor(p.y * ((double)g.ny / (2.0 * g.ymax))) + 1;
    ck = (int)std::floor(p.z * ((double)g.nz / (2.0 * g.zmax))) + 1;
    if (ci > g.nx || ci < 1) ci = -1;
    if (cj > g.ny || cj < 1) cj = -1;
    if (ck > g.nz || ck < 1) ck = -1;
}
inline int64_t cell_index(const GridD& g, int i, int j, int k) {
    return (int64_t)(i - 1) + (int64_t)g.nx * ((int64_t)(j - 1) + (int64_t)g.ny * (int64_t)(k - 1));
}

// update_grids with wall_dist/update_pos/update_voxels exactly as written,
// src/inttau2.f90:213-441.  Returns false on the "dcell < 0" error stop.
template <class R>
bool update_grids_ref(const GridD& g, V3<R> pos, V3<R> dir, R dsdf, R delta, Tally& t, Counters& c, bool& tflag) {
    V3<R> old{pos.x + (R)g.xmax, pos.y + (R)g.ymax, pos.z + (R)g.zmax};
    int ci, cj, ck;
    voxel_of(g, old, ci, cj, ck);
    R d = 0;
    if (ci == -1 || cj == -1 || ck == -1) {
        tflag = true;
        return true;
    }
    for (;;) {
        R dx = -999, dy = -999, dz = -999;
        if (dir.x > 0) dx = ((R)g.xf[ci] - old.x) / dir.x;
        else if (dir.x < 0) dx = ((R)g.xf[ci - 1] - old.x) / dir.x;
        else if (dir.x == 0) dx = (R)100000;
        if (dir.y > 0) dy = ((R)g.yf[cj] - old.y) / dir.y;
        else if (dir.y < 0) dy = ((R)g.yf[cj - 1] - old.y) / dir.y;
        else if (dir.y == 0) dy = (R)100000;
        if (dir.z > 0) dz = ((R)g.zf[ck] - old.z) / dir.z;
        else if (dir.z < 0) dz = ((R)g.zf[ck - 1] - old.z) / dir.z;
        else if (dir.z == 0) dz = (R)100000;
        R dcell = std::min(dx, std::min(dy, dz));
        if (dcell < 0) return false;  // error stop 1 (:337-343)
        bool lx = dcell == dx, ly = dcell == dy, lz = dcell == dz;
        if (d + dcell > dsdf) {
            dcell = dsdf - d;
            d = dsdf;
            t.add(cell_index(g, ci, cj, ck), (double)dcell);
            ++c.vox;
            break;  // update_pos without a wall only moves the local copy
        }
        d = d + dcell;
        t.add(cell_index(g, ci, cj, ck), (double)dcell);
        ++c.vox;
        // update_pos with wall_flag (:365-400)
        if (lx) {
            if (dir.x > 0) old.x = (R)g.xf[ci] + delta;
            else if (dir.x < 0) old.x = (R)g.xf[ci - 1] - delta;
            old.y = old.y + dir.y * dcell;
            old.z = old.z + dir.z * dcell;
        } else if (ly) {
            if (dir.y > 0) old.y = (R)g.yf[cj] + delta;
            else if (dir.y < 0) old.y = (R)g.yf[cj - 1] - delta;
            old.x = old.x + dir.x * dcell;
            old.z = old.z + dir.z * dcell;
        } else if (lz) {
            if (dir.z > 0) old.z = (R)g.zf[ck] + delta;
            else if (dir.z < 0) old.z = (R)g.zf[ck - 1] - delta;
            old.x = old.x + dir.x * dcell;
            old.y = old.y + dir.y * dcell;
        } else {
            return false;  // error stop 1 (:397-400)
        }
        voxel_of(g, old, ci, cj, ck);
        if (ci == -1 || cj == -1 || ck == -1) {
            tflag = true;
            break;
        }
    }
    return true;
}

// Integer-stepping voxel walk (the GPU's): same start cell and exit rule as
// update_grids, but crossings advance the cell index by +-1 and distances are
// measured from the segment start, so no re-indexing from snapped positions.
template <class R>
// The start cell and the distances to its faces come from the FP64 position (an
// FP32 coordinate within an ulp of a grid face could round onto it); the walk
// itself runs in R.
bool update_grids_int(const GridD& g, V3<double> pos, V3<R> dir, R dsdf, Tally& t, Counters& c, bool& tflag) {
    const V3<double> o{pos.x + g.xmax, pos.y + g.ymax, pos.z + g.zmax};
    int ci, cj, ck;
    cell_of<R>(g, o, ci, cj, ck);
    if (ci == -1 || cj == -1 || ck == -1) {
        tflag = true;
        return true;
    }
    const R big = (R)1e30;
    const R vx = (R)2 * (R)g.xmax / (R)g.nx, vy = (R)2 * (R)g.ymax / (R)g.ny, vz = (R)2 * (R)g.zmax / (R)g.nz;
    const int sx = dir.x > 0 ? 1 : (dir.x < 0 ? -1 : 0);
    const int sy = dir.y > 0 ? 1 : (dir.y < 0 ? -1 : 0);
    const int sz = dir.z > 0 ? 1 : (dir.z < 0 ? -1 : 0);
    // the first faces at FP64 multiples of the FP64 voxel size
    auto tnext = [&](int cell, int s, double v, double o1, R d1) -> R {
        if (s == 0) return big;
        const double face = (double)(s > 0 ? cell : cell - 1) * v;
        R tt = (R)(face - o1) / d1;
        return tt < (R)0 ? (R)0 : tt;
    };
    const double vxd = 2.0 * g.xmax / g.nx, vyd = 2.0 * g.ymax / g.ny, vzd = 2.0 * g.zmax / g.nz;
    R tx = tnext(ci, sx, vxd, o.x, dir.x), ty = tnext(cj, sy, vyd, o.y, dir.y), tz = tnext(ck, sz, vzd, o.z, dir.z);
    R d = 0;
    for (;;) {
        R tm = std::min(tx, std::min(ty, tz));
        if (tm > dsdf) {
            t.add(cell_index(g, ci, cj, ck), (double)(dsdf - d));
            ++c.vox;
            break;
        }
        t.add(cell_index(g, ci, cj, ck), (double)(tm - d));
        ++c.vox;
        d = tm;
        // next face on the crossed axis: one face spacing v/|d| further (Amanatides & Woo)
        if (tm == tx) {
            ci += sx;
            if (ci < 1 || ci > g.nx) { tflag = true; break; }
            tx = tm + vx / std::fabs(dir.x);
        } else if (tm == ty) {
            cj += sy;
            if (cj < 1 || cj > g.ny) { tflag = true; break; }
            ty = tm + vy / std::fabs(dir.y);
        } else {
            ck += sz;
            if (ck < 1 || ck > g.nz) { tflag = true; break; }
            tz = tm + vz / std::fabs(dir.z);
        }
    }
    return true;
}

template <class R>
inline V3<R> cv(V3<double> p) { return V3<R>{(R)p.x, (R)p.y, (R)p.z}; }
template <class R>
inline V3<double> advance(V3<double> p, R d, V3<R> dir) {
    return V3<double>{p.x + (double)(d * dir.x), p.y + (double)(d * dir.y), p.z + (double)(d * dir.z)};
}

// ---------------------------------------------------------------------------
// One sweep of every region at a point (the N evaluations of inttau2.f90:52-56,
// 86-90, 104-108, 117-121 and kernelsMod.f90:275-280): the values in transport
// precision R, their signed minimum, minimum |d|, the first region containing the
// point (-1: none) and the innermost containing region (the launch layer; 0 when
// none contains it).  Device FP32 semantics (pol.near_f64), as the GPU's FP32
// kernels do it: a sweep whose FP32 minimum |d| is within pol.near_band of a
// surface (16 FP32 ulps of the scene size, at least 2 eps), and
// every sweep after a crossing step (force64), is taken instead in FP64 at the
// FP64 position with the FP64 scene; its values are rounded to R and its region
// indices come from the FP64 values.
template <class R>
struct SweepRes {
    R mn, mna;
    int nl, lay;
    bool f64;  // taken in FP64
};
template <class T>
void sweep_stats(const T* v, int N, T& mn, T& mna, int& nl, int& lay) {
    mn = mna = std::numeric_limits<T>::infinity();
    nl = -1;
    lay = 0;
    T inner = std::numeric_limits<T>::infinity();
    for (int i = 0; i < N; ++i) {
        const T d = v[i];
        mn = std::min(mn, d);
        mna = std::min(mna, std::fabs(d));
        if (nl < 0 && d < (T)0) nl = i;
        const T a = (d > (T)0) ? (T)999.0 : std::fabs(d);
        if (a < inner) {
            inner = a;
            lay = i;
        }
    }
}
template <class R>
SweepRes<R> sweep(const Scene<R>& sc, const Scene<double>& sc64, const Pol& pol, V3<double> pos, bool force64,
                  R* out) {
    const int N = (int)sc.regions.size();
    SweepRes<R> o;
    o.f64 = sizeof(R) == 8;
    if (!(pol.near_f64 && force64)) {
        const V3<R> p = cv<R>(pos);
        for (int i = 0; i < N; ++i) out[i] = eval_region(sc, i, p);
        sweep_stats(out, N, o.mn, o.mna, o.nl, o.lay);
        if (!pol.near_f64 || sizeof(R) == 8 || o.mna > (R)pol.near_band) return o;
    }
    o.f64 = true;
    thread_local std::vector<double> v64;
    v64.resize(N);
    for (int i = 0; i < N; ++i) v64[i] = eval_region(sc64, i, pos);
    double mn, mna;
    sweep_stats(v64.data(), N, mn, mna, o.nl, o.lay);
    for (int i = 0; i < N; ++i) out[i] = (R)v64[i];
    o.mn = (R)mn;
    o.mna = (R)mna;
    return o;
}

// ---------------------------------------------------------------------------
// Boundary event: normal (calcNormal) + reflect_refract in precision E.
template <class R, class E, class Rng>
bool boundary_event(const Scene<E>& scE, int which, int L, int nl, V3<double> pos, V3<R>& dir, R h, Rng& rng,
                    R& Ri, Counters& c) {
    V3<E> p{(E)pos.x, (E)pos.y, (E)pos.z};
    V3<E> N = calc_normal(scE, which, p, (E)h);
    c.sdf += 4;
    V3<E> I{(E)dir.x, (E)dir.y, (E)dir.z};
    const E n1 = scE.regions[L].n_idx, n2 = scE.regions[nl].n_idx;
    E R_ = fresnel(I, N, n1, n2);
    E u = (E)rng.next();
    bool refl;
    if (u <= R_) {
        I = reflect(I, N);
        refl = true;
    } else {
        I = refract(I, N, n1 / n2);
        refl = false;
    }
    dir = V3<R>{(R)I.x, (R)I.y, (R)I.z};
    Ri = (R)R_;
    return refl;
}

// tauint2, src/inttau2.f90:15-210
// len (perturbation MC, optional): path length per region of the flights traced,
// added to; by_tau: whether the last flight ended at its optical depth (an
// interaction), not at an escape or a kill.
template <class R, class Rng>
void tauint2(const Scene<R>& sc, const Scene<double>& sc64, const GridD& g, const Pol& pol, Packet<R>& pk, Rng& rng,
             Tally& t, Counters& c, double* len = nullptr, bool* by_tau = nullptr) {
    const int N = (int)sc.regions.size();
    V3<double> pos = pk.pos, oldpos = pos;
    V3<R> dir = pk.dir;
    const R eps = (R)pol.eps;
    R tau = -std::log(rng.next());
    R taurun = 0;
    thread_local std::vector<R> ds, dstmp;
    if ((int)ds.size() < N) {
        ds.resize(N);
        dstmp.resize(N);
    }
    bool ok = true;
    for (;;) {
        // dstmp holds the values of the latest sweep: at a surface they are the
        // reference's dstmp sweep (:104-108), taken at the same point
        const SweepRes<R> top = sweep(sc, sc64, pol, pos, false, dstmp.data());
        R dsdf = top.mna;
        c.sdf += N;
        // device FP32 semantics: an FP64 sweep that finds the surface within half
        // of near_band sends the next step's sweep straight to FP64 (a move of
        // min|d| changes every |d| by at most that, so it is within near_band)
        bool near = pol.near_f64 && top.f64 && (R)2 * top.mna <= (R)pol.near_band;
        // reference: kill if d < eps (inttau2.f90:58); device semantics also kills
        // at d == eps, where the trace loop (d > eps, :63) has already stopped
        if (pol.kill_le ? dsdf <= eps : dsdf < eps) {
            pk.tflag = true;
            break;
        }
        int64_t steps = 0;
        while (dsdf > eps) {
            ++c.steps;
            R kap = sc.regions[pk.layer].kappa;
            R tsdf = dsdf * kap;
            if (taurun + tsdf <= tau) {
                taurun = taurun + tsdf;
                if (len) len[pk.layer] += (double)dsdf;
                oldpos = pos;
                ok = pol.ref_dda ? update_grids_ref(g, cv<R>(oldpos), dir, dsdf, (R)pol.delta, t, c, pk.tflag)
                                 : update_grids_int(g, oldpos, dir, dsdf, t, c, pk.tflag);
                pos = advance(pos, dsdf, dir);
            } else {
                dsdf = (tau - taurun) / kap;
                taurun = tau;
                if (len) len[pk.layer] += (double)dsdf;
                oldpos = pos;
                pos = advance(pos, dsdf, dir);
                ok = pol.ref_dda ? update_grids_ref(g, cv<R>(oldpos), dir, dsdf, (R)pol.delta, t, c, pk.tflag)
                                 : update_grids_int(g, oldpos, dir, dsdf, t, c, pk.tflag);
                if (!ok) break;
                break;
            }
            if (!ok) break;
            const SweepRes<R> sw = sweep(sc, sc64, pol, pos, near, dstmp.data());
            c.sdf += N;
            dsdf = sw.mna;
            near = pol.near_f64 && sw.f64 && (R)2 * sw.mna <= (R)pol.near_band;
            if (sw.mn >= (R)0) {
                pk.tflag = true;
                break;
            }
            if (++steps >= pol.max_steps) {
                pk.tflag = true;
                pk.flags |= 1;
                ++c.stepcap;
                break;
            }
        }
        if (!ok) {
            pk.tflag = true;
            pk.flags |= 2;
            ++c.err;
            break;
        }
        if (taurun >= tau || pk.tflag) break;

        R mind = std::numeric_limits<R>::infinity();
        for (int i = 0; i < N; ++i) mind = std::min(mind, std::fabs(dstmp[i]));
        c.sdf += N;
        R dstep = mind + (R)2 * eps;
        oldpos = pos;
        pos = advance(pos, dstep, dir);
        int nl = sweep(sc, sc64, pol, pos, true, ds.data()).nl;
        c.sdf += N;
        if (nl < 0) nl = 0;  // minloc of an all-zero array
        const int L = pk.layer;
        R n1 = sc.regions[L].n_idx, n2 = sc.regions[nl].n_idx;
        if (n1 != n2) {
            int pick;  // 1 -> packet%layer, 2 -> new_layer (:146-162)
            if (ds[L] < 0 && ds[nl] < 0) {
                pick = (std::fabs(ds[L]) <= std::fabs(ds[nl])) ? 1 : 2;
            } else if (dstmp[L] < 0 && dstmp[nl] < 0) {
                pick = (dstmp[L] >= dstmp[nl]) ? 1 : 2;
            } else if (ds[L] >= 0 && ds[nl] < 0) {
                // exactly 0 counts as outside (the `ds(i) < 0` membership rule); the
                // reference's error stop (:155-156) is then reached only by NaN
                pick = L + 1;  // oldlayer = packet%layer (1-based), then compared with 1
            } else if (ds[L] >= 0 && ds[nl] >= 0) {
                pk.tflag = true;
                break;
            } else {
                pk.tflag = true;  // "This should not be reached!" (:156)
                pk.flags |= 2;
                ++c.err;
                break;
            }
            int which = (pick == 1) ? L : nl;
            R Ri;
            bool refl;
            ++c.fres;
            if (pol.crossing_f64)
                refl = boundary_event<R, double>(sc64, which, L, nl, pos, dir, (R)pol.h, rng, Ri, c);
            else
                refl = boundary_event<R, R>(sc, which, L, nl, pos, dir, (R)pol.h, rng, Ri, c);
            pk.weight = pk.weight * Ri;
            tau = -std::log(rng.next());
            taurun = 0;
            if (!refl) {
                pk.layer = nl;
            } else {
                ++c.refl;
                pos = oldpos;
                pk.bounces += 1;
                if (pk.bounces > 1000) {
                    pk.tflag = true;
                    break;
                }
            }
        } else {
            pk.layer = nl;
        }
        if (pk.tflag) break;
    }
    if (by_tau) *by_tau = taurun >= tau;
    pk.pos = pos;
    pk.dir = dir;
    if (std::fabs(pos.x) > g.xmax) pk.tflag = true;
    if (std::fabs(pos.y) > g.ymax) pk.tflag = true;
    if (std::fabs(pos.z) > g.zmax) pk.tflag = true;
}

// scatter, src/photon.f90:713-779 (bias test p = 0 consumes one draw when g != 0).
// FP64: the reference's formulas.  FP32 (device semantics): the same angles from
// forms free of 1 - cos^2 cancellation -- 1 -+ cos(theta) factored out of the HG
// inverse CDF, and sin/cos(phi) of 2 pi u evaluated accurately.
inline void hg_angles(float hgg, float g2, float u, float& cost, float& sint) {
    float omc, opc;
    if (hgg == 0.0f) {
        omc = 2.0f * (1.0f - u);
        opc = 2.0f * u;
    } else {
        const float den = 1.0f - hgg + 2.0f * hgg * u;
        const float temp = (1.0f - g2) / den;
        omc = (1.0f - hgg) * (1.0f - u) * (temp + (1.0f - hgg)) / den;
        opc = (1.0f + hgg) * u * (1.0f + hgg + temp) / den;
    }
    cost = (omc < opc) ? 1.0f - omc : opc - 1.0f;
    sint = std::sqrt(omc * opc);
}
inline void hg_angles(double hgg, double g2, double u, double& cost, double& sint) {
    if (hgg == 0.0) {
        cost = 2.0 * u - 1.0;
    } else {
        const double temp = (1.0 - g2) / (1.0 - hgg + 2.0 * hgg * u);
        cost = (1.0 + g2 - temp * temp) / (2.0 * hgg);
    }
    sint = std::sqrt(1.0 - cost * cost);
}
inline void phi_angles(float u, float& cosp, float& sinp) {
    const double a = 2.0 * kPI * (double)u;
    cosp = (float)std::cos(a);
    sinp = (float)std::sin(a);
}
inline void phi_angles(double u, double& cosp, double& sinp) {
    const double phi = (2.0 * kPI) * u;
    cosp = std::cos(phi);
    sinp = (phi < kPI) ? std::sqrt(1.0 - cosp * cosp) : -std::sqrt(1.0 - cosp * cosp);
}

template <class R, class Rng>
void scatter(V3<R>& dir, R hgg, R g2, Rng& rng, double* cost_out = nullptr) {
    const R one = 1;
    R cost, sint;
    if (hgg == (R)0) {
        hg_angles(hgg, g2, rng.next(), cost, sint);
    } else {
        (void)rng.next();  // ran2() < p with p = 0 (:739)
        hg_angles(hgg, g2, rng.next(), cost, sint);
    }
    if (cost_out) *cost_out = (double)cost;
    R cosp, sinp;
    phi_angles(rng.next(), cosp, sinp);
    R uxx, uyy, uzz;
    R nx = dir.x, ny = dir.y, nz = dir.z;
    bool vertical = (one - std::fabs(nz) <= (R)1e-12);
    R temp = 0;
    if (!vertical) {
        // FP32 uses sqrt(nx^2+ny^2) (no cancellation near |nz| = 1); FP64 the reference form
        temp = (sizeof(R) == 4) ? std::sqrt(nx * nx + ny * ny) : std::sqrt(one - nz * nz);
        if (temp == (R)0) vertical = true;
    }
    if (vertical) {
        uxx = sint * cosp;
        uyy = sint * sinp;
        uzz = fsign(cost, nz);
    } else {
        uxx = sint * (nx * nz * cosp - ny * sinp) / temp + nx * cost;
        uyy = sint * (ny * nz * cosp + nx * sinp) / temp + ny * cost;
        uzz = -one * sint * cosp * temp + nz * cost;
    }
    dir = V3<R>{uxx, uyy, uzz};
}

// ---------------------------------------------------------------------------
// Emitters, src/photon.f90
template <class R, class Rng>
void emit(const smcrt_source& s, const GridD& g, Packet<R>& pk, Rng& rng) {
    const R TWOPI = (R)(2.0 * kPI);
    pk.tflag = false;
    pk.bounces = 0;
    pk.weight = 1;
    pk.layer = 0;
    pk.flags = 0;
    pk.nscatt = 0;
    V3<R> opos{(R)s.pos[0], (R)s.pos[1], (R)s.pos[2]}, odir{(R)s.dir[0], (R)s.dir[1], (R)s.dir[2]};
    V3<R> ep = opos;
    switch (s.kind) {
        case SMCRT_SRC_PENCIL:  // :464-505
            ep = opos;
            pk.dir = odir;
            break;
        case SMCRT_SRC_POINT: {  // :290-338
            ep = opos;
            R phi = rng.next() * TWOPI;
            R cosp = std::cos(phi), sinp = std::sin(phi);
            R u2 = rng.next();
            R cost = (R)2 * u2 - (R)1;
            R sint = (sizeof(R) == 4) ? (R)2 * std::sqrt(u2 * ((R)1 - u2)) : std::sqrt((R)1 - cost * cost);
            pk.dir = V3<R>{sint * cosp, sint * sinp, cost};
            break;
        }
        case SMCRT_SRC_UNIFORM: {  // :397-461
            pk.dir = odir;
            R rx = rng.next(), ry = rng.next();
            ep.x = (R)s.point1[0] + rx * (R)s.point2[0] + ry * (R)s.point3[0];
            ep.y = (R)s.point1[1] + rx * (R)s.point2[1] + ry * (R)s.point3[1];
            ep.z = (R)s.point1[2] + rx * (R)s.point2[2] + ry * (R)s.point3[2];
            break;
        }
        case SMCRT_SRC_CIRCULAR: {  // :214-287
            pk.dir = odir;
            R r = (R)s.radius * std::sqrt(rng.next());
            R theta = rng.next() * TWOPI;
            V3<R> a{1, 0, 0};
            V3<R> b = magnitude(odir);
            V3<R> p;
            if (std::fabs(a.x) == std::fabs(b.x) && std::fabs(a.y) == std::fabs(b.y) && std::fabs(a.z) == std::fabs(b.z)) {
                a = V3<R>{0, 0, 1};
                p = V3<R>{r * std::cos(theta), r * std::sin(theta), 0};
            } else {
                p = V3<R>{0, r * std::cos(theta), r * std::sin(theta)};
            }
            // rotationAlign(a, b) (sdfHelpers.f90:114-140), then p.R - origin
            V3<R> v{a.y * b.z - a.z * b.y, -a.x * b.z + a.z * b.x, a.x * b.y - a.y * b.x};
            R cc = dot(a, b);
            R k = (R)1 / ((R)1 + cc);
            R Vx[3][3] = {{0, v.z, -v.y}, {-v.z, 0, v.x}, {v.y, -v.x, 0}};  // Vx[row][col]
            R M[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    R s2 = 0;
                    for (int q = 0; q < 3; ++q) s2 += Vx[i][q] * Vx[q][j];
                    M[i][j] = (R)(i == j) + Vx[i][j] + s2 * k;
                }
            ep.x = M[0][0] * p.x + M[1][0] * p.y + M[2][0] * p.z - opos.x;
            ep.y = M[0][1] * p.x + M[1][1] * p.y + M[2][1] * p.z - opos.y;
            ep.z = M[0][2] * p.x + M[1][2] * p.y + M[2][2] * p.z - opos.z;
            break;
        }
        case SMCRT_SRC_ANNULUS: {  // :645-711
            R rlo = (R)s.radius, rhi = (R)s.radius_hi, radius;
            if (s.annulus_type == SMCRT_ANNULUS_TOPHAT) {
                radius = rlo + (rhi - rlo) * std::sqrt(rng.next());
            } else {  // rang (random_mod.f90:105-133), mid = (rhi-rlo)/2, sigma = 0.04
                R mid = (rhi - rlo) / (R)2, x, y, ss = 1;
                do {
                    x = (R)(-1) + rng.next() * (R)2;
                    y = (R)(-1) + rng.next() * (R)2;
                    ss = y * y + x * x;
                } while (ss >= (R)1);
                radius = mid + (R)0.04 * (x * std::sqrt((R)(-2) * std::log(ss) / ss));
            }
            R phi = TWOPI * rng.next();
            R angle = (R)(s.beta * kPI / 180.0);
            R cosp = std::cos(phi), sinp = std::sin(phi);
            ep = V3<R>{radius * cosp, radius * sinp, (R)(g.zmax - s.z_inset)};
            pk.dir = V3<R>{std::sin(angle) * cosp, std::sin(angle) * sinp, -std::cos(angle)};
            break;
        }
        case SMCRT_SRC_FOCUS: {  // :340-394
            R x = (R)(-g.xmax) + rng.next() * (R)(2.0 * g.xmax);
            R y = (R)(-g.ymax) + rng.next() * (R)(2.0 * g.ymax);
            ep = V3<R>{x, y, (R)(g.zmax - s.z_inset)};
            R dist = length(ep);
            V3<R> d = magnitude(V3<R>{(R)(-1) * ep.x / dist, (R)(-1) * ep.y / dist, (R)(-1) * ep.z / dist});
            R phi = std::atan2(d.y, d.x);
            R cosp = std::cos(phi), sinp = std::sin(phi);
            R cost = d.z, sint = std::sqrt((R)1 - cost * cost);
            pk.dir = V3<R>{sint * cosp, sint * sinp, cost};
            break;
        }
        default:
            ep = opos;
            pk.dir = odir;
    }
    pk.pos = V3<double>{(double)ep.x, (double)ep.y, (double)ep.z};
}

// Launch layer: innermost containing region (src/kernelsMod.f90:275-280).
template <class R>
int launch_layer(const Scene<R>& sc, const Scene<double>& sc64, const Pol& pol, V3<double> p, Counters& c) {
    thread_local std::vector<R> v;
    v.resize(sc.regions.size());
    c.sdf += sc.regions.size();
    return sweep(sc, sc64, pol, p, false, v.data()).lay;
}

// ---------------------------------------------------------------------------
// Detectors, src/detectors/detector_base.f90:106-162, detectors.f90, geometryMod.f90:217-270
struct Det {
    smcrt_detector d;
    int64_t off;
    int nb;             // total bins (1D) or per axis (2D)
    double bw, bwy;     // bin widths
    double e1[3], e2[3], n[3], width, height;
};

std::vector<Det> make_dets(const smcrt_detector* dets, int ndet, int64_t& total) {
    std::vector<Det> out;
    total = 0;
    for (int i = 0; i < ndet; ++i) {
        Det D{};
        D.d = dets[i];
        D.off = total;
        int nb = dets[i].nbins;
        if (dets[i].kind == SMCRT_DET_CAMERA) {
            D.nb = nb + 1;
            D.bw = D.bwy = (nb == 0) ? 1.0 : dets[i].maxval / (double)D.nb;
            for (int a = 0; a < 3; ++a) {
                D.e1[a] = dets[i].p2[a] - dets[i].pos[a];
                D.e2[a] = dets[i].p3[a] - dets[i].pos[a];
            }
            D.width = std::sqrt(D.e1[0] * D.e1[0] + D.e1[1] * D.e1[1] + D.e1[2] * D.e1[2]);
            D.height = std::sqrt(D.e2[0] * D.e2[0] + D.e2[1] * D.e2[1] + D.e2[2] * D.e2[2]);
            double nx = D.e2[1] * D.e1[2] - D.e2[2] * D.e1[1];
            double ny = -D.e2[0] * D.e1[2] + D.e2[2] * D.e1[0];
            double nz = D.e2[0] * D.e1[1] - D.e2[1] * D.e1[0];
            double ln = std::sqrt(nx * nx + ny * ny + nz * nz);
            D.n[0] = nx / ln; D.n[1] = ny / ln; D.n[2] = nz / ln;
            total += (int64_t)D.nb * D.nb;
        } else {
            D.nb = nb + 1;
            if (nb == 0) D.bw = 1.0;
            else if (dets[i].kind == SMCRT_DET_CIRCLE) D.bw = dets[i].maxval / (double)(nb - 1);
            else D.bw = dets[i].maxval / (double)nb;
            total += D.nb;
        }
        out.push_back(D);
    }
    return out;
}

inline int64_t nint_(double x) { return (int64_t)std::llround(x); }  // Fortran nint: half away from zero

// returns global bin or -1
// intersectPlane, src/geometryMod.f90:217-241: the ray l0 + t l meets the plane
// through p0 with normal n from its front side (n . l > 1e-6) at t >= 0.
inline bool intersect_plane(const double n[3], const double p0[3], const double l0[3], const double l[3],
                            double& t) {
    const double denom = n[0] * l[0] + n[1] * l[1] + n[2] * l[2];
    if (!(denom > 1e-6)) return false;
    t = ((p0[0] - l0[0]) * n[0] + (p0[1] - l0[1]) * n[1] + (p0[2] - l0[2]) * n[2]) / denom;
    return t >= 0.0;
}

// intersectCircle, src/geometryMod.f90:244-270: the plane hit lies within radius of p0.
inline bool intersect_circle(const double n[3], const double p0[3], double radius, const double l0[3],
                             const double l[3], double& t) {
    t = 0.0;
    if (!intersect_plane(n, p0, l0, l, t)) return false;
    const double q[3] = {l0[0] + l[0] * t - p0[0], l0[1] + l[1] * t - p0[1], l0[2] + l[2] * t - p0[2]};
    return std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) <= radius;
}

int64_t det_bin(const Det& D, const double p[3], const double l[3], double value, int layer1) {
    const smcrt_detector& d = D.d;
    if (d.layer != layer1) return -1;
    if (d.kind == SMCRT_DET_ANNULUS) {
        double r = std::sqrt((p[0] - d.pos[0]) * (p[0] - d.pos[0]) + (p[1] - d.pos[1]) * (p[1] - d.pos[1]) +
                             (p[2] - d.pos[2]) * (p[2] - d.pos[2]));
        if (!(r >= d.r1 && r <= d.r2)) return -1;
    } else if (d.kind == SMCRT_DET_CIRCLE) {
        double t;
        if (!intersect_circle(d.dir, d.pos, d.r1, p, l, t)) return -1;
        if (t > 5e-3) return -1;
    } else {  // camera
        double num = (d.pos[0] - p[0]) * D.n[0] + (d.pos[1] - p[1]) * D.n[1] + (d.pos[2] - p[2]) * D.n[2];
        double den = l[0] * D.n[0] + l[1] * D.n[1] + l[2] * D.n[2];
        double t = num / den;
        if (!(t >= 0)) return -1;
        double v[3] = {p[0] + t * l[0] - d.pos[0], p[1] + t * l[1] - d.pos[1], p[2] + t * l[2] - d.pos[2]};
        double pr1 = (v[0] * D.e1[0] + v[1] * D.e1[1] + v[2] * D.e1[2]) / D.width;
        double pr2 = (v[0] * D.e2[0] + v[1] * D.e2[1] + v[2] * D.e2[2]) / D.height;
        if (!((pr1 < D.width && pr1 > 0) && (pr2 < D.height && pr2 > 0))) return -1;
        double x = p[2] + d.pos[0], y = p[1] + d.pos[1];
        int64_t ix = std::min((int64_t)(x / D.bw) + 1, (int64_t)D.nb);
        int64_t iy = std::min((int64_t)(y / D.bwy) + 1, (int64_t)D.nb);
        if (ix < 1) ix = D.nb;
        if (iy < 1) iy = D.nb;
        return D.off + (ix - 1) + (int64_t)D.nb * (iy - 1);
    }
    int64_t idx = std::min(nint_(value / D.bw) + 1, (int64_t)D.nb);
    if (idx < 1) idx = 1;  // value >= 0 on every reference path; guard the array
    return D.off + idx - 1;
}

// ---------------------------------------------------------------------------
// The packet loops (src/kernelsMod.f90).
// The GPU's FP32 near-surface band: 16 FP32 ulps of the largest grid half-size,
// at least twice eps.
inline double near_band(const smcrt_grid* g, double eps) {
    int e;
    std::frexp(std::max(g->xmax, std::max(g->ymax, g->zmax)), &e);
    return std::max(2.0 * eps, 16.0 * std::ldexp(1.0, e - 24));
}

struct RunArgs {
    const smcrt_scene* scene;
    const smcrt_grid* grid;
    const smcrt_source* src;
    std::vector<Det> dets;
    int kernel, end_early;
    Pol pol;
    int64_t first, count;
    uint64_t seed;
    uint32_t instance;
    const double* uniforms;
    const int64_t* offsets;
    Tally tally;
    double* jmean2 = nullptr;  // per-voxel sum over packets of the packet's score squared
    double* bins;
    smcrt_packet_state* states;
    const struct AdjArgs* adj = nullptr;  // perturbation MC gradient (pathlength kernel)
};

// Perturbation Monte Carlo (likelihood-ratio) reference gradient of
// L = sum_v w[v] jmean[v] + sum_b h[b] bins[b] with respect to each region
// group's (mua, mus, g): per packet, its contribution C to L times the derivative
// of the log density of its whole path.  That density is, per flight, the
// survival exp(-kappa l) in every region crossed and, where the flight ends at
// its optical depth, the interaction density kappa; per interaction the roulette
// probability mus/kappa (scatter) or mua/kappa (absorption); per scatter the
// Henyey-Greenstein density of the sampled cos(theta).  Fresnel choices and
// emission do not depend on these parameters.
struct AdjArgs {
    const double* w;        // voxel weights, nxg*nyg*nzg
    const double* h;        // detector bin weights or null
    const int32_t* group;   // region -> group, -1: not differentiated
    int ngroups;
};

// d/dg log p_HG(mu; g), p_HG = (1 - g^2) / (2 (1 + g^2 - 2 g mu)^(3/2))
inline double hg_score(double g, double mu) {
    return -2.0 * g / (1.0 - g * g) - 3.0 * (g - mu) / (1.0 + g * g - 2.0 * g * mu);
}

template <class R, class Rng>
void run_packet(const Scene<R>& sc, const Scene<double>& sc64, const GridD& g, const RunArgs& A, Rng& rng,
                Counters& c, int64_t pid) {
    Tally t = A.tally;
    thread_local std::unordered_map<int64_t, double> scores;
    if (A.jmean2) {
        scores.clear();
        t.packet = &scores;
    }
    struct Flush {  // at every return: the packet's squared scores
        const RunArgs& A;
        std::unordered_map<int64_t, double>& m;
        ~Flush() {
            if (!A.jmean2) return;
            for (const auto& kv : m) {
                double* a = A.jmean2 + kv.first;
#pragma omp atomic
                *a += kv.second * kv.second;
            }
        }
    } flush{A, scores};
    Packet<R> pk{};
    const AdjArgs* adj = (A.kernel == SMCRT_KERNEL_PATHLENGTH) ? A.adj : nullptr;
    double C = 0, S[3][kAdjGroups] = {};
    thread_local std::vector<double> len;
    double* lp = nullptr;
    bool by_tau = false;
    if (adj) {
        t.w = adj->w;
        t.csum = &C;
        len.assign(sc.regions.size(), 0.0);
        lp = len.data();
    }
    auto mua_of = [&](int r) { return A.scene->regions[r].mua; };
    auto mus_of = [&](int r) { return A.scene->regions[r].mus; };
    // score of the flights just traced: survival per region, and the interaction
    // density where the last flight ended at its optical depth
    auto flights = [&]() {
        for (size_t r = 0; r < len.size(); ++r) {
            const int gi = adj->group[r];
            if (gi >= 0 && len[r] != 0.0) {
                S[0][gi] -= len[r];
                S[1][gi] -= len[r];
            }
            len[r] = 0.0;
        }
        const int gi = adj->group[pk.layer];
        if (by_tau && gi >= 0) {
            const double k = mua_of(pk.layer) + mus_of(pk.layer);
            S[0][gi] += 1.0 / k;
            S[1][gi] += 1.0 / k;
        }
    };
    emit(*A.src, g, pk, rng);
    pk.layer = launch_layer(sc, sc64, A.pol, pk.pos, c);
    tauint2(sc, sc64, g, A.pol, pk, rng, t, c, lp, adj ? &by_tau : nullptr);
    if (adj) flights();
    if (A.kernel == SMCRT_KERNEL_WEIGHT) {  // weight_scatter :99-134
        while (!pk.tflag) {
            const Region<R>& rg = sc.regions[pk.layer];
            R wa = pk.weight * ((R)1 - rg.albedo);
            pk.weight = pk.weight - wa;
            int ci, cj, ck;
            cell_of<R>(g, V3<double>{pk.pos.x + g.xmax, pk.pos.y + g.ymax, pk.pos.z + g.zmax}, ci, cj, ck);
            if (ci < 1 || cj < 1 || ck < 1) {
                pk.tflag = true;
                break;
            }
            t.add(cell_index(g, ci, cj, ck), (double)wa);
            scatter(pk.dir, rg.hgg, rg.g2, rng);
            ++c.scat;
            if (pk.weight < (R)0.01) {  // THRESHOLD, CHANCE (constants.f90:28-30)
                if (rng.next() < (R)0.1) pk.weight = pk.weight / (R)0.1;
                else {
                    pk.tflag = true;
                    break;
                }
            }
            tauint2(sc, sc64, g, A.pol, pk, rng, t, c);
        }
    } else {  // pathlength_scatter :285-300, test_kernel :408-436
        while (!pk.tflag) {
            R ran = rng.next();
            const Region<R>& rg = sc.regions[pk.layer];
            const int gi = adj ? adj->group[pk.layer] : -1;
            if (ran < rg.albedo) {
                double mu = 0.0;
                scatter(pk.dir, rg.hgg, rg.g2, rng, adj ? &mu : nullptr);
                if (gi >= 0) {  // roulette mus/kappa, then the phase function
                    // an albedo-1 region (mua < 1e-9, init_mono, opticalProperties.f90:115-119)
                    // scatters with probability 1 whatever its parameters: no roulette term
                    const double k = mua_of(pk.layer) + mus_of(pk.layer);
                    if (!(mua_of(pk.layer) < 1e-9)) {
                        S[0][gi] -= 1.0 / k;
                        S[1][gi] += 1.0 / mus_of(pk.layer) - 1.0 / k;
                    }
                    const double hg = A.scene->regions[pk.layer].hgg;
                    S[2][gi] += (hg == 0.0) ? 3.0 * mu : hg_score(hg, mu);
                }
                ++c.scat;
                c.nscatt += 1.0;
                pk.nscatt += 1;
                if (A.kernel == SMCRT_KERNEL_TEST) {
                    int s = pk.nscatt;
                    if (s >= 1 && s <= 4) {
                        double px = pk.pos.x, py = pk.pos.y, pz = pk.pos.z;
                        c.mom[(s - 1) * 3 + 0] += px;
                        c.mom[(s - 1) * 3 + 1] += py;
                        c.mom[(s - 1) * 3 + 2] += pz;
                        c.mom[12 + (s - 1) * 3 + 0] += px * px;
                        c.mom[12 + (s - 1) * 3 + 1] += py * py;
                        c.mom[12 + (s - 1) * 3 + 2] += pz * pz;
                    } else if (A.end_early) {
                        pk.tflag = true;
                    }
                }
            } else {
                if (gi >= 0) {  // roulette mua/kappa
                    const double k = mua_of(pk.layer) + mus_of(pk.layer);
                    S[0][gi] += 1.0 / mua_of(pk.layer) - 1.0 / k;
                    S[1][gi] -= 1.0 / k;
                }
                pk.tflag = true;
                break;
            }
            tauint2(sc, sc64, g, A.pol, pk, rng, t, c, lp, adj ? &by_tau : nullptr);
            if (adj) flights();
        }
    }
    // detectors (:302-306 / :136-140)
    if (!A.dets.empty() && A.kernel != SMCRT_KERNEL_TEST) {
        double p[3] = {(double)pk.pos.x, (double)pk.pos.y, (double)pk.pos.z};
        double l[3] = {(double)pk.dir.x, (double)pk.dir.y, (double)pk.dir.z};
        double value = (A.kernel == SMCRT_KERNEL_WEIGHT)
                           ? (double)pk.weight
                           : std::sqrt(pk.pos.x * pk.pos.x + pk.pos.y * pk.pos.y);
        for (const Det& D : A.dets) {
            int64_t b = det_bin(D, p, l, value, pk.layer + 1);
            if (b >= 0) {
                double* a = A.bins + b;
#pragma omp atomic
                *a += 1.0;
                if (adj && adj->h) C += adj->h[b];
            }
        }
    }
    if (adj) {
        for (int k = 0; k < 3; ++k)
            for (int gi = 0; gi < adj->ngroups; ++gi) c.adj[k * kAdjGroups + gi] += C * S[k][gi];
        c.loss += C;
    }
    c.draws += (uint64_t)rng.ndraws;
    if (A.states) {
        smcrt_packet_state& s = A.states[pid - A.first];
        s.pos[0] = pk.pos.x; s.pos[1] = pk.pos.y; s.pos[2] = pk.pos.z;
        s.dir[0] = pk.dir.x; s.dir[1] = pk.dir.y; s.dir[2] = pk.dir.z;
        s.weight = pk.weight;
        s.layer = pk.layer + 1;
        s.nscatt = pk.nscatt;
        s.ndraws = (int32_t)rng.ndraws;
        s.flags = pk.flags | rng.flags;
    }
}

template <class R>
void run_all(const RunArgs& A, smcrt_stats* st, int threads, double* adj_out = nullptr) {
    Scene<R> sc = make_scene<R>(A.scene);
    Scene<double> sc64 = make_scene<double>(A.scene);
    GridD g(*A.grid);
    Counters tot;
    const int64_t n = A.count;
#pragma omp parallel num_threads(threads)
    {
        Counters c;
#pragma omp for schedule(dynamic, 16)
        for (int64_t q = 0; q < n; ++q) {
            int64_t pid = A.first + q;
            if (A.uniforms) {
                InjectedStream<R> rng{A.uniforms + A.offsets[q], A.offsets[q + 1] - A.offsets[q]};
                run_packet<R>(sc, sc64, g, A, rng, c, pid);
            } else {
                PhiloxStream<R> rng(A.seed, A.instance, (uint64_t)pid);
                run_packet<R>(sc, sc64, g, A, rng, c, pid);
            }
        }
#pragma omp critical
        {
            tot.sdf += c.sdf; tot.vox += c.vox; tot.steps += c.steps; tot.scat += c.scat;
            tot.fres += c.fres; tot.refl += c.refl; tot.stepcap += c.stepcap; tot.err += c.err;
            tot.draws += c.draws; tot.nscatt += c.nscatt;
            for (int i = 0; i < 24; ++i) tot.mom[i] += c.mom[i];
            for (int i = 0; i < 3 * kAdjGroups; ++i) tot.adj[i] += c.adj[i];
            tot.loss += c.loss;
        }
    }
    if (adj_out && A.adj) {  // [d/d mua of groups..., d/d mus..., d/d g...], then L
        const int G = A.adj->ngroups;
        for (int k = 0; k < 3; ++k)
            for (int gi = 0; gi < G; ++gi) adj_out[k * G + gi] = tot.adj[k * kAdjGroups + gi];
        adj_out[3 * G] = tot.loss;
    }
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->nscatt = tot.nscatt;
        st->packets = (uint64_t)n;
        st->sdf_evals = tot.sdf;
        st->voxel_segments = tot.vox;
        st->trace_steps = tot.steps;
        st->scatters = tot.scat;
        st->fresnel_events = tot.fres;
        st->reflections = tot.refl;
        st->kills_step_cap = tot.stepcap;
        st->kills_error = tot.err;
        st->rng_draws = tot.draws;
        for (int i = 0; i < 24; ++i) st->moments[i] = tot.mom[i];
    }
}

template <class R>
V3<R> v3(const double* p) { return V3<R>{(R)p[0], (R)p[1], (R)p[2]}; }

}  // namespace

// ===========================================================================
// render_sub, src/sdfs/sdf_base.f90:302-346: ns = nint(samples / 2) (:320),
// wid = extent / ns (:322), voxel (i, j, k) at ((i - ns) wid) (:326-331), the
// minval over regions (:332-336) stored as real(sp), image(i, j, k) column-major.
template <class R>
static void render_t(const smcrt_scene* scene, const int32_t* samples, const double* extent, float* image) {
    const Scene<R> sc = make_scene<R>(scene);
    double ns[3], wid[3];
    for (int a = 0; a < 3; ++a) {
        ns[a] = std::round(samples[a] / 2.0);  // nint: half away from zero
        wid[a] = extent[a] / ns[a];
    }
    const int64_t n0 = samples[0], n1 = samples[1], n2 = samples[2];
#pragma omp parallel for schedule(dynamic)
    for (int64_t k = 1; k <= n2; ++k) {
        const double z = ((double)k - ns[2]) * wid[2];
        for (int64_t j = 1; j <= n1; ++j) {
            const double y = ((double)j - ns[1]) * wid[1];
            for (int64_t i = 1; i <= n0; ++i) {
                const double x = ((double)i - ns[0]) * wid[0];
                const V3<R> pos{(R)x, (R)y, (R)z};
                R d = eval_region(sc, 0, pos);
                for (int r = 1; r < scene->nregions; ++r) {
                    const R e = eval_region(sc, r, pos);
                    if (e < d) d = e;
                }
                image[(i - 1) + n0 * ((j - 1) + n1 * (k - 1))] = (float)d;
            }
        }
    }
}

extern "C" {

int32_t oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int64_t oracle_detector_bins(const smcrt_detector* dets, int32_t ndet) {
    int64_t total = 0;
    if (ndet > 0) make_dets(dets, ndet, total);
    return total;
}

int32_t oracle_run(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* src,
                   const smcrt_detector* dets, int32_t ndet, int32_t kernel, int32_t end_early,
                   const oracle_policy* pol, int64_t first, int64_t count, uint64_t seed,
                   uint32_t instance, const double* uniforms, const int64_t* offsets,
                   double* jmean, double* det_bins, smcrt_stats* stats,
                   smcrt_packet_state* states, double* jmean2) {
    if (validate_scene(scene) || !grid || !src || !pol || count < 0 || (ndet > 0 && !dets)) return SMCRT_ERR_ARG;
    if (grid->nxg <= 0 || grid->nyg <= 0 || grid->nzg <= 0) return SMCRT_ERR_ARG;
    if (uniforms && !offsets) return SMCRT_ERR_ARG;
    RunArgs A{};
    A.scene = scene;
    A.grid = grid;
    A.src = src;
    int64_t nbins = 0;
    if (ndet > 0) A.dets = make_dets(dets, ndet, nbins);
    for (const Det& D : A.dets) {
        if (D.d.layer < 1 || D.d.layer > scene->nregions) return SMCRT_ERR_ARG;
    }
    A.kernel = kernel;
    A.end_early = end_early;
    A.pol.eps = pol->eps;
    A.pol.delta = pol->delta;
    A.pol.h = pol->normal_h;
    A.pol.ref_dda = pol->ref_dda != 0;
    A.pol.crossing_f64 = pol->crossing_f64 != 0;
    A.pol.kill_le = pol->ref_dda == 0;  // device semantics
    A.pol.near_f64 = pol->near_surface_f64 != 0;
    A.pol.near_band = near_band(grid, pol->eps);
    A.pol.max_steps = pol->max_trace_steps > 0 ? pol->max_trace_steps : 1000000;
    A.first = first;
    A.count = count;
    A.seed = seed;
    A.instance = instance;
    A.uniforms = uniforms;
    A.offsets = offsets;
    const int64_t ncell = (int64_t)grid->nxg * grid->nyg * grid->nzg;
    std::vector<float> j32;
    if (jmean) {
        if (pol->tally_f32) {
            j32.assign(ncell, 0.0f);
            A.tally.j32 = j32.data();
        } else {
            std::fill(jmean, jmean + ncell, 0.0);
            A.tally.j64 = jmean;
        }
    }
    std::vector<double> binbuf;
    if (det_bins) {
        std::fill(det_bins, det_bins + nbins, 0.0);
        A.bins = det_bins;
    } else {
        binbuf.assign(std::max<int64_t>(nbins, 1), 0.0);
        A.bins = binbuf.data();
    }
    A.states = states;
    if (jmean2) {
        std::fill(jmean2, jmean2 + ncell, 0.0);
        A.jmean2 = jmean2;
    }
    int threads = pol->threads > 0 ? pol->threads : oracle_max_threads();
    if (pol->precision == SMCRT_FP32) run_all<float>(A, stats, threads);
    else run_all<double>(A, stats, threads);
    if (jmean && pol->tally_f32)
        for (int64_t i = 0; i < ncell; ++i) jmean[i] = (double)j32[i];
    return SMCRT_OK;
}

int32_t oracle_adjoint(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* src,
                       const smcrt_detector* dets, int32_t ndet, const oracle_policy* pol, int64_t nphotons,
                       uint64_t seed, const double* w, const double* h, const int32_t* region_group,
                       int32_t ngroups, double* grad) {
    if (validate_scene(scene) || !grid || !src || !pol || !w || !region_group || !grad || nphotons < 0 ||
        ngroups < 1 || ngroups > kAdjGroups || (ndet > 0 && !dets))
        return SMCRT_ERR_ARG;
    if (grid->nxg <= 0 || grid->nyg <= 0 || grid->nzg <= 0) return SMCRT_ERR_ARG;
    for (int r = 0; r < scene->nregions; ++r)
        if (region_group[r] < -1 || region_group[r] >= ngroups) return SMCRT_ERR_ARG;
    RunArgs A{};
    A.scene = scene;
    A.grid = grid;
    A.src = src;
    int64_t nbins = 0;
    if (ndet > 0) A.dets = make_dets(dets, ndet, nbins);
    for (const Det& D : A.dets)
        if (D.d.layer < 1 || D.d.layer > scene->nregions) return SMCRT_ERR_ARG;
    A.kernel = SMCRT_KERNEL_PATHLENGTH;
    A.pol.eps = pol->eps;
    A.pol.delta = pol->delta;
    A.pol.h = pol->normal_h;
    A.pol.ref_dda = pol->ref_dda != 0;
    A.pol.crossing_f64 = pol->crossing_f64 != 0;
    A.pol.kill_le = pol->ref_dda == 0;
    A.pol.near_f64 = pol->near_surface_f64 != 0;
    A.pol.near_band = near_band(grid, pol->eps);
    A.pol.max_steps = pol->max_trace_steps > 0 ? pol->max_trace_steps : 1000000;
    A.first = 0;
    A.count = nphotons;
    A.seed = seed;
    std::vector<double> binbuf(std::max<int64_t>(nbins, 1), 0.0);
    A.bins = binbuf.data();
    AdjArgs adj{w, h, region_group, ngroups};
    A.adj = &adj;
    const int threads = pol->threads > 0 ? pol->threads : oracle_max_threads();
    if (pol->precision == SMCRT_FP32) run_all<float>(A, nullptr, threads, grad);
    else run_all<double>(A, nullptr, threads, grad);
    return SMCRT_OK;
}

int32_t oracle_intersect_plane(const double* n, const double* p0, const double* l0, const double* l, double* t) {
    double tt = 0.0;
    const bool hit = intersect_plane(n, p0, l0, l, tt);
    if (t) *t = tt;
    return hit ? 1 : 0;
}

int32_t oracle_intersect_circle(const double* n, const double* p0, double radius, const double* l0, const double* l,
                                double* t) {
    double tt = 0.0;
    const bool hit = intersect_circle(n, p0, radius, l0, l, tt);
    if (t) *t = tt;
    return hit ? 1 : 0;
}

int32_t oracle_eval_sdf(const smcrt_scene* scene, int32_t precision, const double* pts, int64_t npts, double* out) {
    if (validate_scene(scene) || !pts || !out) return SMCRT_ERR_ARG;
    const int nr = scene->nregions;
    if (precision == SMCRT_FP32) {
        Scene<float> sc = make_scene<float>(scene);
        for (int64_t p = 0; p < npts; ++p)
            for (int r = 0; r < nr; ++r) out[p * nr + r] = eval_region(sc, r, v3<float>(pts + 3 * p));
    } else {
        Scene<double> sc = make_scene<double>(scene);
        for (int64_t p = 0; p < npts; ++p)
            for (int r = 0; r < nr; ++r) out[p * nr + r] = eval_region(sc, r, v3<double>(pts + 3 * p));
    }
    return SMCRT_OK;
}

int32_t oracle_render(const smcrt_scene* scene, int32_t precision, const int32_t* samples, const double* extent,
                      float* image) {
    if (validate_scene(scene) || !samples || !extent || !image) return SMCRT_ERR_ARG;
    for (int a = 0; a < 3; ++a)
        if (samples[a] < 1) return SMCRT_ERR_ARG;
    if (precision == SMCRT_FP32) render_t<float>(scene, samples, extent, image);
    else render_t<double>(scene, samples, extent, image);
    return SMCRT_OK;
}

int32_t oracle_calc_normal(const smcrt_scene* scene, int32_t region0, double h, const double* pts, int64_t npts,
                           double* out) {
    if (validate_scene(scene) || region0 < 0 || region0 >= scene->nregions || !pts || !out) return SMCRT_ERR_ARG;
    Scene<double> sc = make_scene<double>(scene);
    for (int64_t p = 0; p < npts; ++p) {
        V3<double> n = calc_normal(sc, region0, v3<double>(pts + 3 * p), h);
        out[3 * p] = n.x; out[3 * p + 1] = n.y; out[3 * p + 2] = n.z;
    }
    return SMCRT_OK;
}

int32_t oracle_fresnel(int32_t precision, const double* I, const double* N, const double* n1, const double* n2,
                       int64_t n, double* R) {
    for (int64_t i = 0; i < n; ++i) {
        if (precision == SMCRT_FP32) R[i] = fresnel(v3<float>(I + 3 * i), v3<float>(N + 3 * i), (float)n1[i], (float)n2[i]);
        else R[i] = fresnel(v3<double>(I + 3 * i), v3<double>(N + 3 * i), n1[i], n2[i]);
    }
    return SMCRT_OK;
}

int32_t oracle_reflect_refract(int32_t precision, const double* I, const double* N, const double* n1,
                               const double* n2, const double* u, int64_t n, double* Iout, int32_t* refl) {
    for (int64_t i = 0; i < n; ++i) {
        if (precision == SMCRT_FP32) {
            V3<float> d = v3<float>(I + 3 * i), nn = v3<float>(N + 3 * i);
            float Rr = fresnel(d, nn, (float)n1[i], (float)n2[i]);
            bool r = (float)u[i] <= Rr;
            d = r ? reflect(d, nn) : refract(d, nn, (float)n1[i] / (float)n2[i]);
            Iout[3 * i] = d.x; Iout[3 * i + 1] = d.y; Iout[3 * i + 2] = d.z;
            refl[i] = r;
        } else {
            V3<double> d = v3<double>(I + 3 * i), nn = v3<double>(N + 3 * i);
            double Rr = fresnel(d, nn, n1[i], n2[i]);
            bool r = u[i] <= Rr;
            d = r ? reflect(d, nn) : refract(d, nn, n1[i] / n2[i]);
            Iout[3 * i] = d.x; Iout[3 * i + 1] = d.y; Iout[3 * i + 2] = d.z;
            refl[i] = r;
        }
    }
    return SMCRT_OK;
}

int32_t oracle_scatter_dir(int32_t precision, const double* dir_in, const double* g, const double* u, int64_t n,
                           double* dir_out) {
    for (int64_t i = 0; i < n; ++i) {
        InjectedStream<double> s64{u + 3 * i, 3};
        if (precision == SMCRT_FP32) {
            InjectedStream<float> s{u + 3 * i, 3};
            V3<float> d = v3<float>(dir_in + 3 * i);
            float gg = (float)g[i];
            scatter(d, gg, (float)(g[i] * g[i]), s);
            dir_out[3 * i] = d.x; dir_out[3 * i + 1] = d.y; dir_out[3 * i + 2] = d.z;
        } else {
            V3<double> d = v3<double>(dir_in + 3 * i);
            scatter(d, g[i], g[i] * g[i], s64);
            dir_out[3 * i] = d.x; dir_out[3 * i + 1] = d.y; dir_out[3 * i + 2] = d.z;
        }
    }
    return SMCRT_OK;
}

int32_t oracle_philox(const uint32_t* key2, const uint32_t* ctr4, int64_t n, uint32_t* out4) {
    for (int64_t i = 0; i < n; ++i) philox(key2 + 2 * i, ctr4 + 4 * i, out4 + 4 * i);
    return SMCRT_OK;
}

int32_t oracle_emit(const smcrt_scene* scene, const smcrt_grid* grid, const smcrt_source* src, int32_t precision,
                    int64_t first, int64_t npk, uint64_t seed, double* pos, double* dir, int32_t* layer) {
    if (validate_scene(scene) || !grid || !src) return SMCRT_ERR_ARG;
    GridD g(*grid);
    Counters c;
    // the launch layer as the transport kernels take it: FP32 with the
    // near-surface FP64 rule and the FP32 default epsilon, or FP64
    Pol pol{};
    pol.near_f64 = precision == SMCRT_FP32;
    pol.eps = 1e-8;
    pol.near_band = near_band(grid, pol.eps);
    const Scene<double> sc64 = make_scene<double>(scene);
    for (int64_t q = 0; q < npk; ++q) {
        if (precision == SMCRT_FP32) {
            Scene<float> sc = make_scene<float>(scene);
            PhiloxStream<float> rng(seed, 0, (uint64_t)(first + q));
            Packet<float> pk{};
            emit(*src, g, pk, rng);
            layer[q] = launch_layer(sc, sc64, pol, pk.pos, c) + 1;
            pos[3 * q] = pk.pos.x; pos[3 * q + 1] = pk.pos.y; pos[3 * q + 2] = pk.pos.z;
            dir[3 * q] = pk.dir.x; dir[3 * q + 1] = pk.dir.y; dir[3 * q + 2] = pk.dir.z;
        } else {
            PhiloxStream<double> rng(seed, 0, (uint64_t)(first + q));
            Packet<double> pk{};
            emit(*src, g, pk, rng);
            layer[q] = launch_layer(sc64, sc64, pol, pk.pos, c) + 1;
            pos[3 * q] = pk.pos.x; pos[3 * q + 1] = pk.pos.y; pos[3 * q + 2] = pk.pos.z;
            dir[3 * q] = pk.dir.x; dir[3 * q + 1] = pk.dir.y; dir[3 * q + 2] = pk.dir.z;
        }
    }
    return SMCRT_OK;
}

int64_t oracle_detector_bin(const smcrt_detector* dets, int32_t ndet, int32_t det, const double* pos,
                            const double* dir, double value, int32_t layer1) {
    int64_t total = 0;
    std::vector<Det> D = make_dets(dets, ndet, total);
    if (det < 0 || det >= ndet) return -1;
    return det_bin(D[det], pos, dir, value, layer1);
}

}  // extern "C"
