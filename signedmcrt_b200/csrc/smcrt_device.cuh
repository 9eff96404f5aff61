// smcrt_device.cuh -- device building blocks of the B200 photon-packet transport.
//
// Everything here is templated on the transport precision R (float or double);
// boundary events (normal + Fresnel + reflect/refract) always run in double.
// Reference formulas are cited by file:line of the signedMCRT sources.
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "../../include/smcrt.h"

namespace smcrt {

// Scenes up to kMaxRegions regions and kMaxPrims primitives travel in the
// launch's parameter block (constant bank: warp-broadcast operands); larger
// scenes, up to kMaxRegionsDev regions, live in device memory (SceneG).
constexpr int kMaxPrims = 32;
constexpr int kMaxRegions = 16;
constexpr int kMaxRegionsDev = 255;
constexpr int kMaxPrimsDev = 4096;
constexpr int kMaxDetectors = 16;
// Detector bins privatized per CTA as 32-bit counts in shared memory (16 KiB);
// larger bin sets (camera images) add straight into the global FP64 bins.
constexpr int kMaxSharedBins = 4096;
constexpr int kMaxTallyCopies = 16;
constexpr int kMaxAdjGroups = 5;  // parameter groups of one adjoint launch (3 parameters each)
constexpr double kPI = 3.14159265358979323846264338327950288;

// Device status flags (smcrt_stats.device_status).
enum : int { STATUS_STEP_CAP = 1, STATUS_ERROR_STATE = 2, STATUS_STREAM_EXHAUSTED = 4, STATUS_BAD_INDEX = 8, STATUS_ABORTED = 16 };

// ---------------------------------------------------------------------------
template <class R>
struct V3 {
    R x, y, z;
};
template <class R> __host__ __device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> __host__ __device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> __host__ __device__ __forceinline__ V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> __host__ __device__ __forceinline__ V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> __device__ __forceinline__ R dot3(V3<R> a, V3<R> b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
template <class R> __device__ __forceinline__ R len3(V3<R> a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
template <class R> __device__ __forceinline__ R clampr(R x, R lo, R hi) { return fmin(fmax(x, lo), hi); }
template <class R> __device__ __forceinline__ R fsign(R a, R b) { return copysign(fabs(a), b); }  // Fortran sign(a,b)
__device__ __forceinline__ void sincos_r(float x, float* s, float* c) { sincosf(x, s, c); }
__device__ __forceinline__ void sincos_r(double x, double* s, double* c) { sincos(x, s, c); }
__device__ __forceinline__ float cospi_r(float x) { return cospif(x); }
__device__ __forceinline__ double cospi_r(double x) { return cospi(x); }

// ---------------------------------------------------------------------------
// Scene tables (kernel-parameter resident: constant bank, warp-broadcast reads).
template <class R>
struct DPrim {
    R m[12];  // row-vector affine, m[3*i+j] = M[i][j]
    R q[8];
    int kind;
    int nmods;   // modifiers, innermost first
    int mod[2];
    R mp[2][3];
};
template <class R>
struct DRegion {
    int first, n, op, pad;
    R k, kappa, albedo, hgg, g2, nidx;
    R mus, mua;  // for the adjoint's scatter/absorption terms
};

// Optical properties of one batch instance, per region (the per-region fields of
// DRegion; the geometry is shared by all instances of a batch).
template <class R>
struct InstOptics {
    R kappa[kMaxRegions], albedo[kMaxRegions], hgg[kMaxRegions], g2[kMaxRegions], nidx[kMaxRegions];
    double nidx64[kMaxRegions];
};

template <class R>
struct SceneT {
    int nregions, nprims;
    int has_mods, pad;  // some primitive carries modifiers
    DPrim<R> prim[kMaxPrims];
    DRegion<R> region[kMaxRegions];
};

// A scene in device memory (the same tables behind pointers, read through the
// L1 cache with warp-uniform addresses), with a bounding sphere per region:
// bound[4 r .. 4 r + 3] = world centre and radius, radius < 0 when the region
// has none (see sweep_regions).  cull_margin covers the rounding of the test.
template <class R>
struct SceneG {
    int nregions, nprims;
    int has_mods, pad;
    const DPrim<R>* prim;
    const DRegion<R>* region;
    const R* bound;
    R cull_margin;
};

// pos .dot. transform, src/vector_class.f90:292-304
template <class R>
__device__ __forceinline__ V3<R> xform(const R* m, V3<R> a) {
    V3<R> d;
    d.x = m[0] * a.x + m[3] * a.y + m[6] * a.z + m[9];
    d.y = m[1] * a.x + m[4] * a.y + m[7] * a.z + m[10];
    d.z = m[2] * a.x + m[5] * a.y + m[8] * a.z + m[11];
    return d;
}

// Primitive SDFs, src/sdfs/sdfs.f90:494-735
template <class R>
__device__ __forceinline__ R eval_prim_base(const DPrim<R>& pr, V3<R> pos) {
    const V3<R> p = xform(pr.m, pos);
    const R* q = pr.q;
    const R zero = 0, one = 1, half = (R)0.5;
    switch (pr.kind) {
        case SMCRT_SPHERE:
            return sqrt(p.x * p.x + p.y * p.y + p.z * p.z) - q[0];
        case SMCRT_BOX: {
            R dx = fabs(p.x) - q[0], dy = fabs(p.y) - q[1], dz = fabs(p.z) - q[2];
            R mx = fmax(dx, zero), my = fmax(dy, zero), mz = fmax(dz, zero);
            return sqrt(mx * mx + my * my + mz * mz) + fmin(fmax(dx, fmax(dy, dz)), zero);
        }
        case SMCRT_TORUS: {
            R tx = sqrt(p.x * p.x + zero * zero + p.z * p.z) - q[0];
            return sqrt(tx * tx + p.y * p.y + zero * zero) - q[1];
        }
        case SMCRT_CYLINDER: {
            V3<R> a{q[0], q[1], q[2]}, b{q[3], q[4], q[5]};
            V3<R> ba = b - a, pa = p - a;
            R baba = dot3(ba, ba), paba = dot3(pa, ba);
            R x = len3(pa * baba - ba * paba) - q[6] * baba;
            R y = fabs(paba - baba * half) - baba * half;
            R x2 = x * x, y2 = (y * y) * baba, d;
            if (fmax(x, y) < zero) {
                d = -fmin(x2, y2);
            } else {
                if (x > zero && y > zero) d = x2 + y2;
                else if (x > zero) d = x2;
                else if (y > zero) d = y2;
                else d = zero;
            }
            return fsign(sqrt(fabs(d)) / baba, d);
        }
        case SMCRT_TRIPRISM: {
            return fmax(fabs(p.z) - q[1], fmax(fabs(p.x) * (R)0.866025 + p.y * half, -p.y) - q[0] * half);
        }
        case SMCRT_SEGMENT:
        case SMCRT_CAPSULE: {
            V3<R> a{q[0], q[1], q[2]}, b{q[3], q[4], q[5]};
            V3<R> pa = p - a, ba = b - a;
            R h = clampr(dot3(pa, ba) / dot3(ba, ba), zero, one);
            R r = (pr.kind == SMCRT_SEGMENT) ? (R)0.1 : q[6];
            return len3(pa - ba * h) - r;
        }
        case SMCRT_CONE: {
            V3<R> a{q[0], q[1], q[2]}, b{q[3], q[4], q[5]};
            R ra = q[6], rb = q[7];
            R rba = rb - ra;
            R baba = dot3(b - a, b - a);
            R papa = dot3(p - a, p - a);
            R paba = dot3(p - a, b - a) / baba;
            R x = sqrt(fmax(papa - baba * paba * paba, zero));
            R cax = (paba < half) ? fmax(zero, x - ra) : fmax(zero, x - rb);
            R cay = fabs(paba - half) - half;
            R k = rba * rba + baba;
            R f = clampr((rba * (x - ra) + paba * baba) / k, zero, one);
            R cbx = x - ra - f * rba;
            R cby = paba - f;
            R s = (cbx < zero && cay < zero) ? -one : one;
            return s * sqrt(fmin(cax * cax + baba * cay * cay, cbx * cbx + baba * cby * cby));
        }
        case SMCRT_EGG: {
            V3<R> pin{fabs(p.x), p.y, p.z};
            R r = q[0] - q[1];
            R hin = q[2] + r;
            R l = (hin * hin - r * r) / ((R)2 * r);
            if (pin.y <= zero) return len3(pin) - q[0];
            if ((pin.y - hin) * l > pin.x * hin)
                return len3(V3<R>{pin.x, pin.y - hin, pin.z}) - ((q[0] + l) - sqrt(hin * hin + l * l));
            return len3(V3<R>{pin.x + l, pin.y, pin.z}) - (q[0] + l);
        }
        case SMCRT_PLANE:
            return p.x * q[0] + p.y * q[1] + p.z * q[2];
    }
    return zero;
}

// Modifiers (src/sdfs/sdfModifiers.f90:273-375): the point the wrapped SDF is
// evaluated at, and the value the modifier returns from the wrapped SDF's value.
template <class R>
__device__ __forceinline__ V3<R> mod_point(int kind, const R* q, V3<R> p) {
    const R zero = 0;
    switch (kind) {
        case SMCRT_MOD_REVOLUTION:  // (|(x, z)| - o, y, 0)
            return V3<R>{sqrt(p.x * p.x + p.z * p.z + zero * zero) - q[0], p.y, zero};
        case SMCRT_MOD_ELONGATE:  // max(|p| - size, 0)
            return V3<R>{fmax(fabs(p.x) - q[0], zero), fmax(fabs(p.y) - q[1], zero), fmax(fabs(p.z) - q[2], zero)};
        case SMCRT_MOD_TWIST: {  // rotation by k z about z
            R s, c;
            sincos_r(q[0] * p.z, &s, &c);
            return V3<R>{c * p.x - s * p.y, s * p.x + c * p.y, p.z};
        }
        case SMCRT_MOD_BEND: {  // rotation by k x about z
            R s, c;
            sincos_r(q[0] * p.x, &s, &c);
            return V3<R>{c * p.x - s * p.y, s * p.x + c * p.y, p.z};
        }
        default:  // onion, extrude: the wrapped SDF sees the point itself
            return p;
    }
}
template <class R>
__device__ __forceinline__ R mod_value(int kind, const R* q, R d, V3<R> p) {
    const R zero = 0;
    switch (kind) {
        case SMCRT_MOD_ONION:
            return fabs(d) - q[0];
        case SMCRT_MOD_EXTRUDE: {  // w = (d, |z| - h, 0)
            const R wy = fabs(p.z) - q[0];
            const R mx = fmax(d, zero), my = fmax(wy, zero);
            return fmin(fmax(d, wy), zero) + sqrt(mx * mx + my * my + zero * zero);
        }
        case SMCRT_MOD_ELONGATE: {
            const R qx = fabs(p.x) - q[0], qy = fabs(p.y) - q[1], qz = fabs(p.z) - q[2];
            return d + fmin(fmax(qx, fmax(qy, qz)), zero);
        }
        default:
            return d;
    }
}

// A primitive with its modifiers: points map outermost modifier first, values
// innermost first, as the nested evaluate calls of the reference do.  MODS =
// false compiles the primitive alone, for scenes without modifiers.
template <class R, bool MODS = true>
__device__ __forceinline__ R eval_prim(const DPrim<R>& pr, V3<R> pos) {
    if (!MODS || pr.nmods == 0) return eval_prim_base(pr, pos);
    const V3<R> p1 = pr.nmods == 2 ? mod_point(pr.mod[1], pr.mp[1], pos) : pos;
    const V3<R> p2 = mod_point(pr.mod[0], pr.mp[0], p1);
    R d = mod_value(pr.mod[0], pr.mp[0], eval_prim_base(pr, p2), p1);
    if (pr.nmods == 2) d = mod_value(pr.mod[1], pr.mp[1], d, pos);
    return d;
}

// eval_model (src/sdfs/sdf_base.f90:145-160), CSG ops src/sdfs/sdfModifiers.f90:412-475
// S: SceneT (parameter block) or SceneG (device memory).
template <class R, bool MODS = true, class S = SceneT<R>>
__device__ __forceinline__ R eval_region(const S& sc, int r, V3<R> pos) {
    const DRegion<R>& g = sc.region[r];
    R d = eval_prim<R, MODS>(sc.prim[g.first], pos);
    for (int i = 1; i < g.n; ++i) {
        R d2 = eval_prim<R, MODS>(sc.prim[g.first + i], pos);
        switch (g.op) {
            case SMCRT_OP_UNION: d = fmin(d, d2); break;
            case SMCRT_OP_SMOOTH_UNION: {
                R h = fmax(g.k - fabs(d - d2), (R)0) / g.k;
                d = fmin(d, d2) - h * h * h * g.k * ((R)1 / (R)6);
                break;
            }
            case SMCRT_OP_SUBTRACTION: d = fmax(-d, d2); break;
            case SMCRT_OP_INTERSECTION: d = fmax(d, d2); break;
        }
    }
    return d;
}

// calcNormal, src/sdfs/sdf_base.f90:165-189 (always double)
template <bool MODS = true, class S = SceneT<double>>
__device__ __forceinline__ V3<double> calc_normal(const S& sc, int r, V3<double> p, double h) {
    const V3<double> xyy{1, -1, -1}, yyx{-1, -1, 1}, yxy{-1, 1, -1}, xxx{1, 1, 1};
    V3<double> n = xyy * eval_region<double, MODS, S>(sc, r, p + xyy * h) +
                   yyx * eval_region<double, MODS, S>(sc, r, p + yyx * h) +
                   yxy * eval_region<double, MODS, S>(sc, r, p + yxy * h) +
                   xxx * eval_region<double, MODS, S>(sc, r, p + xxx * h);
    double t = len3(n);
    return V3<double>{n.x / t, n.y / t, n.z / t};
}

// fresnel / reflect / refract, src/surfaces.f90:42-120
template <class R>
__device__ __forceinline__ R fresnel(V3<R> I, V3<R> N, R n1, R n2) {
    R costt = fabs(dot3(I, N));
    R sintt = sqrt((R)1 - costt * costt);
    R sint2 = n1 / n2 * sintt;
    if (sint2 > (R)1) return (R)1;
    if (costt == (R)1) return (R)0;
    R cost2 = sqrt((R)1 - sint2 * sint2);
    R f1 = fabs((n1 * costt - n2 * cost2) / (n1 * costt + n2 * cost2));
    R f2 = fabs((n1 * cost2 - n2 * costt) / (n1 * cost2 + n2 * costt));
    return (R)0.5 * (f1 * f1 + f2 * f2);
}
template <class R>
__device__ __forceinline__ V3<R> reflect(V3<R> I, V3<R> N) {
    return I - (R)2 * dot3(N, I) * N;
}
template <class R>
__device__ __forceinline__ V3<R> refract(V3<R> I, V3<R> N, R eta) {
    V3<R> Nt = N;
    R c1 = dot3(Nt, I);
    if (c1 < (R)0) c1 = -c1;
    else Nt = (R)(-1) * N;
    R c2 = sqrt((R)1 - (eta * eta) * ((R)1 - c1 * c1));
    return eta * I + (eta * c1 - c2) * Nt;
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11).
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2,
                                                       uint32_t c3, uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

template <class R> struct U01;
template <> struct U01<float> {
    static constexpr int kWords = 1;
    __device__ __forceinline__ static float from(uint32_t a, uint32_t) { return (float)(a >> 9) * 0x1p-23f + 0x1p-24f; }
};
template <> struct U01<double> {
    static constexpr int kWords = 2;
    __device__ __forceinline__ static double from(uint32_t a, uint32_t b) {
        uint64_t m = ((uint64_t)a << 20) | (uint64_t)(b >> 12);
        return (double)m * 0x1p-52 + 0x1p-53;
    }
};

// One Philox block (out of line unless SMCRT_PHILOX_INLINE: one copy of the 10
// rounds per kernel, at the cost of a call per four draws).
#ifdef SMCRT_PHILOX_INLINE
static __device__ __forceinline__ uint4 philox_block(
#else
static __device__ __noinline__ uint4 philox_block(
#endif
    uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2,
                                                 uint32_t c3) {
    uint32_t o[4];
    philox4x32_10(k0, k1, c0, c1, c2, c3, o);
    return make_uint4(o[0], o[1], o[2], o[3]);
}

// Per-packet uniform stream: counter RNG keyed (seed, instance, packet id); in
// replay builds (INJ) an injected uniform stream instead.  The key words live in
// the caller's constant bank (seed, instance) and are passed at each refill.
template <class R, bool INJ = false>
struct Stream {
    uint32_t p0, p1, block;
    uint32_t b0, b1, b2, b3;  // unconsumed Philox words, consumed from b0 (register queue)
    int left;
    int ndraws;
    const double* inj;
    int ninj;
    int flags;
    unsigned long long seed;
    uint32_t inst;

    __device__ __forceinline__ void init(uint64_t seed_, uint32_t instance, uint64_t pid, const double* injected,
                                         int n) {
        seed = seed_;
        inst = instance;
        p0 = (uint32_t)pid;
        p1 = (uint32_t)(pid >> 32);
        block = 0;
        left = 0;
        ndraws = 0;
        inj = injected;
        ninj = n;
        flags = 0;
    }
    __device__ __forceinline__ R next() {
        if (INJ) {
            if (ndraws >= ninj) {
                flags |= STATUS_STREAM_EXHAUSTED;
                ++ndraws;
                return (R)0.5;
            }
            return (R)inj[ndraws++];
        }
        if (left < U01<R>::kWords) {
            const uint4 o = philox_block((uint32_t)seed, (uint32_t)(seed >> 32), block, inst, p0, p1);
            b0 = o.x;
            b1 = o.y;
            b2 = o.z;
            b3 = o.w;
            ++block;
            left = 4;
        }
        R u;
        if (U01<R>::kWords == 1) {
            u = U01<R>::from(b0, 0u);
            b0 = b1;
            b1 = b2;
            b2 = b3;
        } else {
            u = U01<R>::from(b0, b1);
            b0 = b2;
            b1 = b3;
        }
        left -= U01<R>::kWords;
        ++ndraws;
        return u;
    }
};

// scatter, src/photon.f90:713-779 (the bias test with p = 0 consumes one draw
// when g != 0).  FP64 uses the reference's formulas; FP32 evaluates the same
// angles in forms free of the 1 - cos^2 cancellations: 1 -+ cos(theta) come
// factored out of the HG inverse CDF, and sin/cos(phi) from sincospi, so the
// FP32 direction is accurate to a few ulps even for near-forward scatters.
__device__ __forceinline__ void hg_angles(float hgg, float g2, float u, float& cost, float& sint) {
    float omc, opc;  // 1 - cos(theta), 1 + cos(theta)
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
    sint = sqrtf(omc * opc);
}
__device__ __forceinline__ void hg_angles(double hgg, double g2, double u, double& cost, double& sint) {
    if (hgg == 0.0) {
        cost = 2.0 * u - 1.0;
    } else {
        const double temp = (1.0 - g2) / (1.0 - hgg + 2.0 * hgg * u);
        cost = (1.0 + g2 - temp * temp) / (2.0 * hgg);
    }
    sint = sqrt(1.0 - cost * cost);
}
__device__ __forceinline__ void phi_angles(float u, float& cosp, float& sinp) { sincospif(2.0f * u, &sinp, &cosp); }
__device__ __forceinline__ void phi_angles(double u, double& cosp, double& sinp) {
    cosp = cospi(2.0 * u);
    const double s = sqrt(1.0 - cosp * cosp);
    sinp = (u < 0.5) ? s : -s;  // phi = 2 pi u < pi  <=>  u < 1/2
}

// mu_out: the sampled cos(theta) (the HG variate, before the vertical-case sign
// rule), for the adjoint's d log p_HG / dg.
template <class R, class Rng>
__device__ __forceinline__ V3<R> hg_scatter(V3<R> d, R hgg, R g2, Rng& rng, R* mu_out = nullptr) {
    const R one = 1;
    R cost, sint;
    if (hgg == (R)0) {
        hg_angles(hgg, g2, rng.next(), cost, sint);
    } else {
        (void)rng.next();
        hg_angles(hgg, g2, rng.next(), cost, sint);
    }
    if (mu_out) *mu_out = cost;
    R cosp, sinp;
    phi_angles(rng.next(), cosp, sinp);
    bool vertical = (one - fabs(d.z) <= (R)1e-12);
    R temp = 0;
    if (!vertical) {
        temp = (sizeof(R) == 4) ? sqrt(d.x * d.x + d.y * d.y) : sqrt(one - d.z * d.z);
        if (temp == (R)0) vertical = true;
    }
    V3<R> o;
    if (vertical) {
        o.x = sint * cosp;
        o.y = sint * sinp;
        o.z = fsign(cost, d.z);
    } else {
        o.x = sint * (d.x * d.z * cosp - d.y * sinp) / temp + d.x * cost;
        o.y = sint * (d.y * d.z * cosp + d.x * sinp) / temp + d.y * cost;
        o.z = -one * sint * cosp * temp + d.z * cost;
    }
    return o;
}

// ---------------------------------------------------------------------------
// Grid and detectors.
template <class R>
struct GridT {
    int nx, ny, nz, pad;
    R xmax, ymax, zmax;
    R vx, vy, vz;       // voxel sizes 2*max/n
    R sx, sy, sz;       // n/(2*max) as written: n * p / (2 * max)
    double xmax_d, ymax_d, zmax_d;  // exact half sizes (grid-exit test on FP64 positions)
    double sx_d, sy_d, sz_d;        // n / (2 max) in FP64 (FP32 transport's cell index of an FP64 position)
    double vx_d, vy_d, vz_d;        // voxel sizes 2 max / n in FP64 (the walk's face positions)
};

struct DetT {
    int kind, layer, nb, pad;  // nb = bins per axis (nbins + 1)
    long long off;
    double pos[3], dir[3];
    double r1, r2, bw, bwy;
    double e1[3], e2[3], n[3], width, height;
};

template <class R>
struct SourceT {
    int kind, annulus_type;
    R pos[3], dir[3], p1[3], p2[3], p3[3];
    R radius, radius_hi, sin_beta, cos_beta, zstart;
    R rot[9];  // circular source rotation (rotationAlign), row-major M[i][j]
    int circ_swap;
};

// Launch parameters (one __grid_constant__ block in the constant bank).
template <class R>
struct Params {
    SceneT<R> sc;
    SceneT<double> sc64;  // boundary events
    // scenes beyond the parameter block (the BIG kernel instantiation): device tables
    SceneG<R> gsc;
    SceneG<double> gsc64;
    GridT<R> grid;
    SourceT<R> src;
    DetT det[kMaxDetectors];
    int ndet;
    int kernel;
    int end_early;
    int max_steps;
    R eps;
    R near_band;  // FP32 transport: sweeps closer than this to a surface are taken in FP64
    // nearest-region cache: allowed (every region 1-Lipschitz) and the rounding
    // margin of its test (FP32 transport: the FP32 sweeps' margin for both sweeps)
    int cache_ok;
    double cache_margin;
    // sort group of each action, one nibble per action (the round's list order)
    unsigned group_order;
    // shared-memory fluence privatisation (FP32 plain launches): a sub-box of
    // voxels (0-based origin, extents; priv_n cells, 0 = off) whose segments each
    // CTA sums in shared memory as 64-bit fixed point and adds to the grid once
    int priv_n;
    int priv_o[3], priv_d[3];
    double normal_h;
    unsigned long long seed;
    unsigned long long budget_ns;  // per-launch device time budget (0 = none)
    unsigned int instance;
    long long first;
    long long count;
    int sbins;    // detector bins counted in shared memory (0: global atomics)
    int tcopies;                     // fluence-grid copies the CTAs spread their adds over
    unsigned tmask;                  // tcopies - 1 (tcopies is a power of two)
    long long ncell;
    double* jtab[kMaxTallyCopies];   // the grid of each copy; jtab[0] is the output grid
    // batch launches: instance i has packets [bprefix[i], bprefix[i+1]) of the
    // launch, seed bseed[i], optics bopt[i], tally jtab[0] + i * ncell and
    // detector bins + i * nbins; per-instance packets/draws/scatters in bstats
    const InstOptics<R>* bopt;
    const long long* bprefix;
    const unsigned long long* bseed;
    unsigned long long* bstats;  // [ninst][3]
    int ninst;
    long long nbins;
    // adjoint launches: d loss / d (per-packet fluence) per voxel, d loss / d
    // (per-packet detector counts) per bin, the parameter group of each region
    // (255: none) and the output sums [3][ngroups] (d/d mua, d/d mus, d/d g)
    const float* adj_w;
    const double* adj_gbins;
    double* adj_out;
    int adj_ngroups;
    unsigned char adj_group[kMaxRegions];
    // second-moment runs (the VAR instantiation): each packet slot's voxel-score
    // table (kVarSlotBytes each: (voxel, score) pairs, the used list and its
    // count; slot-major over the persistent grid's CTAs) and the per-voxel sum of
    // squared per-packet scores
    unsigned char* var_tab;
    double* jmean2;
};

}  // namespace smcrt
