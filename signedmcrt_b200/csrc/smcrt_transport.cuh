// smcrt_transport.cuh -- the persistent, regenerating packet-transport kernel.
//
// One thread carries one packet at a time.  The loop body is ONE flight
// (tauint2) per lane: a lane whose packet died launches a fresh packet at the
// top of the next iteration (warp-aggregated work grab), so lanes do not idle
// at the end of a long-lived packet the way a per-packet loop does.
#pragma once

#include "smcrt_device.cuh"

namespace smcrt {

enum CounterIdx {
    C_PACKETS = 0,
    C_SDF,
    C_VOX,
    C_STEPS,
    C_SCAT,
    C_FRES,
    C_REFL,
    C_STEPCAP,
    C_ERR,
    C_DRAWS,
    C_NUM
};

struct Buffers {
    double* jmean;                 // FP64 fluence grid (column-major)
    double* bins;                  // detector bins
    unsigned long long* work;      // [0] next packet (relative to P.first)
    unsigned long long* counters;  // C_NUM
    double* moments;               // 24 (test kernel) + 1 (nscatt)
    int* status;                   // device status bitmask
    const double* uniforms;        // replay streams
    const long long* offsets;
    smcrt_packet_state* states;
};

struct Cnt {
    uint32_t sdf, vox, steps, scat, fres, refl;
};

template <class R>
struct Pk {
    V3<double> pos;  // FP64 position accumulator: FP32 steps below half an ulp of a
                     // coordinate would otherwise be lost (grazing approaches stall)
    V3<R> dir;
    R weight;
    int layer;  // 0-based region index
    int bounces;
    int nscatt;
    int flags;
    bool tflag;
};

template <class R>
__device__ __forceinline__ V3<R> cv(V3<double> p) {
    return V3<R>{(R)p.x, (R)p.y, (R)p.z};
}
template <class R>
__device__ __forceinline__ V3<double> advance(V3<double> p, R d, V3<R> dir) {
    return V3<double>{p.x + (double)(d * dir.x), p.y + (double)(d * dir.y), p.z + (double)(d * dir.z)};
}

// Integer-stepping voxel walk over one sphere-tracing segment (the tally of
// update_grids, src/inttau2.f90:213-292): same start cell (floor index,
// :433-435) and grid-exit rule, with crossings advancing the index by +-1.
template <class R>
__device__ __forceinline__ void voxel_walk(const GridT<R>& g, double* __restrict__ jm, V3<R> pos, V3<R> dir, R L,
                                           bool& tflag, Cnt& c) {
    const V3<R> o{pos.x + g.xmax, pos.y + g.ymax, pos.z + g.zmax};
    int ci = (int)floor((R)g.nx * o.x / ((R)2 * g.xmax)) + 1;
    int cj = (int)floor((R)g.ny * o.y / ((R)2 * g.ymax)) + 1;
    int ck = (int)floor((R)g.nz * o.z / ((R)2 * g.zmax)) + 1;
    if (ci < 1 || ci > g.nx || cj < 1 || cj > g.ny || ck < 1 || ck > g.nz) {
        tflag = true;
        return;
    }
    const R big = (R)1e30;
    const int sx = dir.x > (R)0 ? 1 : (dir.x < (R)0 ? -1 : 0);
    const int sy = dir.y > (R)0 ? 1 : (dir.y < (R)0 ? -1 : 0);
    const int sz = dir.z > (R)0 ? 1 : (dir.z < (R)0 ? -1 : 0);
    R tx = big, ty = big, tz = big;
    if (sx) tx = fmax(((R)(sx > 0 ? ci : ci - 1) * g.vx - o.x) / dir.x, (R)0);
    if (sy) ty = fmax(((R)(sy > 0 ? cj : cj - 1) * g.vy - o.y) / dir.y, (R)0);
    if (sz) tz = fmax(((R)(sz > 0 ? ck : ck - 1) * g.vz - o.z) / dir.z, (R)0);
    long long idx = (long long)(ci - 1) + (long long)g.nx * ((long long)(cj - 1) + (long long)g.ny * (ck - 1));
    const long long stride_y = g.nx, stride_z = (long long)g.nx * g.ny;
    R d = 0;
    for (;;) {
        const R tm = fmin(tx, fmin(ty, tz));
        if (tm > L) {
            atomicAdd(jm + idx, (double)(L - d));
            ++c.vox;
            break;
        }
        atomicAdd(jm + idx, (double)(tm - d));
        ++c.vox;
        d = tm;
        if (tm == tx) {
            ci += sx;
            if (ci < 1 || ci > g.nx) { tflag = true; break; }
            idx += sx;
            tx = fmax(((R)(sx > 0 ? ci : ci - 1) * g.vx - o.x) / dir.x, (R)0);
        } else if (tm == ty) {
            cj += sy;
            if (cj < 1 || cj > g.ny) { tflag = true; break; }
            idx += sy * stride_y;
            ty = fmax(((R)(sy > 0 ? cj : cj - 1) * g.vy - o.y) / dir.y, (R)0);
        } else {
            ck += sz;
            if (ck < 1 || ck > g.nz) { tflag = true; break; }
            idx += sz * stride_z;
            tz = fmax(((R)(sz > 0 ? ck : ck - 1) * g.vz - o.z) / dir.z, (R)0);
        }
    }
}

// tauint2, src/inttau2.f90:15-210
template <class R, class Rng>
__device__ __forceinline__ void tauint2(const Params<R>& P, double* __restrict__ jm, Pk<R>& pk, Rng& rng, Cnt& c) {
    const SceneT<R>& sc = P.sc;
    const int N = sc.nregions;
    const R eps = P.eps;
    const R inf = (R)INFINITY;
    V3<double> pos = pk.pos, oldpos = pos;
    V3<R> dir = pk.dir;
    R tau = -log(rng.next());
    R taurun = 0;
    for (;;) {
        R dsdf = inf;
        {
            const V3<R> pf = cv<R>(pos);
            for (int i = 0; i < N; ++i) dsdf = fmin(dsdf, fabs(eval_region(sc, i, pf)));
        }
        c.sdf += N;
        // The reference kills here when d < eps and stops tracing when d <= eps
        // (inttau2.f90:58,63); a packet left at d == eps (reachable on the FP32
        // coordinate grid) is treated as on the surface, like a reflected packet.
        if (dsdf <= eps) {
            pk.tflag = true;
            break;
        }
        int steps = 0;
        while (dsdf > eps) {
            ++c.steps;
            const R kap = sc.region[pk.layer].kappa;
            const R tsdf = dsdf * kap;
            bool last = false;
            if (taurun + tsdf <= tau) {
                taurun = taurun + tsdf;
            } else {
                dsdf = (tau - taurun) / kap;
                taurun = tau;
                last = true;
            }
            voxel_walk(P.grid, jm, cv<R>(pos), dir, dsdf, pk.tflag, c);
            pos = advance(pos, dsdf, dir);
            if (last) break;
            R mn = inf, mna = inf;
            const V3<R> pf = cv<R>(pos);
            for (int i = 0; i < N; ++i) {
                const R d = eval_region(sc, i, pf);
                mn = fmin(mn, d);
                mna = fmin(mna, fabs(d));
            }
            c.sdf += N;
            dsdf = mna;
            if (mn >= (R)0) {
                pk.tflag = true;
                break;
            }
            if (++steps >= P.max_steps) {
                pk.tflag = true;
                pk.flags |= STATUS_STEP_CAP;
                break;
            }
        }
        if (taurun >= tau || pk.tflag) break;

        // Surface crossing (:104-184).  min|dstmp| equals the last sweep's dsdf
        // (same position), so that sweep is counted but not repeated.
        c.sdf += N;
        const R dstep = dsdf + (R)2 * eps;
        oldpos = pos;
        pos = advance(pos, dstep, dir);
        const int L = pk.layer;
        int nl = -1;
        R d0 = 0, dsL = 0, dsN = 0;
        const V3<R> pf = cv<R>(pos);
        for (int i = 0; i < N; ++i) {
            const R d = eval_region(sc, i, pf);
            if (i == 0) d0 = d;
            if (i == L) dsL = d;
            if (nl < 0 && d < (R)0) {
                nl = i;
                dsN = d;
            }
        }
        c.sdf += N;
        if (nl < 0) {
            nl = 0;
            dsN = d0;
        }
        const R n1 = sc.region[L].nidx, n2 = sc.region[nl].nidx;
        if (n1 != n2) {
            int which;
            if (dsL < (R)0 && dsN < (R)0) {
                which = (fabs(dsL) <= fabs(dsN)) ? L : nl;
            } else {
                const V3<R> of = cv<R>(oldpos);
                const R tL = eval_region(sc, L, of), tN = eval_region(sc, nl, of);
                if (tL < (R)0 && tN < (R)0) {
                    which = (tL >= tN) ? L : nl;
                } else if (dsL >= (R)0 && dsN < (R)0) {
                    // An SDF value of exactly 0 counts as outside, like the `ds(i) < 0`
                    // membership test; the reference's `error stop` branch (:155-156)
                    // is then reached only by NaN.
                    which = (L == 0) ? L : nl;  // oldlayer = packet%layer, then "== 1" test (:150-162)
                } else if (dsL >= (R)0 && dsN >= (R)0) {
                    pk.tflag = true;
                    break;
                } else {
                    pk.tflag = true;  // "This should not be reached!" (:156)
                    pk.flags |= STATUS_ERROR_STATE;
                    break;
                }
            }
            // Boundary event in FP64: calcNormal + reflect_refract (surfaces.f90:14-40).
            ++c.fres;
            c.sdf += 4;
            const V3<double> Nn =
                calc_normal(P.sc64, which, pos, P.normal_h);
            V3<double> I{(double)dir.x, (double)dir.y, (double)dir.z};
            const double m1 = P.sc64.region[L].nidx, m2 = P.sc64.region[nl].nidx;
            const double Rf = fresnel(I, Nn, m1, m2);
            const double u = (double)rng.next();
            const bool refl = u <= Rf;
            I = refl ? reflect(I, Nn) : refract(I, Nn, m1 / m2);
            dir = V3<R>{(R)I.x, (R)I.y, (R)I.z};
            pk.weight = pk.weight * (R)Rf;
            tau = -log(rng.next());
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
    pk.pos = pos;
    pk.dir = dir;
    if (fabs(pos.x) > P.grid.xmax_d || fabs(pos.y) > P.grid.ymax_d || fabs(pos.z) > P.grid.zmax_d) pk.tflag = true;
}

// Emitters, src/photon.f90
template <class R, class Rng>
__device__ __forceinline__ void emit(const Params<R>& P, Pk<R>& pk, Rng& rng) {
    const SourceT<R>& s = P.src;
    pk.tflag = false;
    pk.bounces = 0;
    pk.weight = (R)1;
    pk.layer = 0;
    pk.flags = 0;
    pk.nscatt = 0;
    const R TWOPI = (R)(2.0 * kPI);
    switch (s.kind) {
        case SMCRT_SRC_POINT: {  // :290-338
            pk.pos = V3<double>{(double)s.pos[0], (double)s.pos[1], (double)s.pos[2]};
            const R phi = rng.next() * TWOPI;
            R sp, cp;
            sincos_r(phi, &sp, &cp);
            const R u2 = rng.next();
            const R cost = (R)2 * u2 - (R)1;
            // FP32: sin(theta) = 2 sqrt(u (1 - u)), free of the 1 - cos^2 cancellation
            const R sint = (sizeof(R) == 4) ? (R)2 * sqrt(u2 * ((R)1 - u2)) : sqrt((R)1 - cost * cost);
            pk.dir = V3<R>{sint * cp, sint * sp, cost};
            break;
        }
        case SMCRT_SRC_UNIFORM: {  // :397-461
            pk.dir = V3<R>{s.dir[0], s.dir[1], s.dir[2]};
            const R rx = rng.next(), ry = rng.next();
            pk.pos.x = (double)(s.p1[0] + rx * s.p2[0] + ry * s.p3[0]);
            pk.pos.y = (double)(s.p1[1] + rx * s.p2[1] + ry * s.p3[1]);
            pk.pos.z = (double)(s.p1[2] + rx * s.p2[2] + ry * s.p3[2]);
            break;
        }
        case SMCRT_SRC_CIRCULAR: {  // :214-287
            pk.dir = V3<R>{s.dir[0], s.dir[1], s.dir[2]};
            const R r = s.radius * sqrt(rng.next());
            const R th = rng.next() * TWOPI;
            R sth, cth;
            sincos_r(th, &sth, &cth);
            const V3<R> p = s.circ_swap ? V3<R>{r * cth, r * sth, (R)0} : V3<R>{(R)0, r * cth, r * sth};
            const R* M = s.rot;
            pk.pos.x = (double)(M[0] * p.x + M[3] * p.y + M[6] * p.z - s.pos[0]);
            pk.pos.y = (double)(M[1] * p.x + M[4] * p.y + M[7] * p.z - s.pos[1]);
            pk.pos.z = (double)(M[2] * p.x + M[5] * p.y + M[8] * p.z - s.pos[2]);
            break;
        }
        case SMCRT_SRC_ANNULUS: {  // :645-711
            R radius;
            if (s.annulus_type == SMCRT_ANNULUS_TOPHAT) {
                radius = s.radius + (s.radius_hi - s.radius) * sqrt(rng.next());
            } else {  // rang, random_mod.f90:105-133
                const R mid = (s.radius_hi - s.radius) / (R)2;
                R x, y, ss;
                int guard = 0;
                do {
                    x = (R)(-1) + rng.next() * (R)2;
                    y = (R)(-1) + rng.next() * (R)2;
                    ss = y * y + x * x;
                } while (ss >= (R)1 && ++guard < 1000);
                radius = mid + (R)0.04 * (x * sqrt((R)(-2) * log(ss) / ss));
            }
            const R phi = TWOPI * rng.next();
            R sp, cp;
            sincos_r(phi, &sp, &cp);
            pk.pos = V3<double>{(double)(radius * cp), (double)(radius * sp), (double)s.zstart};
            pk.dir = V3<R>{s.sin_beta * cp, s.sin_beta * sp, -s.cos_beta};
            break;
        }
        case SMCRT_SRC_FOCUS: {  // :340-394
            const R x = -P.grid.xmax + rng.next() * ((R)2 * P.grid.xmax);
            const R y = -P.grid.ymax + rng.next() * ((R)2 * P.grid.ymax);
            pk.pos = V3<double>{(double)x, (double)y, (double)s.zstart};
            const R dist = len3(V3<R>{x, y, s.zstart});
            V3<R> d{(R)(-1) * x / dist, (R)(-1) * y / dist, (R)(-1) * s.zstart / dist};
            const R l = len3(d);
            d = V3<R>{d.x / l, d.y / l, d.z / l};
            const R phi = atan2(d.y, d.x);
            R sp, cp;
            sincos_r(phi, &sp, &cp);
            const R sint = sqrt((R)1 - d.z * d.z);
            pk.dir = V3<R>{sint * cp, sint * sp, d.z};
            break;
        }
        default:  // pencil, :464-505
            pk.pos = V3<double>{(double)s.pos[0], (double)s.pos[1], (double)s.pos[2]};
            pk.dir = V3<R>{s.dir[0], s.dir[1], s.dir[2]};
    }
}

// Launch layer (src/kernelsMod.f90:275-280): innermost containing region.
template <class R>
__device__ __forceinline__ int launch_layer(const SceneT<R>& sc, V3<R> p) {
    int best = 0;
    R bestv = (R)INFINITY;
    for (int i = 0; i < sc.nregions; ++i) {
        R d = eval_region(sc, i, p);
        if (d > (R)0) d = (R)(-999.0);
        if (fabs(d) < bestv) {
            bestv = fabs(d);
            best = i;
        }
    }
    return best;
}

// Detector hit test + bin (record_hit_1D/2D, detector_base.f90:106-162).
__device__ __forceinline__ long long detector_bin(const DetT& D, const double p[3], const double l[3], double value,
                                                  int layer1) {
    if (D.layer != layer1) return -1;
    if (D.kind == SMCRT_DET_ANNULUS) {  // detectors.f90:169-184
        const double dx = p[0] - D.pos[0], dy = p[1] - D.pos[1], dz = p[2] - D.pos[2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        if (!(r >= D.r1 && r <= D.r2)) return -1;
    } else if (D.kind == SMCRT_DET_CIRCLE) {  // detectors.f90:110-127, geometryMod.f90:217-270
        const double denom = D.dir[0] * l[0] + D.dir[1] * l[1] + D.dir[2] * l[2];
        if (!(denom > 1e-6)) return -1;
        const double t =
            ((D.pos[0] - p[0]) * D.dir[0] + (D.pos[1] - p[1]) * D.dir[1] + (D.pos[2] - p[2]) * D.dir[2]) / denom;
        if (!(t >= 0.0)) return -1;
        const double q0 = p[0] + l[0] * t - D.pos[0], q1 = p[1] + l[1] * t - D.pos[1], q2 = p[2] + l[2] * t - D.pos[2];
        if (!(sqrt(q0 * q0 + q1 * q1 + q2 * q2) <= D.r1)) return -1;
        if (t > 5e-3) return -1;
    } else {  // camera, detectors.f90:231-253
        const double num = (D.pos[0] - p[0]) * D.n[0] + (D.pos[1] - p[1]) * D.n[1] + (D.pos[2] - p[2]) * D.n[2];
        const double den = l[0] * D.n[0] + l[1] * D.n[1] + l[2] * D.n[2];
        const double t = num / den;
        if (!(t >= 0.0)) return -1;
        const double v0 = p[0] + t * l[0] - D.pos[0], v1 = p[1] + t * l[1] - D.pos[1], v2 = p[2] + t * l[2] - D.pos[2];
        const double pr1 = (v0 * D.e1[0] + v1 * D.e1[1] + v2 * D.e1[2]) / D.width;
        const double pr2 = (v0 * D.e2[0] + v1 * D.e2[1] + v2 * D.e2[2]) / D.height;
        if (!((pr1 < D.width && pr1 > 0.0) && (pr2 < D.height && pr2 > 0.0))) return -1;
        const double x = p[2] + D.pos[0], y = p[1] + D.pos[1];
        long long ix = min((long long)(x / D.bw) + 1, (long long)D.nb);
        long long iy = min((long long)(y / D.bwy) + 1, (long long)D.nb);
        if (ix < 1) ix = D.nb;
        if (iy < 1) iy = D.nb;
        return D.off + (ix - 1) + (long long)D.nb * (iy - 1);
    }
    long long idx = min(llround(value / D.bw) + 1, (long long)D.nb);
    if (idx < 1) idx = 1;
    return D.off + idx - 1;
}

template <class R>
__device__ __forceinline__ void record_detectors(const Params<R>& P, const Buffers& B, const Pk<R>& pk) {
    if (P.ndet == 0 || P.kernel == SMCRT_KERNEL_TEST) return;
    const double p[3] = {(double)pk.pos.x, (double)pk.pos.y, (double)pk.pos.z};
    const double l[3] = {(double)pk.dir.x, (double)pk.dir.y, (double)pk.dir.z};
    const double value = (P.kernel == SMCRT_KERNEL_WEIGHT) ? (double)pk.weight
                                                           : sqrt(pk.pos.x * pk.pos.x + pk.pos.y * pk.pos.y);
    for (int d = 0; d < P.ndet; ++d) {
        const long long b = detector_bin(P.det[d], p, l, value, pk.layer + 1);
        if (b >= 0) atomicAdd(B.bins + b, 1.0);
    }
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The persistent kernel.  KERNEL: smcrt_kernel_kind.  REPLAY: injected streams.
template <class R, int KERNEL, bool REPLAY>
__global__ void __launch_bounds__(256, 2) transport_kernel(const __grid_constant__ Params<R> P, const Buffers B) {
    __shared__ unsigned long long s_cnt[C_NUM];
    __shared__ double s_mom[25];
    if (threadIdx.x < C_NUM) s_cnt[threadIdx.x] = 0ull;
    if (threadIdx.x < 25) s_mom[threadIdx.x] = 0.0;
    __syncthreads();

    Pk<R> pk;
    pk.tflag = true;
    Stream<R, REPLAY> rng;
    Cnt c = {0, 0, 0, 0, 0, 0};
    bool need_new = true;  // the lane holds no packet
    long long pid = 0;
    unsigned iter = 0;
    const unsigned long long t0 = P.budget_ns ? global_ns() : 0ull;
    for (;;) {
        // device-side time budget: past it, stop between flights and flag ABORTED
        if (P.budget_ns && ((++iter) & 63u) == 0u && global_ns() - t0 > P.budget_ns) {
            atomicOr(B.status, STATUS_ABORTED);
            break;
        }
        // ---- prepare the next flight: a new packet (emit) or an interaction (scatter)
        bool fly = true;
        if (need_new) {
            const unsigned m = __activemask();
            const unsigned lane = lane_id();
            const int leader = __ffs(m) - 1;
            const unsigned rank = __popc(m & ((1u << lane) - 1u));
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(B.work, (unsigned long long)__popc(m));
            base = __shfl_sync(m, base, leader);
            pid = (long long)(base + rank);
            if (pid >= P.count) break;
            const long long gpid = P.first + pid;
            if (REPLAY) {
                const long long o0 = B.offsets[pid], o1 = B.offsets[pid + 1];
                rng.init(P.seed, P.instance, (uint64_t)gpid, B.uniforms + o0, (int)(o1 - o0));
            } else {
                rng.init(P.seed, P.instance, (uint64_t)gpid, nullptr, 0);
            }
            emit(P, pk, rng);
            pk.layer = launch_layer(P.sc, cv<R>(pk.pos));
            c.sdf += P.sc.nregions;
        } else if (KERNEL == SMCRT_KERNEL_WEIGHT) {  // weight_scatter, kernelsMod.f90:99-134
            const DRegion<R>& rg = P.sc.region[pk.layer];
            const R wa = pk.weight * ((R)1 - rg.albedo);
            pk.weight = pk.weight - wa;
            const R ox = (R)pk.pos.x + P.grid.xmax, oy = (R)pk.pos.y + P.grid.ymax, oz = (R)pk.pos.z + P.grid.zmax;
            const int ci = (int)floor((R)P.grid.nx * ox / ((R)2 * P.grid.xmax)) + 1;
            const int cj = (int)floor((R)P.grid.ny * oy / ((R)2 * P.grid.ymax)) + 1;
            const int ck = (int)floor((R)P.grid.nz * oz / ((R)2 * P.grid.zmax)) + 1;
            if (ci < 1 || ci > P.grid.nx || cj < 1 || cj > P.grid.ny || ck < 1 || ck > P.grid.nz) {
                pk.tflag = true;
                fly = false;
            } else {
                atomicAdd(B.jmean + (long long)(ci - 1) +
                              (long long)P.grid.nx * ((long long)(cj - 1) + (long long)P.grid.ny * (ck - 1)),
                          (double)wa);
                pk.dir = hg_scatter(pk.dir, rg.hgg, rg.g2, rng);
                ++c.scat;
                if (pk.weight < (R)0.01) {
                    if (rng.next() < (R)0.1) pk.weight = pk.weight / (R)0.1;
                    else {
                        pk.tflag = true;
                        fly = false;
                    }
                }
            }
        } else {  // pathlength_scatter :285-300 / test_kernel :408-436
            const R ran = rng.next();
            const DRegion<R>& rg = P.sc.region[pk.layer];
            if (ran < rg.albedo) {
                pk.dir = hg_scatter(pk.dir, rg.hgg, rg.g2, rng);
                ++c.scat;
                pk.nscatt += 1;
                if (KERNEL == SMCRT_KERNEL_TEST) {
                    const int sidx = pk.nscatt;
                    if (sidx >= 1 && sidx <= 4) {
                        const double px = pk.pos.x, py = pk.pos.y, pz = pk.pos.z;
                        atomicAdd(&s_mom[(sidx - 1) * 3 + 0], px);
                        atomicAdd(&s_mom[(sidx - 1) * 3 + 1], py);
                        atomicAdd(&s_mom[(sidx - 1) * 3 + 2], pz);
                        atomicAdd(&s_mom[12 + (sidx - 1) * 3 + 0], px * px);
                        atomicAdd(&s_mom[12 + (sidx - 1) * 3 + 1], py * py);
                        atomicAdd(&s_mom[12 + (sidx - 1) * 3 + 2], pz * pz);
                    } else if (P.end_early) {
                        pk.tflag = true;  // the reference still calls tauint2 once more (:428-435)
                    }
                }
            } else {
                pk.tflag = true;
                fly = false;
            }
        }
        // ---- one flight, from a single call site so the warp enters it together
        if (fly) tauint2(P, B.jmean, pk, rng, c);
        need_new = pk.tflag;
        if (need_new) {
            record_detectors(P, B, pk);
            atomicAdd(&s_cnt[C_PACKETS], 1ull);
            atomicAdd(&s_cnt[C_SDF], (unsigned long long)c.sdf);
            atomicAdd(&s_cnt[C_VOX], (unsigned long long)c.vox);
            atomicAdd(&s_cnt[C_STEPS], (unsigned long long)c.steps);
            atomicAdd(&s_cnt[C_SCAT], (unsigned long long)c.scat);
            atomicAdd(&s_cnt[C_FRES], (unsigned long long)c.fres);
            atomicAdd(&s_cnt[C_REFL], (unsigned long long)c.refl);
            atomicAdd(&s_cnt[C_DRAWS], (unsigned long long)rng.ndraws);
            if (pk.flags & STATUS_STEP_CAP) atomicAdd(&s_cnt[C_STEPCAP], 1ull);
            if (pk.flags & STATUS_ERROR_STATE) atomicAdd(&s_cnt[C_ERR], 1ull);
            const int fl = pk.flags | rng.flags;
            if (fl) atomicOr(B.status, fl);
            if (KERNEL != SMCRT_KERNEL_WEIGHT) atomicAdd(&s_mom[24], (double)pk.nscatt);
            if (REPLAY) {
                smcrt_packet_state& st = B.states[pid];
                st.pos[0] = pk.pos.x; st.pos[1] = pk.pos.y; st.pos[2] = pk.pos.z;
                st.dir[0] = pk.dir.x; st.dir[1] = pk.dir.y; st.dir[2] = pk.dir.z;
                st.weight = pk.weight;
                st.layer = pk.layer + 1;
                st.nscatt = pk.nscatt;
                st.ndraws = rng.ndraws;
                st.flags = fl;
            }
            c = Cnt{0, 0, 0, 0, 0, 0};
        }
    }
    __syncthreads();
    if (threadIdx.x < C_NUM && s_cnt[threadIdx.x]) atomicAdd(B.counters + threadIdx.x, s_cnt[threadIdx.x]);
    if (threadIdx.x < 25 && s_mom[threadIdx.x] != 0.0) atomicAdd(B.moments + threadIdx.x, s_mom[threadIdx.x]);
}

}  // namespace smcrt
