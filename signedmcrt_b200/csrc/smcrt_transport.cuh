// smcrt_transport.cuh -- the persistent, regenerating packet-transport kernel.
//
// One thread carries one packet at a time.  tauint2's nested loops (flights,
// sphere-tracing steps, voxel walk) are flattened into a per-lane state
// machine: every iteration of the persistent loop performs ONE short action --
// launch a packet, sweep the SDFs, walk one voxel segment, handle a boundary,
// interact, or retire a packet -- so lanes whose loops would run for different
// trip counts stay busy instead of waiting at the end of the longest loop.
// The arithmetic of each action is the same, operation for operation, as the
// nested form in tauint2 (src/inttau2.f90:15-441).
#pragma once

#include "smcrt_device.cuh"

namespace smcrt {

// Threads per CTA of the transport kernel (one CTA per SM).
#ifndef SMCRT_BLOCK
#define SMCRT_BLOCK 640
#endif
constexpr int kBlock = SMCRT_BLOCK;

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
    C_VAROVF,  // second-moment contributions squared alone (score table crowded)
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
    uint32_t sdf, vox, steps, scat, fres, refl, varovf;
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
    int inst;  // batch instance (0 outside batches)
    int phase;        // adjoint: 0 = first pass (sum C), 1 = second pass (gradient terms)
    // adjoint: the packet's loss contribution C, and the part of it made so far, in
    // FP64: their difference (the contribution still to come) cancels along
    // histories of hundreds of segments
    double ctot, cpre;
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

// Detector hits at packet death (kernelsMod.f90:302-306).  Each hit adds one
// count; with privatized bins the count goes to the CTA's shared-memory copy.
template <class R>
__device__ __forceinline__ void record_detectors(const Params<R>& P, double* bins, unsigned* sbins, double px,
                                                 double py, double pz, double lx, double ly, double lz,
                                                 double weight, int layer1) {
    const double p[3] = {px, py, pz};
    const double l[3] = {lx, ly, lz};
    const double value = (P.kernel == SMCRT_KERNEL_WEIGHT) ? weight : sqrt(px * px + py * py);
    for (int d = 0; d < P.ndet; ++d) {
        const long long b = detector_bin(P.det[d], p, l, value, layer1);
        if (b >= 0) {
            if (P.sbins) atomicAdd(sbins + b, 1u);
            else atomicAdd(bins + b, 1.0);
        }
    }
}

// The fluence grid this CTA adds into: copy (CTA index mod tcopies).  The CTA
// index is read at each use (volatile) rather than kept in a register across the
// transport loop, and the copy's address comes from the parameter bank.
template <class R, bool BATCH>
__device__ __forceinline__ double* tally_grid(const Params<R>& P, int inst) {
    if (BATCH) return P.jtab[0] + (long long)inst * P.ncell;  // one grid per instance, no copies
    unsigned b;
    asm volatile("mov.u32 %0, %%ctaid.x;" : "=r"(b));
    return P.jtab[b & P.tmask];
}

// Fixed-point unit of the privatised sub-box: 2^-32 cm (a CTA's sum in a voxel stays
// far below 2^31 cm; a segment's rounding, 1e-10 cm, is below its FP32 rounding).
constexpr double kPrivScale = 4294967296.0;

// One voxel segment into the fluence tally: the CTA's shared sub-box when the cell
// lies in it, else the FP64 grid.
template <class R, bool BATCH>
__device__ __forceinline__ void tally_add(const Params<R>& P, int inst, int ci, int cj, int ck, int idx, R len,
                                          unsigned long long* priv) {
    if (!BATCH && P.priv_n) {
        const unsigned li = (unsigned)(ci - 1 - P.priv_o[0]), lj = (unsigned)(cj - 1 - P.priv_o[1]),
                       lk = (unsigned)(ck - 1 - P.priv_o[2]);
        if (li < (unsigned)P.priv_d[0] && lj < (unsigned)P.priv_d[1] && lk < (unsigned)P.priv_d[2]) {
            atomicAdd(priv + li + P.priv_d[0] * (lj + P.priv_d[1] * lk),
                      (unsigned long long)__double2ll_rn((double)len * kPrivScale));
            return;
        }
    }
    atomicAdd(tally_grid<R, BATCH>(P, inst) + idx, (double)len);
}

// The scene a kernel instantiation reads: the parameter block's, or (BIG) the
// device-memory tables of a scene too large for it.
template <bool BIG, class R>
__device__ __forceinline__ const auto& scene_of(const Params<R>& P) {
    if constexpr (BIG) return P.gsc;
    else return P.sc;
}
template <bool BIG, class R>
__device__ __forceinline__ const auto& scene64_of(const Params<R>& P) {
    if constexpr (BIG) return P.gsc64;
    else return P.sc64;
}

// Region optics: the scene's, or the batch instance's.
template <class R, bool BATCH, bool BIG>
__device__ __forceinline__ R opt_kappa(const Params<R>& P, int inst, int r) {
    return BATCH ? P.bopt[inst].kappa[r] : scene_of<BIG>(P).region[r].kappa;
}
template <class R, bool BATCH, bool BIG>
__device__ __forceinline__ R opt_nidx(const Params<R>& P, int inst, int r) {
    return BATCH ? P.bopt[inst].nidx[r] : scene_of<BIG>(P).region[r].nidx;
}
template <class R, bool BATCH, bool BIG>
__device__ __forceinline__ double opt_nidx64(const Params<R>& P, int inst, int r) {
    return BATCH ? P.bopt[inst].nidx64[r] : scene64_of<BIG>(P).region[r].nidx;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The persistent kernel.  KERNEL: smcrt_kernel_kind.  REPLAY: injected streams.
#ifndef SMCRT_MIN_BLOCKS
#define SMCRT_MIN_BLOCKS 1
#endif
#ifndef SMCRT_WALK_SEGMENTS
#define SMCRT_WALK_SEGMENTS 4
#endif
// The nearest-region cache (1: built in; 0: every sweep evaluates every region)
#ifndef SMCRT_NEAREST_CACHE
#define SMCRT_NEAREST_CACHE 1
#endif
constexpr bool kNearestCache = SMCRT_NEAREST_CACHE != 0;
// ... also for the sweep at a flight's start (after a scatter)
#ifndef SMCRT_CACHE_TOP
#define SMCRT_CACHE_TOP 1
#endif
constexpr bool kCacheTop = SMCRT_CACHE_TOP != 0;

// Per-lane actions of the flattened transport loop.
// A_PRECISE (FP32 transport): a sweep within the FP64 band of a surface, or resolving a
// crossing, deferred to the next round and done in FP64 with the other such packets.
enum Act : int { A_NEW = 0, A_SWEEP, A_WALK, A_CROSS, A_INTERACT, A_DEATH, A_DONE, A_PRECISE };
// What the next sweep is for.
enum SweepMode : int { S_LAUNCH = 0, S_TOP, S_STEP, S_CROSS };

// FP32 bounds of a length: rounded down (a clearance) or up (a distance moved).
__device__ __forceinline__ float float_rd(float x) { return x; }
__device__ __forceinline__ float float_rd(double x) { return __double2float_rd(x); }
__device__ __forceinline__ float float_ru(float x) { return x; }
__device__ __forceinline__ float float_ru(double x) { return __double2float_ru(x); }

template <class R>
struct Flight {
    R tau, taurun, dsdf;  // optical depth to spend / spent; current step length
    int steps;            // sphere-tracing steps of the current inner loop
    int mode;             // SweepMode of the next sweep
    bool last;            // the current step spends the remaining optical depth
    // Nearest-region cache (see nearest_cached): valid flag, the nearest region
    // at the last full sweep, whether another region contained the point there,
    // and the clearance -- a lower bound on every other region's |d| less the
    // path travelled since that sweep.
    bool cache, negx;
    int nk;
    float clear;
    float dkup;  // an upper bound on region k's |d| at the current position
    // FP32 transport: the last sweep was taken in FP64 and found the surface
    // within half of near_band, so the next step's sweep is within near_band too
    // (a move of min|d| changes every |d| by at most that) and goes straight to FP64
    bool near;
    // Integer voxel walk of the current step (update_grids, inttau2.f90:213-292):
    // parametric distance to the next x/y/z face, distance walked, and the cell.
    // During a crossing the same storage holds the position before the step.
    union {
        struct {
            R tx, ty, tz, td;
            int ci, cj, ck;
        } w;
        struct {
            V3<double> oldpos;
            int which, nl;
        } x;
    };
};

// A move of f.dsdf: off the clearance, onto the bound on |d_k|.
template <class R>
__device__ __forceinline__ void cache_move(Flight<R>& f) {
    f.clear = __fsub_rd(f.clear, float_ru(f.dsdf));
    f.dkup = __fadd_ru(f.dkup, float_ru(f.dsdf));
}

// All regions at one point (the sweep of tauint2, inttau2.f90:51-55,86-96,104-108):
// signed minimum, minimum |d|, region 0's value, region L's value, the first
// region containing the point (and its value), and the launch layer
// (kernelsMod.f90:275-280: innermost containing region).  For the nearest-region
// cache also: the region of the minimum |d| (k), a lower bound on every other
// region's |d| (m2), and whether another region contains the point (negx).
template <class T>
struct SweepOut {
    T mn, mna, d0, dsL, dsN;
    int nl, lay;
    T m2;
    int k;
    bool negx;
};
//
// Device-memory scenes (SceneG) skip regions by their bounding spheres.  A
// region with a bound (a single primitive whose SDF is the exact Euclidean
// distance -- sphere, box, capsule, segment, cylinder, torus -- under a rigid
// transform) is skipped when the point lies farther from the sphere than the
// smallest |d| found so far plus a rounding margin: its value is then positive
// and larger than that minimum, so it changes none of the outputs (the signed
// minimum only matters through its sign, and the region contains no point
// there).  Regions 0 and L are always evaluated (their values are outputs).
//
// only >= 0: the nearest-region cache holds, so only region `only` is evaluated
// (mn, mna and k then describe that region alone; the caller supplies the sign
// of the other regions).  Lanes of one warp that sweep in full and lanes that
// sweep one region share this loop, so a warp evaluates each region at most once.
template <class T, bool MODS = true, class S = SceneT<T>>
__device__ __forceinline__ SweepOut<T> sweep_regions(const S& sc, V3<T> p, int L, int only = -1) {
    SweepOut<T> o{(T)INFINITY, (T)INFINITY, (T)0, (T)0, (T)0, -1, 0, (T)INFINITY, 0, false};
    T inner = (T)INFINITY;
    int nneg = 0;
    bool kneg = false;
    // the warp's range of regions: all of them when a lane sweeps in full, else
    // from the lowest to the highest cached region of its lanes
    const unsigned am = __activemask();
    const int lo = __reduce_min_sync(am, (unsigned)(only >= 0 ? only : 0));
    const int hi = __reduce_max_sync(am, (unsigned)(only >= 0 ? only : sc.nregions - 1));
    for (int i = lo; i <= hi; ++i) {
        if (only >= 0 && i != only) continue;
        if constexpr (!std::is_same<S, SceneT<T>>::value) {
            const T br = sc.bound[4 * i + 3];
            if (br >= (T)0 && i != 0 && i != L && o.mna < (T)INFINITY) {
                const T dx = p.x - sc.bound[4 * i], dy = p.y - sc.bound[4 * i + 1], dz = p.z - sc.bound[4 * i + 2];
                const T r2 = dx * dx + dy * dy + dz * dz;
                const T lim = o.mna + sc.cull_margin + br;
                if (r2 > lim * lim) {
                    // outside its bounding sphere: |d| >= distance to the sphere
                    o.m2 = fmin(o.m2, sqrt(r2) - br);
                    continue;
                }
            }
        }
        const T d = eval_region<T, MODS, S>(sc, i, p);
        const T a = fabs(d);
        o.mn = fmin(o.mn, d);
        if (a < o.mna) {
            o.m2 = o.mna;
            o.mna = a;
            o.k = i;
            kneg = d < (T)0;
        } else {
            o.m2 = fmin(o.m2, a);
        }
        nneg += d < (T)0;
        if (i == 0) o.d0 = d;
        if (i == L) o.dsL = d;
        if (o.nl < 0 && d < (T)0) {
            o.nl = i;
            o.dsN = d;
        }
        const T ai = (d > (T)0) ? (T)999.0 : a;
        if (ai < inner) {
            inner = ai;
            o.lay = i;
        }
    }
    o.negx = nneg - (int)kneg > 0;
    return o;
}

// Single-region evaluations of the crossing path.  They stay inline: an
// out-of-line function would receive the parameter block by reference and read
// it through generic loads instead of the constant bank.
template <class R, bool MODS, class S>
__device__ __forceinline__ R eval_region_cold(const S& sc, int r, V3<R> p) {
    return eval_region<R, MODS, S>(sc, r, p);
}
template <bool MODS, class S>
__device__ __forceinline__ V3<double> calc_normal_cold(const S& sc, int r, V3<double> p, double h) {
    return calc_normal<MODS, S>(sc, r, p, h);
}

// 1-based cell of a point given in FP64 grid coordinates (position + half size),
// update_voxels' index formula (src/inttau2.f90:433-435): FP64 transport divides
// as the reference does; FP32 transport multiplies by the FP64 n / (2 max) (an
// FP64 division costs tens of instructions, and FP32 transport's walk is
// statistically, not bitwise, the reference's).
template <class R>
__device__ __forceinline__ void cell_of(const GridT<R>& g, double ox, double oy, double oz, int& ci, int& cj,
                                        int& ck) {
    if (sizeof(R) == 8) {
        ci = (int)floor((double)g.nx * ox / (2.0 * g.xmax_d)) + 1;
        cj = (int)floor((double)g.ny * oy / (2.0 * g.ymax_d)) + 1;
        ck = (int)floor((double)g.nz * oz / (2.0 * g.zmax_d)) + 1;
    } else {
        ci = (int)floor(ox * g.sx_d) + 1;
        cj = (int)floor(oy * g.sy_d) + 1;
        ck = (int)floor(oz * g.sz_d) + 1;
    }
}

// Starts a sphere-tracing step of length f.dsdf (body of the while loop at
// inttau2.f90:63-83): optical depth bookkeeping, then the voxel-walk setup.
// Returns A_WALK, or -1 when the step starts outside the grid (no tally).
template <class R, bool BATCH, bool BIG>
__device__ __forceinline__ int start_step(const Params<R>& P, const Pk<R>& pk, Flight<R>& f, Cnt& c, bool& tflag) {
    ++c.steps;
    const R kap = opt_kappa<R, BATCH, BIG>(P, pk.inst, pk.layer);
    const R tsdf = f.dsdf * kap;
    f.last = false;
    if (f.taurun + tsdf <= f.tau) {
        f.taurun = f.taurun + tsdf;
    } else {
        f.dsdf = (f.tau - f.taurun) / kap;
        f.taurun = f.tau;
        f.last = true;
    }
    const GridT<R>& g = P.grid;
    // the start cell and the distances to its faces from the FP64 position: an FP32
    // coordinate within an ulp of a grid face can round onto it, and a packet that
    // stopped eps inside the grid's outer face would then start outside the grid
    const double ox = pk.pos.x + g.xmax_d, oy = pk.pos.y + g.ymax_d, oz = pk.pos.z + g.zmax_d;
    cell_of<R>(g, ox, oy, oz, f.w.ci, f.w.cj, f.w.ck);
    if (f.w.ci < 1 || f.w.ci > g.nx || f.w.cj < 1 || f.w.cj > g.ny || f.w.ck < 1 || f.w.ck > g.nz) {
        tflag = true;  // outside the grid: no tally for this step
        return -1;
    }
    // distance to the first face on each axis, then one face spacing per crossing
    // (Amanatides & Woo): no division per segment
    // (the faces at FP64 multiples of the FP64 voxel size: the FP32 voxel size
    // times a cell index misplaces the grid's outer face by tens of eps)
    const R big = (R)1e30;
    const V3<R>& d = pk.dir;
    const double vx = g.vx_d, vy = g.vy_d, vz = g.vz_d;
    f.w.tx = d.x > (R)0 ? fmax((R)((double)f.w.ci * vx - ox) / d.x, (R)0)
           : d.x < (R)0 ? fmax((R)((double)(f.w.ci - 1) * vx - ox) / d.x, (R)0) : big;
    f.w.ty = d.y > (R)0 ? fmax((R)((double)f.w.cj * vy - oy) / d.y, (R)0)
           : d.y < (R)0 ? fmax((R)((double)(f.w.cj - 1) * vy - oy) / d.y, (R)0) : big;
    f.w.tz = d.z > (R)0 ? fmax((R)((double)f.w.ck * vz - oz) / d.z, (R)0)
           : d.z < (R)0 ? fmax((R)((double)(f.w.ck - 1) * vz - oz) / d.z, (R)0) : big;
    f.w.td = 0;
    return A_WALK;
}

// Distance between successive faces of one axis along the direction.
template <class R>
__device__ __forceinline__ R face_spacing(R v, R dcomp) {
    return v / fabs(dcomp);
}

// ---------------------------------------------------------------------------
// History-based second moment of the fluence tally.  The variance of a voxel's
// tally needs each packet's own total score there (all of its segments in that
// voxel added first), squared.  Every packet slot owns a table in device memory:
// kVarEntries (voxel, score) pairs (open addressing, linear probing), the list of
// the entries in use (16-bit positions, in the order they were taken) and their
// count, stored complemented so that the all-ones fill of a fresh table reads as
// zero.  A segment adds into its voxel's entry; the retiring packet adds each used
// entry's squared score to jmean2 and empties it, so a retire costs the voxels the
// packet visited, not the table size.  Probing runs until the voxel or a free
// entry turns up; only a packet that visits more than kVarEntries distinct voxels
// finds neither: that segment is squared on its own and counted (C_VAROVF), and the
// estimate then lacks the cross terms of that segment.  (A 1-packet census of the
// test scenes gives means of 80-240 distinct voxels and tails below 2000.)
constexpr int kVarLog2 = 12;
constexpr int kVarEntries = 1 << kVarLog2;
constexpr unsigned kVarEmpty = 0xFFFFFFFFu;
// one slot's table: the pairs, the used list, the count (16-byte multiple)
constexpr size_t kVarSlotBytes = (size_t)kVarEntries * 8 + (size_t)kVarEntries * 2 + 16;
static_assert(kVarSlotBytes % 16 == 0, "slot tables keep 16-byte alignment");

struct VarTab {
    uint2* e;
    unsigned short* used;
    unsigned* ncount;  // complement of the number of used entries
};

__device__ __forceinline__ VarTab var_table(unsigned char* base) {
    VarTab t;
    t.e = reinterpret_cast<uint2*>(base);
    t.used = reinterpret_cast<unsigned short*>(base + (size_t)kVarEntries * 8);
    t.ncount = reinterpret_cast<unsigned*>(base + (size_t)kVarEntries * 10);
    return t;
}

__device__ __forceinline__ void var_add(unsigned char* vt, double* jmean2, int idx, float v, Cnt& c) {
    const VarTab t = var_table(vt);
    unsigned h = ((unsigned)idx * 2654435761u) >> (32 - kVarLog2);
    for (int k = 0; k < kVarEntries; ++k) {
        const uint2 e = t.e[h];
        if (e.x == (unsigned)idx) {
            t.e[h].y = __float_as_uint(__uint_as_float(e.y) + v);
            return;
        }
        if (e.x == kVarEmpty) {
            t.e[h] = make_uint2((unsigned)idx, __float_as_uint(v));
            const unsigned n = ~*t.ncount;
            t.used[n] = (unsigned short)h;
            *t.ncount = ~(n + 1u);
            return;
        }
        h = (h + 1u) & (unsigned)(kVarEntries - 1);
    }
    atomicAdd(jmean2 + idx, (double)v * (double)v);
    ++c.varovf;
}

__device__ __forceinline__ void var_flush(unsigned char* vt, double* jmean2) {
    const VarTab t = var_table(vt);
    const unsigned n = ~*t.ncount;
    for (unsigned k = 0; k < n; ++k) {
        const unsigned h = t.used[k];
        const uint2 e = t.e[h];
        const double sc = (double)__uint_as_float(e.y);
        atomicAdd(jmean2 + e.x, sc * sc);
        t.e[h] = make_uint2(kVarEmpty, 0u);
    }
    *t.ncount = kVarEmpty;
}

// One voxel segment of the current step; returns true when the step's walk is over.
// (ADJ: the adjoint's track terms instead of the fluence tally; on leaving the
// grid the rest of the step, untallied, still counts for survival.)
template <class R, bool BATCH, bool ADJ, bool VAR>
__device__ __forceinline__ bool walk_segment(const Params<R>& P, Pk<R>& pk, Flight<R>& f, Cnt& c, float* acc,
                                             unsigned char* vt, unsigned long long* priv) {
    const GridT<R>& g = P.grid;
    const V3<R>& d = pk.dir;
    const R tm = fmin(f.w.tx, fmin(f.w.ty, f.w.tz));
    const int idx = (f.w.ci - 1) + g.nx * ((f.w.cj - 1) + g.ny * (f.w.ck - 1));
    ++c.vox;
    if (tm > f.dsdf) {
        if (ADJ) adj_track(P, pk, acc, (float)(f.dsdf - f.w.td), P.adj_w[idx]);
        else tally_add<R, BATCH>(P, pk.inst, f.w.ci, f.w.cj, f.w.ck, idx, f.dsdf - f.w.td, priv);
        if (VAR) var_add(vt, P.jmean2, idx, (float)(f.dsdf - f.w.td), c);
        return true;
    }
    if (ADJ) adj_track(P, pk, acc, (float)(tm - f.w.td), P.adj_w[idx]);
    else tally_add<R, BATCH>(P, pk.inst, f.w.ci, f.w.cj, f.w.ck, idx, tm - f.w.td, priv);
    if (VAR) var_add(vt, P.jmean2, idx, (float)(tm - f.w.td), c);
    f.w.td = tm;
    bool out = false;
    if (tm == f.w.tx) {
        f.w.ci += d.x > (R)0 ? 1 : -1;
        out = f.w.ci < 1 || f.w.ci > g.nx;
        f.w.tx = tm + face_spacing(g.vx, d.x);
    } else if (tm == f.w.ty) {
        f.w.cj += d.y > (R)0 ? 1 : -1;
        out = f.w.cj < 1 || f.w.cj > g.ny;
        f.w.ty = tm + face_spacing(g.vy, d.y);
    } else {
        f.w.ck += d.z > (R)0 ? 1 : -1;
        out = f.w.ck < 1 || f.w.ck > g.nz;
        f.w.tz = tm + face_spacing(g.vz, d.z);
    }
    if (out) {
        pk.tflag = true;
        if (ADJ) adj_track(P, pk, acc, (float)(f.dsdf - tm), 0.0f);
        return true;
    }
    return false;
}

// The end of a flight (inttau2.f90:188-209): grid-exit test, then interact or retire.
template <class R>
__device__ __forceinline__ int end_flight(const Params<R>& P, Pk<R>& pk) {
    if (fabs(pk.pos.x) > P.grid.xmax_d || fabs(pk.pos.y) > P.grid.ymax_d || fabs(pk.pos.z) > P.grid.zmax_d)
        pk.tflag = true;
    return pk.tflag ? A_DEATH : A_INTERACT;
}

// ---------------------------------------------------------------------------
// Adjoint (pathlength kernel).  For a loss L = sum_v w_v phi_v + sum_b h_b D_b
// over per-packet fluence phi and detector counts D, dL/dtheta = E[f x d log p /
// dtheta] (score function / perturbation Monte Carlo), where f is the packet's
// contribution and p its path density: per unit path length in region r the
// survival exp(-(mus_r + mua_r) l), per scatter mus_r p_HG(cos; g_r), per
// absorption mua_r (the collision density kappa times the albedo test).  By
// causality each score term only pairs with the contributions made after it, so
// each packet is traced twice from its regenerated stream: pass 1 sums its total
// contribution C, pass 2 adds (d log p_e / d theta) x (C - contributions so far)
// at every event e.  A packet carries two numbers instead of one score per
// parameter.  Terms go to per-thread accumulators acc[k][group][thread], k = 0
// d/d mua, 1 d/d mus, 2 d/d g, for the region's parameter group.
__device__ __forceinline__ void adj_add(float* acc, int k, int grp, float v) {
    acc[(k * kMaxAdjGroups + grp) * kBlock + threadIdx.x] += v;
}

// Path length `len` in the packet's region, over which the fluence weight is w
// (0 where nothing is tallied): survival term and contribution.
template <class R>
__device__ __forceinline__ void adj_track(const Params<R>& P, Pk<R>& pk, float* acc, float len, float w) {
    if (pk.phase == 0) {
        pk.ctot += (double)(w * len);
        return;
    }
    const int grp = P.adj_group[pk.layer];
    if (grp < P.adj_ngroups) {
        // integral over the length of -(contributions after each point); the same
        // for mua and mus (d kappa / d mua = d kappa / d mus = 1)
        const float v = len * (float)(pk.ctot - pk.cpre) - 0.5f * w * len * len;
        adj_add(acc, 0, grp, -v);
        adj_add(acc, 1, grp, -v);
    }
    pk.cpre += (double)(w * len);
}

// A scatter in the packet's region with HG variate mu (second pass).
template <class R>
__device__ __forceinline__ void adj_scatter(const Params<R>& P, const Pk<R>& pk, float* acc, R mu) {
    const int grp = P.adj_group[pk.layer];
    if (grp >= P.adj_ngroups) return;
    const DRegion<R>& rg = P.sc.region[pk.layer];
    const float F = (float)(pk.ctot - pk.cpre);
    if ((float)rg.mua < 1e-9f) {  // albedo 1 (init_mono): the interaction density is kappa
        adj_add(acc, 0, grp, F / (float)rg.kappa);
        adj_add(acc, 1, grp, F / (float)rg.kappa);
    } else {
        adj_add(acc, 1, grp, F / (float)rg.mus);
    }
    // d log p_HG(mu; g) / dg, p_HG = (1 - g^2) / (2 (1 + g^2 - 2 g mu)^1.5)
    const float g = (float)rg.hgg, m = (float)mu;
    const float den = (1.0f - g) * (1.0f - g) + 2.0f * g * (1.0f - m);  // 1 + g^2 - 2 g mu
    adj_add(acc, 2, grp, F * (-2.0f * g / (1.0f - g * g) - 3.0f * (g - m) / den));
}

// An absorption in the packet's region (second pass).
template <class R>
__device__ __forceinline__ void adj_absorb(const Params<R>& P, const Pk<R>& pk, float* acc) {
    const int grp = P.adj_group[pk.layer];
    if (grp >= P.adj_ngroups) return;
    adj_add(acc, 0, grp, (float)(pk.ctot - pk.cpre) / (float)P.sc.region[pk.layer].mua);
}

// Detector part of a retiring packet's contribution: sum of h_b over its bins.
template <class R>
__device__ __forceinline__ float adj_detector_term(const Params<R>& P, const Pk<R>& pk) {
    if (P.ndet == 0 || !P.adj_gbins) return 0.0f;
    const double p[3] = {pk.pos.x, pk.pos.y, pk.pos.z};
    const double l[3] = {(double)pk.dir.x, (double)pk.dir.y, (double)pk.dir.z};
    const double value = sqrt(pk.pos.x * pk.pos.x + pk.pos.y * pk.pos.y);
    double sum = 0.0;
    for (int d = 0; d < P.ndet; ++d) {
        const long long b = detector_bin(P.det[d], p, l, value, pk.layer + 1);
        if (b >= 0) sum += P.adj_gbins[b];
    }
    return (float)sum;
}

template <class R, class Rng>
__device__ __forceinline__ void start_flight(Flight<R>& f, Rng& rng) {
    f.tau = -log(rng.next());  // inttau2.f90:46
    f.taurun = 0;
}

// Moves through a step that starts outside the grid (no walk), then continues.
template <class R, bool BATCH, bool ADJ, bool BIG>
__device__ __forceinline__ int step_or_skip(const Params<R>& P, Pk<R>& pk, Flight<R>& f, Cnt& c, float* acc) {
    int a = start_step<R, BATCH, BIG>(P, pk, f, c, pk.tflag);
    if (a < 0) {
        if (ADJ) adj_track(P, pk, acc, (float)f.dsdf, 0.0f);  // a step outside the grid
        pk.pos = advance(pk.pos, f.dsdf, pk.dir);
        cache_move(f);
        if (f.last) return end_flight(P, pk);
        f.mode = S_STEP;
        return A_SWEEP;
    }
    return a;
}

// One pass of the transport state machine for one packet: the actions in a
// fixed order -- retire, launch, interact, sweep, cross -- then at most
// SMCRT_WALK_SEGMENTS voxel segments.  A packet can pass through several
// actions in one pass (retire -> launch -> sweep -> walk, interact -> sweep ->
// walk, sweep -> cross).  `c` counts this thread's events since its last flush.
template <class R, int KERNEL, bool REPLAY, bool BATCH, bool ADJ, bool MODS, bool BIG, bool VAR>
__device__ __forceinline__ void transport_pass(const Params<R>& P, const Buffers& B, Pk<R>& pk, Flight<R>& f,
                                               Stream<R, REPLAY>& rng, Cnt& c, int& act, unsigned long long* s_cnt,
                                               double* s_mom, unsigned* s_bins, float* acc, unsigned char* vt,
                                               unsigned long long* priv) {
    const auto& sc = scene_of<BIG>(P);
    const auto& sc64 = scene64_of<BIG>(P);
    using S = std::decay_t<decltype(sc)>;
    using S64 = std::decay_t<decltype(sc64)>;
    const int N = sc.nregions;
    const R eps = P.eps;
    // ---- adjoint: the end of a packet's first pass -- add its detector term to C
    // and trace the same packet again from its regenerated stream
    if (ADJ && act == A_DEATH && pk.phase == 0) {
        pk.ctot += (double)adj_detector_term(P, pk);
        rng.init(rng.seed, rng.inst, ((uint64_t)rng.p1 << 32) | rng.p0, nullptr, 0);
        emit(P, pk, rng);
        start_flight(f, rng);
        f.mode = S_LAUNCH;
        pk.phase = 1;
        pk.cpre = 0.0;
        act = A_SWEEP;
    }
    // ---- retire a finished packet: detectors (kernelsMod.f90:302-306), counters
    if (act == A_DEATH) {
        if (VAR) var_flush(vt, P.jmean2);  // the packet's squared voxel scores
        if (!ADJ && P.ndet > 0 && KERNEL != SMCRT_KERNEL_TEST)
            record_detectors(P, BATCH ? B.bins + (long long)pk.inst * P.nbins : B.bins, s_bins, pk.pos.x, pk.pos.y,
                             pk.pos.z, (double)pk.dir.x, (double)pk.dir.y,
                             (double)pk.dir.z, (double)pk.weight, pk.layer + 1);
        // per-packet totals, summed over the retiring lanes first: one shared
        // atomic per warp (a shared-memory FP64 add is a compare-and-swap loop)
        const unsigned m = __activemask();
        const unsigned draws = __reduce_add_sync(m, (unsigned)rng.ndraws);
        const unsigned ns = KERNEL != SMCRT_KERNEL_WEIGHT ? __reduce_add_sync(m, (unsigned)pk.nscatt) : 0u;
        if (lane_id() == (unsigned)(__ffs(m) - 1)) {
            atomicAdd(&s_cnt[C_PACKETS], (unsigned long long)__popc(m));
            atomicAdd(&s_cnt[C_DRAWS], (unsigned long long)draws);
            if (KERNEL != SMCRT_KERNEL_WEIGHT) atomicAdd(&s_mom[24], (double)ns);
        }
        if (pk.flags & STATUS_STEP_CAP) atomicAdd(&s_cnt[C_STEPCAP], 1ull);
        if (pk.flags & STATUS_ERROR_STATE) atomicAdd(&s_cnt[C_ERR], 1ull);
        const int fl = pk.flags | rng.flags;
        if (fl) atomicOr(B.status, fl);
        if (BATCH) {
            unsigned long long* bs = P.bstats + 3ll * pk.inst;
            atomicAdd(bs + 0, 1ull);
            atomicAdd(bs + 1, (unsigned long long)rng.ndraws);
            atomicAdd(bs + 2, (unsigned long long)pk.nscatt);
        }
        // this thread's event counts stay in registers until the kernel ends;
        // flushed early only long before they could wrap
        if ((c.sdf | c.vox | c.steps) > (1u << 30)) {
            atomicAdd(&s_cnt[C_SDF], (unsigned long long)c.sdf);
            atomicAdd(&s_cnt[C_VOX], (unsigned long long)c.vox);
            atomicAdd(&s_cnt[C_STEPS], (unsigned long long)c.steps);
            atomicAdd(&s_cnt[C_SCAT], (unsigned long long)c.scat);
            atomicAdd(&s_cnt[C_FRES], (unsigned long long)c.fres);
            atomicAdd(&s_cnt[C_REFL], (unsigned long long)c.refl);
            atomicAdd(&s_cnt[C_VAROVF], (unsigned long long)c.varovf);
            c = Cnt{0, 0, 0, 0, 0, 0, 0};
        }
        if (REPLAY) {
            smcrt_packet_state& st = B.states[(long long)(((uint64_t)rng.p1 << 32) | rng.p0) - P.first];
            st.pos[0] = pk.pos.x; st.pos[1] = pk.pos.y; st.pos[2] = pk.pos.z;
            st.dir[0] = pk.dir.x; st.dir[1] = pk.dir.y; st.dir[2] = pk.dir.z;
            st.weight = pk.weight;
            st.layer = pk.layer + 1;
            st.nscatt = pk.nscatt;
            st.ndraws = rng.ndraws;
            st.flags = fl;
        }
        act = A_NEW;
    }
    // ---- take the next packet id (warp-aggregated) and emit it
    if (act == A_NEW) {
        const unsigned m = __activemask();
        const unsigned lane = lane_id();
        const int leader = __ffs(m) - 1;
        const unsigned rank = __popc(m & ((1u << lane) - 1u));
        unsigned long long base = 0;
        if ((int)lane == leader) base = atomicAdd(B.work, (unsigned long long)__popc(m));
        base = __shfl_sync(m, base, leader);
        const long long pid = (long long)(base + rank);
        const long long total = BATCH ? P.bprefix[P.ninst] : P.count;
        if (pid >= total) {
            act = A_DONE;
        } else if (BATCH) {
            // the instance holding launch packet `pid`: last i with bprefix[i] <= pid
            int lo = 0, hi = P.ninst - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (P.bprefix[mid] <= pid) lo = mid;
                else hi = mid - 1;
            }
            pk.inst = lo;
            rng.init(P.bseed[lo], P.instance, (uint64_t)(pid - P.bprefix[lo]), nullptr, 0);
            emit(P, pk, rng);
            start_flight(f, rng);
            f.mode = S_LAUNCH;
            act = A_SWEEP;
        } else {
            const long long gpid = P.first + pid;
            if (REPLAY) {
                const long long o0 = B.offsets[pid], o1 = B.offsets[pid + 1];
                rng.init(P.seed, P.instance, (uint64_t)gpid, B.uniforms + o0, (int)(o1 - o0));
            } else {
                rng.init(P.seed, P.instance, (uint64_t)gpid, nullptr, 0);
            }
            if (ADJ) {
                pk.phase = 0;
                pk.ctot = 0.0;
                pk.cpre = 0.0;
            }
            emit(P, pk, rng);
            start_flight(f, rng);
            f.mode = S_LAUNCH;
            act = A_SWEEP;
        }
    }
    if (act == A_DONE) return;
    // ---- between flights (kernelsMod.f90:285-300 / 99-134 / 408-436)
    if (act == A_INTERACT) {
        const DRegion<R>& rg = sc.region[pk.layer];
        const R albedo = BATCH ? P.bopt[pk.inst].albedo[pk.layer] : rg.albedo;
        const R hgg = BATCH ? P.bopt[pk.inst].hgg[pk.layer] : rg.hgg;
        const R g2 = BATCH ? P.bopt[pk.inst].g2[pk.layer] : rg.g2;
        act = A_SWEEP;
        if (KERNEL == SMCRT_KERNEL_WEIGHT) {
            const R wa = pk.weight * ((R)1 - albedo);
            pk.weight = pk.weight - wa;
            // the interaction's voxel from the FP64 position (see start_step)
            const double ox = pk.pos.x + P.grid.xmax_d, oy = pk.pos.y + P.grid.ymax_d, oz = pk.pos.z + P.grid.zmax_d;
            int ci, cj, ck;
            cell_of<R>(P.grid, ox, oy, oz, ci, cj, ck);
            if (ci < 1 || ci > P.grid.nx || cj < 1 || cj > P.grid.ny || ck < 1 || ck > P.grid.nz) {
                pk.tflag = true;
                act = A_DEATH;
            } else {
                const int cell = (ci - 1) + P.grid.nx * ((cj - 1) + P.grid.ny * (ck - 1));
                atomicAdd(tally_grid<R, BATCH>(P, pk.inst) + cell, (double)wa);
                if (VAR) var_add(vt, P.jmean2, cell, (float)wa, c);
                pk.dir = hg_scatter(pk.dir, hgg, g2, rng);
                ++c.scat;
                if (pk.weight < (R)0.01) {  // THRESHOLD, CHANCE (constants.f90:28-30)
                    if (rng.next() < (R)0.1) pk.weight = pk.weight / (R)0.1;
                    else {
                        pk.tflag = true;
                        act = A_DEATH;
                    }
                }
            }
        } else {
            const R ran = rng.next();
            if (ran < albedo) {
                R mu = 0;
                pk.dir = hg_scatter(pk.dir, hgg, g2, rng, ADJ ? &mu : nullptr);
                if (ADJ && pk.phase) adj_scatter(P, pk, acc, mu);
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
                if (ADJ && pk.phase) adj_absorb(P, pk, acc);
                pk.tflag = true;
                act = A_DEATH;
            }
        }
        if (act == A_SWEEP) {
            start_flight(f, rng);
            f.mode = S_TOP;
        }
    }
    // ---- evaluate every region at the current position (the one inlined sweep)
    // Within near_band of a surface (16 FP32 ulps of the scene size, where FP32
    // coordinate rounding could move a distance across eps), or resolving a
    // crossing, FP32 transport takes the decisions (surface reached, crossing step,
    // new region, the kill at a flight's start) on the FP64 position with the FP64
    // scene, against the reference's eps: FP32 coordinates near 1 cm are only good
    // to ~1e-7 cm, ten times eps, and that noise changed how many refracted packets
    // the eps rule kills (-0.8% fluence).  Such sweeps are deferred as A_PRECISE so
    // that they run together, not one lane per warp.
    //
    // Nearest-region cache.  A full sweep records its nearest region k, a lower
    // bound m2 on every other region's |d|, and whether another region contains
    // the point; every move subtracts its length from the bound (regions are
    // 1-Lipschitz: exact distances under rigid transforms, checked on the host).
    // While |d_k| plus a rounding margin stays below that clearance, no other
    // region can be nearer or have changed sign, so region k alone gives the
    // sweep's outputs that a tracing step uses (min |d| and the sign of the
    // signed minimum) -- the same values as the full sweep.  Boundary events
    // (crossing sweeps, launches) always sweep in full; the counters still count
    // the reference's evaluations of every region.
    if (act == A_SWEEP || act == A_PRECISE) {
        const int L = pk.layer;
        SweepOut<R> sw{};
        bool precise = false, defer = false;
        // the cache holds for a tracing step or a flight start when the bound on
        // |d_k| plus the margin stays below the clearance
        const bool cached = kNearestCache && !ADJ && f.cache && (f.mode == S_STEP || (kCacheTop && f.mode == S_TOP)) &&
                            (double)f.dkup + P.cache_margin < (double)f.clear;
        const int only = cached ? f.nk : -1;
        // FP64 at once: the FP64 group, or a tracing step right after an FP64 sweep
        // that found the surface within half of near_band (f.near)
        bool want64 = sizeof(R) == 4 && (act == A_PRECISE || (f.near && f.mode == S_STEP));
        if (!want64) {
            sw = sweep_regions<R, MODS, S>(sc, cv<R>(pk.pos), L, only);
            defer = sizeof(R) == 4 && (sw.mna <= P.near_band || f.mode == S_CROSS);
            // a lane on the cache has one region to evaluate in FP64: it does so
            // now instead of waiting a round for the FP64 group (same values)
            if (defer && cached) {
                defer = false;
                want64 = true;
            }
        }
        if (want64) {
            const SweepOut<double> s64 = sweep_regions<double, MODS, S64>(sc64, pk.pos, L, only);
            sw = SweepOut<R>{(R)s64.mn, (R)s64.mna, (R)s64.d0, (R)s64.dsL, (R)s64.dsN, s64.nl, s64.lay,
                             (R)s64.m2, s64.k, s64.negx};
            precise = true;
        }
        if (cached) {
            // another region containing the point keeps the signed minimum negative
            if (f.negx && sw.mn >= (R)0) sw.mn = (R)-1;
        } else {
            f.cache = kNearestCache && !ADJ && P.cache_ok && f.mode != S_CROSS;
            f.nk = sw.k;
            f.negx = sw.negx;
            f.clear = float_rd(sw.m2);
        }
        f.dkup = float_ru(sw.mna);  // |d_k| here: the minimum found
        if (defer) {
            f.near = false;
            act = A_PRECISE;
        } else {
            act = A_SWEEP;
            const R mn = sw.mn, mna = sw.mna, d0 = sw.d0, dsL = sw.dsL;
            R dsN = sw.dsN;
            int nl = sw.nl;
            const int lay = sw.lay;
            c.sdf += N;
            f.dsdf = mna;
            const int mode = f.mode;
            f.near = sizeof(R) == 4 && precise && mode != S_CROSS && (R)2 * mna <= P.near_band;
            if (mode == S_LAUNCH || mode == S_TOP) {
                // top of tauint2's outer loop (:51-61).  At launch the same sweep also
                // gives the layer (the reference evaluates the same point twice).
                if (mode == S_LAUNCH) {
                    pk.layer = lay;
                    c.sdf += N;
                }
                f.steps = 0;
                // d == eps (reachable on the FP32 coordinate grid) counts as on the
                // surface, like the reflected packets the reference kills here
                if (mna <= eps) {
                    pk.tflag = true;
                    act = end_flight(P, pk);
                } else {
                    act = step_or_skip<R, BATCH, ADJ, BIG>(P, pk, f, c, acc);
                }
            } else if (mode == S_STEP) {
                if (mn >= (R)0) {  // outside every region (:92-96)
                    pk.tflag = true;
                    act = end_flight(P, pk);
                } else if (++f.steps >= P.max_steps) {
                    pk.tflag = true;
                    pk.flags |= STATUS_STEP_CAP;
                    act = end_flight(P, pk);
                } else if (mna > eps) {
                    act = step_or_skip<R, BATCH, ADJ, BIG>(P, pk, f, c, acc);
                } else if (f.taurun >= f.tau || pk.tflag) {
                    act = end_flight(P, pk);  // (:99-102)
                } else {
                    // surface reached: count the reference's dstmp sweep (values of this
                    // one, :104-108) and take the crossing step of min|d| + 2 eps
                    c.sdf += N;
                    f.x.oldpos = pk.pos;
                    pk.pos = advance(pk.pos, mna + (R)2 * eps, pk.dir);
                    f.mode = S_CROSS;
                    // sweep again at the new position, next round (FP32: in FP64)
                    act = sizeof(R) == 4 ? A_PRECISE : A_SWEEP + 100;
                }
            } else {  // S_CROSS: sweep at the stepped position (:117-184)
                if (nl < 0) {
                    nl = 0;
                    dsN = d0;
                }
                act = A_CROSS;
                f.mode = S_TOP;
                if (opt_nidx<R, BATCH, BIG>(P, pk.inst, L) != opt_nidx<R, BATCH, BIG>(P, pk.inst, nl)) {
                    int which = -1;
                    if (dsL < (R)0 && dsN < (R)0) {
                        which = (fabs(dsL) <= fabs(dsN)) ? L : nl;
                    } else {
                        R tL, tN;
                        if (precise) {
                            tL = (R)eval_region_cold<double, MODS, S64>(sc64, L, f.x.oldpos);
                            tN = (R)eval_region_cold<double, MODS, S64>(sc64, nl, f.x.oldpos);
                        } else {
                            const V3<R> of = cv<R>(f.x.oldpos);
                            tL = eval_region_cold<R, MODS, S>(sc, L, of);
                            tN = eval_region_cold<R, MODS, S>(sc, nl, of);
                        }
                        if (tL < (R)0 && tN < (R)0) {
                            which = (tL >= tN) ? L : nl;
                        } else if (dsL >= (R)0 && dsN < (R)0) {
                            // exactly 0 counts as outside, like the `ds(i) < 0` membership
                            // test; the `error stop` branch (:155-156) is then reached only by NaN
                            which = (L == 0) ? L : nl;  // oldlayer = packet%layer, then "== 1" (:150-162)
                        } else if (dsL >= (R)0 && dsN >= (R)0) {
                            pk.tflag = true;
                        } else {
                            pk.tflag = true;
                            pk.flags |= STATUS_ERROR_STATE;
                        }
                    }
                    f.x.which = which;  // the boundary event runs in the A_CROSS phase below
                    f.x.nl = nl;
                } else {
                    pk.layer = nl;
                    f.x.which = -2;  // same refractive index: continue with the same tau
                }
                if (pk.tflag) act = end_flight(P, pk);
            }
        }
    }
    if (act == A_SWEEP + 100) act = A_SWEEP;
    // ---- boundary event in FP64: calcNormal + reflect_refract (surfaces.f90:14-40)
    if (act == A_CROSS) {
        act = sizeof(R) == 4 ? A_PRECISE : A_SWEEP;  // the next flight starts on the surface
        const int which = f.x.which;
        if (which >= 0) {
            const int L = pk.layer, nl = f.x.nl;
            ++c.fres;
            c.sdf += 4;
            const V3<double> Nn = calc_normal_cold<MODS, S64>(sc64, which, pk.pos, P.normal_h);
            V3<double> I{(double)pk.dir.x, (double)pk.dir.y, (double)pk.dir.z};
            const double m1 = opt_nidx64<R, BATCH, BIG>(P, pk.inst, L), m2 = opt_nidx64<R, BATCH, BIG>(P, pk.inst, nl);
            const double Rf = fresnel(I, Nn, m1, m2);
            const double u = (double)rng.next();
            const bool refl = u <= Rf;
            I = refl ? reflect(I, Nn) : refract(I, Nn, m1 / m2);
            pk.dir = V3<R>{(R)I.x, (R)I.y, (R)I.z};
            pk.weight = pk.weight * (R)Rf;
            f.tau = -log(rng.next());
            f.taurun = 0;
            if (!refl) {
                pk.layer = nl;
            } else {
                ++c.refl;
                pk.pos = f.x.oldpos;
                pk.bounces += 1;
                if (pk.bounces > 1000) {
                    pk.tflag = true;
                    act = end_flight(P, pk);
                }
            }
        }
    }
    // ---- walk voxel segments: at most SMCRT_WALK_SEGMENTS per lane per
    // iteration, so one long walk does not hold up the other lanes' actions
    for (int k = 0; k < SMCRT_WALK_SEGMENTS && act == A_WALK; ++k) {
        if (walk_segment<R, BATCH, ADJ, VAR>(P, pk, f, c, acc, vt, priv)) {
            pk.pos = advance(pk.pos, f.dsdf, pk.dir);
            cache_move(f);
            if (f.last) {
                act = end_flight(P, pk);  // taurun >= tau ends the flight (:100)
            } else {
                f.mode = S_STEP;
                // near a surface the next sweep is FP64: in the FP64 group, or (a
                // lane on the cache, one region) in its own next pass
                act = (sizeof(R) == 4 && f.near && !f.cache) ? A_PRECISE : A_SWEEP;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Packet slots of one CTA in shared memory (structure of arrays).  Between
// passes a packet is one slot; the union of the flight record is live only in
// two states (a voxel walk in progress; a crossing sweep pending) and is stored
// as raw 32-bit words.
#ifndef SMCRT_SLOTS_PER_THREAD
#define SMCRT_SLOTS_PER_THREAD 2
#endif
// Slots per thread: two for FP32 transport (124 bytes a slot); one for FP64
// (168 bytes), so that a CTA's slots stay within the 227 KiB of shared memory.
template <class R>
struct SlotCount {
    static constexpr int per_thread = sizeof(R) == 4 ? SMCRT_SLOTS_PER_THREAD : 1;
    static constexpr int n = kBlock * per_thread;
};
// Sort groups of the actions a packet can wait in between rounds, in list
// order: FP64 near-surface sweep, sweep (or a pending crossing), then walk,
// interact and retire/launch in the order of the launch's group_order.  Each
// warp's first chunk is fixed (warp w, chunk w), so the costly FP64 chunks at
// the head of the list go to different warps; the rest of the list goes to
// whichever warp finishes first, so the last group's chunks end each round.
// A_DONE maps to kGroups (not listed).  Nibble `act` of an order is the group
// of action `act`.
constexpr unsigned kOrderWalkLast = 0x05421314u;      // sweep, interact, walk, launch
constexpr unsigned kOrderInteractLast = 0x05431214u;  // sweep, walk, interact, launch
constexpr int kGroups = 5;
// Drain mode: at most this many live slots in a CTA (a few per warp), each run
// for kDrainPasses passes per round.
#ifndef SMCRT_DRAIN_LIVE_PER_WARP
#define SMCRT_DRAIN_LIVE_PER_WARP 4
#endif
#ifndef SMCRT_DRAIN_PASSES
#define SMCRT_DRAIN_PASSES 16
#endif
constexpr int kDrainLive = SMCRT_DRAIN_LIVE_PER_WARP * (kBlock / 32);
constexpr int kDrainPasses = SMCRT_DRAIN_PASSES;
static_assert(SMCRT_DRAIN_LIVE_PER_WARP <= 32, "one drain item per lane at most");
__device__ __forceinline__ int act_group(unsigned order, int act) { return (int)((order >> (4 * act)) & 0xFu); }
template <class R, bool ADJ, int kSlots = SlotCount<R>::n>
struct Slots {
    static constexpr int kRW = sizeof(R) / 4;  // 32-bit words per R
    // union words: walk (tx, ty, tz, td, step length, ci, cj, ck) or crossing
    // (position before the step, which, nl)
    static constexpr int kUW = 5 * kRW + 3 > 8 ? 5 * kRW + 3 : 8;
    static constexpr int kA = ADJ ? kSlots : 1;
    double px[kSlots], py[kSlots], pz[kSlots];
    R dx[kSlots], dy[kSlots], dz[kSlots], w[kSlots];
    R tau[kSlots], taurun[kSlots];
    uint32_t u[kUW][kSlots];
    // act | mode << 3 | last << 5 | tflag << 6 | adjoint pass << 7 | layer << 8 |
    // pk.flags << 16 | rng.flags << 24
    uint32_t meta[kSlots];
    // trace steps | nearest region << 21 | negx << 29 | cache valid << 30 | near << 31
    uint32_t steps[kSlots];
    int nscatt[kSlots];
    // nearest-region cache: clearance and the bound on |d_k| (not in adjoint launches)
    float clr[ADJ ? 1 : kSlots], dku[ADJ ? 1 : kSlots];
    uint32_t bl[kSlots];  // bounces (<= 1001) | rng.left << 11 | batch instance << 14
    // Philox block counter (replay builds: the injected uniforms consumed); the
    // draw count of a Philox stream is 4 words a block less the words left
    uint32_t p0[kSlots], p1[kSlots], block[kSlots];
    uint32_t b0[kSlots], b1[kSlots], b2[kSlots], b3[kSlots];
    double ctot[kA], cpre[kA];  // adjoint launches only (FP64, see Pk)
};
// Regions addressable by the 8-bit layer field of a slot.
constexpr int kMaxLayerField = 256;

template <class R, int kSlots>
__device__ __forceinline__ void put_r(uint32_t (*u)[kSlots], int k, int s, R v) {
    if (sizeof(R) == 4) {
        u[k][s] = __float_as_uint((float)v);
    } else {
        const unsigned long long b = (unsigned long long)__double_as_longlong((double)v);
        u[k][s] = (uint32_t)b;
        u[k + 1][s] = (uint32_t)(b >> 32);
    }
}
template <class R, int kSlots>
__device__ __forceinline__ R get_r(const uint32_t (*u)[kSlots], int k, int s) {
    if (sizeof(R) == 4) return (R)__uint_as_float(u[k][s]);
    return (R)__longlong_as_double((long long)(((unsigned long long)u[k + 1][s] << 32) | u[k][s]));
}

template <class R, bool REPLAY, bool BATCH, bool ADJ>
__device__ __forceinline__ int load_slot(const Slots<R, ADJ>& sl, int s, const Params<R>& P, const Buffers& B,
                                         Pk<R>& pk, Flight<R>& f, Stream<R, REPLAY>& rng) {
    const uint32_t m = sl.meta[s];
    const int act = (int)(m & 7u);
    f.mode = (int)((m >> 3) & 3u);
    f.last = (m >> 5) & 1u;
    pk.tflag = (m >> 6) & 1u;
    pk.phase = ADJ ? (int)((m >> 7) & 1u) : 0;
    pk.layer = (int)((m >> 8) & 255u);
    pk.flags = (int)((m >> 16) & 255u);
    rng.flags = (int)(m >> 24);
    pk.inst = 0;
    if (act == A_NEW) return act;
    pk.pos = V3<double>{sl.px[s], sl.py[s], sl.pz[s]};
    pk.dir = V3<R>{sl.dx[s], sl.dy[s], sl.dz[s]};
    pk.weight = sl.w[s];
    f.tau = sl.tau[s];
    f.taurun = sl.taurun[s];
    const uint32_t sw = sl.steps[s];
    f.steps = (int)(sw & 0x1FFFFFu);
    f.nk = (int)((sw >> 21) & 255u);
    f.negx = (sw >> 29) & 1u;
    f.cache = !ADJ && ((sw >> 30) & 1u);
    f.near = (sw >> 31) & 1u;
    f.clear = ADJ ? 0.0f : sl.clr[ADJ ? 0 : s];
    f.dkup = ADJ ? 0.0f : sl.dku[ADJ ? 0 : s];
    pk.nscatt = sl.nscatt[s];
    const uint32_t bl = sl.bl[s];
    pk.bounces = (int)(bl & 0x7FFu);
    rng.left = (int)((bl >> 11) & 7u);
    pk.inst = BATCH ? (int)(bl >> 14) : 0;
    rng.p0 = sl.p0[s];
    rng.p1 = sl.p1[s];
    if (REPLAY) {
        rng.block = 0;
        rng.ndraws = (int)sl.block[s];
    } else {
        rng.block = sl.block[s];
        rng.ndraws = (int)((4u * rng.block - (unsigned)rng.left) / (unsigned)U01<R>::kWords);
    }
    rng.b0 = sl.b0[s];
    rng.b1 = sl.b1[s];
    rng.b2 = sl.b2[s];
    rng.b3 = sl.b3[s];
    rng.seed = BATCH ? P.bseed[pk.inst] : P.seed;  // the stream key: the launch's, or the instance's
    if (ADJ) {
        pk.ctot = sl.ctot[s];
        pk.cpre = sl.cpre[s];
    }
    rng.inst = P.instance;
    if (REPLAY) {
        const long long pid = (long long)(((uint64_t)rng.p1 << 32) | rng.p0) - P.first;
        const long long o0 = B.offsets[pid], o1 = B.offsets[pid + 1];
        rng.inj = B.uniforms + o0;
        rng.ninj = (int)(o1 - o0);
    }
    constexpr int W = Slots<R, ADJ>::kRW;
    if (act == A_WALK) {
        f.w.tx = get_r<R>(sl.u, 0, s);
        f.w.ty = get_r<R>(sl.u, W, s);
        f.w.tz = get_r<R>(sl.u, 2 * W, s);
        f.w.td = get_r<R>(sl.u, 3 * W, s);
        f.dsdf = get_r<R>(sl.u, 4 * W, s);
        f.w.ci = (int)sl.u[5 * W][s];
        f.w.cj = (int)sl.u[5 * W + 1][s];
        f.w.ck = (int)sl.u[5 * W + 2][s];
    } else if ((act == A_SWEEP || act == A_PRECISE) && f.mode == S_CROSS) {
        f.x.oldpos.x = get_r<double>(sl.u, 0, s);
        f.x.oldpos.y = get_r<double>(sl.u, 2, s);
        f.x.oldpos.z = get_r<double>(sl.u, 4, s);
        f.x.which = (int)sl.u[6][s];
        f.x.nl = (int)sl.u[7][s];
    }
    return act;
}

template <class R, bool REPLAY, bool BATCH, bool ADJ>
__device__ __forceinline__ void store_slot(Slots<R, ADJ>& sl, int s, int act, const Pk<R>& pk, const Flight<R>& f,
                                           const Stream<R, REPLAY>& rng) {
    sl.meta[s] = (uint32_t)act | ((uint32_t)f.mode << 3) | ((uint32_t)f.last << 5) | ((uint32_t)pk.tflag << 6) |
                 ((uint32_t)(ADJ ? pk.phase & 1 : 0) << 7) | ((uint32_t)pk.layer << 8) | ((uint32_t)pk.flags << 16) |
                 ((uint32_t)rng.flags << 24);
    if (act == A_DONE) return;
    sl.px[s] = pk.pos.x;
    sl.py[s] = pk.pos.y;
    sl.pz[s] = pk.pos.z;
    sl.dx[s] = pk.dir.x;
    sl.dy[s] = pk.dir.y;
    sl.dz[s] = pk.dir.z;
    sl.w[s] = pk.weight;
    sl.tau[s] = f.tau;
    sl.taurun[s] = f.taurun;
    sl.steps[s] = (uint32_t)f.steps | ((uint32_t)f.nk << 21) | ((uint32_t)f.negx << 29) |
                  ((uint32_t)(!ADJ && f.cache) << 30) | ((uint32_t)f.near << 31);
    if (!ADJ) {
        sl.clr[ADJ ? 0 : s] = f.clear;
        sl.dku[ADJ ? 0 : s] = f.dkup;
    }
    sl.nscatt[s] = pk.nscatt;
    sl.bl[s] = (uint32_t)pk.bounces | ((uint32_t)rng.left << 11) | ((uint32_t)(BATCH ? pk.inst : 0) << 14);
    sl.p0[s] = rng.p0;
    sl.p1[s] = rng.p1;
    sl.block[s] = REPLAY ? (uint32_t)rng.ndraws : rng.block;
    sl.b0[s] = rng.b0;
    sl.b1[s] = rng.b1;
    sl.b2[s] = rng.b2;
    sl.b3[s] = rng.b3;
    if (ADJ) {
        sl.ctot[s] = pk.ctot;
        sl.cpre[s] = pk.cpre;
    }
    constexpr int W = Slots<R, ADJ>::kRW;
    if (act == A_WALK) {
        put_r<R>(sl.u, 0, s, f.w.tx);
        put_r<R>(sl.u, W, s, f.w.ty);
        put_r<R>(sl.u, 2 * W, s, f.w.tz);
        put_r<R>(sl.u, 3 * W, s, f.w.td);
        put_r<R>(sl.u, 4 * W, s, f.dsdf);
        sl.u[5 * W][s] = (uint32_t)f.w.ci;
        sl.u[5 * W + 1][s] = (uint32_t)f.w.cj;
        sl.u[5 * W + 2][s] = (uint32_t)f.w.ck;
    } else if ((act == A_SWEEP || act == A_PRECISE) && f.mode == S_CROSS) {
        put_r<double>(sl.u, 0, s, f.x.oldpos.x);
        put_r<double>(sl.u, 2, s, f.x.oldpos.y);
        put_r<double>(sl.u, 4, s, f.x.oldpos.z);
        sl.u[6][s] = (uint32_t)f.x.which;
        sl.u[7][s] = (uint32_t)f.x.nl;
    }
}

// Byte offset of the privatised fluence sub-box after the detector bins (8-aligned).
__host__ __device__ constexpr size_t priv_offset(int sbins) { return ((size_t)sbins * 4 + 7) / 8 * 8; }

// Dynamic shared memory of one CTA: the slots, then the privatized detector bins.
template <class R, bool ADJ = false>
__host__ __device__ constexpr size_t slots_bytes() {
    return (sizeof(Slots<R, ADJ>) + 15) / 16 * 16;
}

// The persistent, compacted kernel.  KERNEL: smcrt_kernel_kind.  REPLAY:
// injected streams.
//
// A CTA holds SlotCount<R>::n packets in shared memory.  Each round it counting-sorts
// its live slots by their next action (warp ballots, stable in slot order), then
// the warps take 32-item chunks of the sorted list, run one pass of each packet's
// state machine and write the packets back.  A warp therefore works on 32
// packets that start the pass with the same action, whatever mix of actions the
// CTA's packets are in; rare actions (boundary events, retire and launch) are
// gathered across the CTA instead of stalling 31 idle lanes.  Chunks of a group
// hold consecutive slots, so the structure-of-arrays slot accesses of a warp fall
// in different shared-memory banks, and the warps of a round run the same
// action's code at about the same time.
// MODS = false compiles every distance evaluation without the modifier code,
// for scenes whose primitives carry no modifiers.  BIG reads the scene from
// device memory (scenes beyond the parameter block's kMaxRegions/kMaxPrims).
template <class R, int KERNEL, bool REPLAY, bool BATCH = false, bool ADJ = false, bool MODS = true, bool BIG = false,
          bool VAR = false>
__global__ void __launch_bounds__(kBlock, SMCRT_MIN_BLOCKS) transport_kernel(const __grid_constant__ Params<R> P,
                                                                             const Buffers B) {
    constexpr int NS = SlotCount<R>::n;
    __shared__ unsigned long long s_cnt[C_NUM];
    __shared__ double s_mom[25];
    __shared__ int s_stop;  // the time budget ran out
    extern __shared__ __align__(16) unsigned char s_dyn[];
    Slots<R, ADJ>& sl = *reinterpret_cast<Slots<R, ADJ>*>(s_dyn);
    unsigned* s_bins = reinterpret_cast<unsigned*>(s_dyn + slots_bytes<R, ADJ>());
    unsigned long long* s_priv =
        reinterpret_cast<unsigned long long*>(s_dyn + slots_bytes<R, ADJ>() + priv_offset(P.sbins));
    const int t = threadIdx.x;
    const unsigned lane = lane_id();
    if (t < C_NUM) s_cnt[t] = 0ull;
    if (t < 25) s_mom[t] = 0.0;
    for (int i = t; i < P.sbins; i += kBlock) s_bins[i] = 0u;
    if (!ADJ && !BATCH)
        for (int i = t; i < P.priv_n; i += kBlock) s_priv[i] = 0ull;
    for (int i = t; i < NS; i += kBlock) sl.meta[i] = (uint32_t)A_NEW;
    // adjoint: per-thread gradient accumulators [3][kMaxAdjGroups][kBlock]
    __shared__ float s_acc[ADJ ? 3 * kMaxAdjGroups * kBlock : 1];
    if (ADJ)
        for (int i = t; i < 3 * kMaxAdjGroups * kBlock; i += kBlock) s_acc[i] = 0.0f;
    Pk<R> pk;
    pk.inst = 0;
    pk.phase = 0;
    pk.ctot = pk.cpre = 0.0;
    Flight<R> f;
    Stream<R, REPLAY> rng;
    Cnt c = {0, 0, 0, 0, 0, 0, 0};
    const unsigned long long t0 = global_ns();
    // this CTA's voxel-score tables (second-moment runs)
    unsigned char* const vbase = VAR ? P.var_tab + (size_t)blockIdx.x * NS * kVarSlotBytes : nullptr;
    const unsigned lt = (1u << lane) - 1u;
    // ---- rounds: each round counting-sorts the live slots by action (warp
    // ballots and a per-warp scan, stable in slot order) and the warps take
    // 32-item chunks of the sorted list; three CTA barriers a round
    constexpr int Q = SlotCount<R>::per_thread;
    constexpr int NW = kBlock / 32;
    __shared__ int s_off[kGroups][Q][NW];
    __shared__ unsigned short s_list[NS];
    __shared__ int s_next;
    const int warp = t >> 5;
    for (;;) {
        __syncthreads();  // the previous round's slot writes are visible
        int a[Q], rank[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            a[q] = act_group(P.group_order, (int)(sl.meta[t + q * kBlock] & 7u));
            rank[q] = 0;
#pragma unroll
            for (int g = 0; g < kGroups; ++g) {
                const unsigned m = __ballot_sync(0xffffffffu, a[q] == g);
                if (a[q] == g) rank[q] = __popc(m & lt);
                if (lane == 0) s_off[g][q][warp] = __popc(m);
            }
        }
        if (t == 0) {
            int stop = 0;
            if (P.budget_ns && global_ns() - t0 > P.budget_ns) {
                atomicOr(B.status, STATUS_ABORTED);
                stop = 1;
            }
            s_stop = stop;
            s_next = NW;
        }
        __syncthreads();
        int total;
        {
            constexpr int E = kGroups * Q * NW;
            constexpr int PER = (E + 31) / 32;
            const int* flat = &s_off[0][0][0];
            int v[PER], sum = 0;
#pragma unroll
            for (int k = 0; k < PER; ++k) {
                const int e = (int)lane * PER + k;
                v[k] = e < E ? flat[e] : 0;
                sum += v[k];
            }
            int incl = sum;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, d);
                if ((int)lane >= d) incl += y;
            }
            total = __shfl_sync(0xffffffffu, incl, 31);
            const int excl = incl - sum;
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int g = a[q] < kGroups ? a[q] : 0;
                const int e = (g * Q + q) * NW + warp;
                const int src = e / PER, k = e % PER;
                int off = __shfl_sync(0xffffffffu, excl, src);
#pragma unroll
                for (int kk = 0; kk < PER; ++kk) {
                    const int vk = __shfl_sync(0xffffffffu, v[kk], src);
                    if (kk < k) off += vk;
                }
                if (a[q] < kGroups) s_list[off + rank[q]] = (unsigned short)(t + q * kBlock);
            }
        }
        const int stop = s_stop;
        __syncthreads();
        if (total == 0 || stop) break;
        // drain: few live packets left in this CTA (the end of a launch, or long
        // histories such as a packet creeping along a wall in steps of its
        // distance to it).  They are spread one to a few per warp (item
        // warp + NW x lane) and each runs kDrainPasses passes before it goes back
        // to its slot, so that a long chain of dependent steps does not wait for
        // a sort per step.  Otherwise warps take 32-item chunks.  One call site
        // of the pass serves both.
        const bool drain = total <= kDrainLive;
        const int nchunks = drain ? NW : (total + 31) >> 5;
        const int reps = drain ? kDrainPasses : 1;
        for (int chunk = warp; chunk < nchunks;) {
            const int i = drain ? chunk + NW * (int)lane : chunk * 32 + (int)lane;
            if (i < total) {
                const int s = s_list[i];
                int act = load_slot<R, REPLAY, BATCH, ADJ>(sl, s, P, B, pk, f, rng);
                for (int r = 0; r < reps; ++r) {
                    transport_pass<R, KERNEL, REPLAY, BATCH, ADJ, MODS, BIG, VAR>(
                        P, B, pk, f, rng, c, act, s_cnt, s_mom, s_bins, s_acc,
                        VAR ? vbase + (size_t)s * kVarSlotBytes : nullptr, s_priv);
                    if (act == A_DONE) break;
                }
                store_slot<R, REPLAY, BATCH, ADJ>(sl, s, act, pk, f, rng);
            }
            if (drain) break;
            int next = 0;
            if (lane == 0) next = atomicAdd(&s_next, 1);
            chunk = __shfl_sync(0xffffffffu, next, 0);
        }
    }
    // events of packets still in flight (time budget) and since the last retire
    atomicAdd(&s_cnt[C_SDF], (unsigned long long)c.sdf);
    atomicAdd(&s_cnt[C_VOX], (unsigned long long)c.vox);
    atomicAdd(&s_cnt[C_STEPS], (unsigned long long)c.steps);
    atomicAdd(&s_cnt[C_SCAT], (unsigned long long)c.scat);
    atomicAdd(&s_cnt[C_FRES], (unsigned long long)c.fres);
    atomicAdd(&s_cnt[C_REFL], (unsigned long long)c.refl);
    if (VAR) atomicAdd(&s_cnt[C_VAROVF], (unsigned long long)c.varovf);
    __syncthreads();
    if (t < C_NUM && s_cnt[t]) atomicAdd(B.counters + t, s_cnt[t]);
    if (t < 25 && s_mom[t] != 0.0) atomicAdd(B.moments + t, s_mom[t]);
    for (int i = t; i < P.sbins; i += kBlock)
        if (s_bins[i]) atomicAdd(B.bins + i, (double)s_bins[i]);
    if (!ADJ && !BATCH && P.priv_n) {  // the privatised sub-box, one FP64 add per nonzero cell
        double* grid = tally_grid<R, BATCH>(P, 0);
        for (int i = t; i < P.priv_n; i += kBlock) {
            const unsigned long long v = s_priv[i];
            if (!v) continue;
            const int li = i % P.priv_d[0], lj = (i / P.priv_d[0]) % P.priv_d[1], lk = i / (P.priv_d[0] * P.priv_d[1]);
            const long long g = (long long)(P.priv_o[0] + li) +
                                (long long)P.grid.nx * ((P.priv_o[1] + lj) + (long long)P.grid.ny * (P.priv_o[2] + lk));
            atomicAdd(grid + g, (double)(long long)v / kPrivScale);
        }
    }
    if (ADJ && t < 3 * P.adj_ngroups) {  // thread (k, group) sums its row over the CTA's threads
        const int k = t / P.adj_ngroups, grp = t % P.adj_ngroups;
        const float* row = s_acc + (k * kMaxAdjGroups + grp) * kBlock;
        double sum = 0.0;
        for (int i = 0; i < kBlock; ++i) sum += (double)row[i];
        atomicAdd(P.adj_out + k * P.adj_ngroups + grp, sum);
    }
}

}  // namespace smcrt
