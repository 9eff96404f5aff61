"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (oracle/lib/libsmcrt_oracle.so).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker.  The oracle restates signedMCRT's transport path on the CPU; see
oracle/smcrt_oracle.cpp for the reference lines each part follows.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from signedmcrt_b200 import abi
from signedmcrt_b200.config import Settings
from signedmcrt_b200.scene import FlatScene

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "libsmcrt_oracle.so"


class Policy(C.Structure):
    _fields_ = [("precision", C.c_int32), ("ref_dda", C.c_int32), ("crossing_f64", C.c_int32),
                ("tally_f32", C.c_int32), ("threads", C.c_int32), ("near_surface_f64", C.c_int32),
                ("eps", C.c_double), ("delta", C.c_double), ("normal_h", C.c_double),
                ("max_trace_steps", C.c_int64)]


def reference_policy(threads: int = 0, tally_f32: bool = False) -> Policy:
    """The reference algorithm as written: FP64, eps = 1e-8, snapping voxel walk."""
    return Policy(abi.FP64, 1, 1, int(tally_f32), threads, 0, 1e-8, 1e-8, 1e-6, 0)


def device_policy(precision: str, grid: abi.Grid, threads: int = 0) -> Policy:
    """The GPU algorithm: integer voxel walk, FP64 boundary events, the reference's
    eps; in FP32, sweeps within 16 FP32 ulps of a surface (of the scene size) and
    after crossing steps in FP64."""
    eps = 1e-8
    near = 1 if precision == "fp32" else 0
    return Policy(abi.FP32 if precision == "fp32" else abi.FP64, 0, 1, 0, threads, near, eps, 1e-8, 1e-6, 0)


_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        P = C.POINTER
        sig = {
            "oracle_run": ([P(abi.Scene), P(abi.Grid), P(abi.Source), P(abi.Detector), C.c_int32, C.c_int32,
                            C.c_int32, P(Policy), C.c_int64, C.c_int64, C.c_uint64, C.c_uint32, P(C.c_double),
                            P(C.c_int64), P(C.c_double), P(C.c_double), P(abi.Stats), C.c_void_p,
                            P(C.c_double)], C.c_int32),
            "oracle_detector_bins": ([P(abi.Detector), C.c_int32], C.c_int64),
            "oracle_adjoint": ([P(abi.Scene), P(abi.Grid), P(abi.Source), P(abi.Detector), C.c_int32, P(Policy),
                                C.c_int64, C.c_uint64, P(C.c_double), P(C.c_double), P(C.c_int32), C.c_int32,
                                P(C.c_double)], C.c_int32),
            "oracle_eval_sdf": ([P(abi.Scene), C.c_int32, P(C.c_double), C.c_int64, P(C.c_double)], C.c_int32),
            "oracle_intersect_plane": ([P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double)],
                                       C.c_int32),
            "oracle_intersect_circle": ([P(C.c_double), P(C.c_double), C.c_double, P(C.c_double), P(C.c_double),
                                        P(C.c_double)], C.c_int32),
            "oracle_calc_normal": ([P(abi.Scene), C.c_int32, C.c_double, P(C.c_double), C.c_int64,
                                    P(C.c_double)], C.c_int32),
            "oracle_render": ([P(abi.Scene), C.c_int32, P(C.c_int32), P(C.c_double), P(C.c_float)], C.c_int32),
            "oracle_fresnel": ([C.c_int32, P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double),
                                C.c_int64, P(C.c_double)], C.c_int32),
            "oracle_reflect_refract": ([C.c_int32, P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double),
                                        P(C.c_double), C.c_int64, P(C.c_double), P(C.c_int32)], C.c_int32),
            "oracle_scatter_dir": ([C.c_int32, P(C.c_double), P(C.c_double), P(C.c_double), C.c_int64,
                                    P(C.c_double)], C.c_int32),
            "oracle_philox": ([P(C.c_uint32), P(C.c_uint32), C.c_int64, P(C.c_uint32)], C.c_int32),
            "oracle_emit": ([P(abi.Scene), P(abi.Grid), P(abi.Source), C.c_int32, C.c_int64, C.c_int64,
                             C.c_uint64, P(C.c_double), P(C.c_double), P(C.c_int32)], C.c_int32),
            "oracle_detector_bin": ([P(abi.Detector), C.c_int32, C.c_int32, P(C.c_double), P(C.c_double),
                                     C.c_double, C.c_int32], C.c_int64),
            "oracle_max_threads": ([], C.c_int32),
        }
        abi.bind(L, sig)
        _lib = L
    return _lib


@dataclass
class OracleResult:
    jmean: np.ndarray | None
    bins: np.ndarray
    stats: dict
    states: np.ndarray | None = None
    jmean2: np.ndarray | None = None  # per voxel: sum over packets of the packet's score squared

    @property
    def nscatt(self) -> float:
        return self.stats["nscatt"]


KERNELS = {"pathlength": abi.KERNEL_PATHLENGTH, "weight": abi.KERNEL_WEIGHT, "test": abi.KERNEL_TEST}


def run(array, st: Settings, *, nphotons: int, seed: int, policy: Policy | None = None, kernel: str = "pathlength",
        end_early: bool = False, first: int = 0, instance: int = 0, uniforms=None, offsets=None,
        want_jmean: bool = True, want_states: bool = False, want_moments: bool = False) -> OracleResult:
    flat = array if isinstance(array, FlatScene) else FlatScene(array)
    grid, src = st.grid_c(), st.source_c()
    dets = st.detectors_c()
    darr = (abi.Detector * max(1, len(dets)))(*dets)
    nb = int(lib().oracle_detector_bins(darr, len(dets))) if dets else 0
    pol = policy if policy is not None else reference_policy()
    g = st.grid
    jm = np.empty(g.nxg * g.nyg * g.nzg, dtype=np.float64) if want_jmean else None
    bins = np.zeros(max(nb, 1), dtype=np.float64)
    stats = abi.Stats()
    states = np.zeros(max(nphotons, 1), dtype=abi.PACKET_STATE_DTYPE) if want_states else None
    j2 = np.empty(g.nxg * g.nyg * g.nzg, dtype=np.float64) if want_moments else None
    u = o = None
    if uniforms is not None:
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        o = np.ascontiguousarray(offsets, dtype=np.int64)
    rc = lib().oracle_run(flat.ptr(), C.byref(grid), C.byref(src), darr, len(dets), KERNELS[kernel],
                          int(end_early), C.byref(pol), first, nphotons, seed, instance, abi.dptr(u), abi.i64ptr(o),
                          abi.dptr(jm), abi.dptr(bins), C.byref(stats),
                          states.ctypes.data_as(C.c_void_p) if states is not None else None, abi.dptr(j2))
    if rc != 0:
        raise RuntimeError(f"oracle_run failed ({rc})")
    shape = (g.nxg, g.nyg, g.nzg)
    return OracleResult(jm.reshape(shape, order="F") if jm is not None else None, bins[:nb],
                        stats.to_dict(), states[:nphotons] if states is not None else None,
                        j2.reshape(shape, order="F") if j2 is not None else None)


def adjoint(array, st: Settings, *, nphotons: int, seed: int, w, h, region_group, ngroups: int,
            policy: Policy | None = None) -> tuple[np.ndarray, float]:
    """Perturbation Monte Carlo reference gradient of L = sum_v w[v] jmean[v] +
    sum_b h[b] bins[b] over packets [0, nphotons) of the pathlength kernel:
    (grad (3, ngroups) -- rows d/d mua, d/d mus, d/d g of each group, summed over
    packets -- and L).  w: voxel weights in Fortran order (nxg, nyg, nzg); h: bin
    weights or None."""
    flat = array if isinstance(array, FlatScene) else FlatScene(array)
    grid, src = st.grid_c(), st.source_c()
    dets = st.detectors_c()
    darr = (abi.Detector * max(1, len(dets)))(*dets)
    pol = policy if policy is not None else reference_policy()
    wv = np.ascontiguousarray(np.asarray(w, dtype=np.float64).reshape(-1, order="F"))
    if wv.size != st.grid.nxg * st.grid.nyg * st.grid.nzg:
        raise ValueError("adjoint: w needs one weight per voxel")
    hv = None if h is None else np.ascontiguousarray(h, dtype=np.float64)
    rg = np.ascontiguousarray(region_group, dtype=np.int32)
    out = np.zeros(3 * ngroups + 1)
    rc = lib().oracle_adjoint(flat.ptr(), C.byref(grid), C.byref(src), darr, len(dets), C.byref(pol), nphotons,
                              seed, abi.dptr(wv), abi.dptr(hv), abi.i32ptr(rg), ngroups, abi.dptr(out))
    if rc != 0:
        raise RuntimeError(f"oracle_adjoint failed ({rc})")
    return out[: 3 * ngroups].reshape(3, ngroups), float(out[3 * ngroups])


def eval_sdf(flat: FlatScene, pts, precision: str = "fp64") -> np.ndarray:
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.empty((len(pts), flat.nregions))
    assert lib().oracle_eval_sdf(flat.ptr(), abi.FP32 if precision == "fp32" else abi.FP64, abi.dptr(pts),
                                 len(pts), abi.dptr(out)) == 0
    return out


def render(flat: FlatScene, samples, extent, precision: str = "fp64") -> np.ndarray:
    """render_sub (src/sdfs/sdf_base.f90:302-346): the FP32 voxel image, shape samples."""
    ns = np.ascontiguousarray(samples, dtype=np.int32)
    ext = np.ascontiguousarray(extent, dtype=np.float64)
    img = np.empty(int(np.prod(ns, dtype=np.int64)), dtype=np.float32)
    assert lib().oracle_render(flat.ptr(), abi.FP32 if precision == "fp32" else abi.FP64,
                               ns.ctypes.data_as(C.POINTER(C.c_int32)), abi.dptr(ext),
                               img.ctypes.data_as(C.POINTER(C.c_float))) == 0
    return img.reshape(tuple(int(x) for x in ns), order="F")


def _v3(v):
    return np.ascontiguousarray(v, dtype=np.float64)


def intersect_plane(n, p0, l0, l) -> tuple[bool, float]:
    """intersectPlane (src/geometryMod.f90:217-241): (hit, t)."""
    t = C.c_double(0.0)
    hit = lib().oracle_intersect_plane(abi.dptr(_v3(n)), abi.dptr(_v3(p0)), abi.dptr(_v3(l0)), abi.dptr(_v3(l)),
                                       C.byref(t))
    return bool(hit), t.value


def intersect_circle(n, p0, radius, l0, l) -> tuple[bool, float]:
    """intersectCircle (src/geometryMod.f90:244-270): (hit, t)."""
    t = C.c_double(0.0)
    hit = lib().oracle_intersect_circle(abi.dptr(_v3(n)), abi.dptr(_v3(p0)), float(radius), abi.dptr(_v3(l0)),
                                        abi.dptr(_v3(l)), C.byref(t))
    return bool(hit), t.value


def calc_normal(flat: FlatScene, region0: int, pts, h: float = 1e-6) -> np.ndarray:
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.empty_like(pts)
    assert lib().oracle_calc_normal(flat.ptr(), region0, h, abi.dptr(pts), len(pts), abi.dptr(out)) == 0
    return out


def fresnel(I, N, n1, n2, precision: str = "fp64") -> np.ndarray:
    I = np.ascontiguousarray(I, dtype=np.float64).reshape(-1, 3)
    N = np.ascontiguousarray(N, dtype=np.float64).reshape(-1, 3)
    n1 = np.ascontiguousarray(np.broadcast_to(n1, len(I)), dtype=np.float64)
    n2 = np.ascontiguousarray(np.broadcast_to(n2, len(I)), dtype=np.float64)
    R = np.empty(len(I))
    assert lib().oracle_fresnel(abi.FP32 if precision == "fp32" else abi.FP64, abi.dptr(I), abi.dptr(N),
                                abi.dptr(n1), abi.dptr(n2), len(I), abi.dptr(R)) == 0
    return R


def reflect_refract(I, N, n1, n2, u, precision: str = "fp64"):
    I = np.ascontiguousarray(I, dtype=np.float64).reshape(-1, 3)
    N = np.ascontiguousarray(N, dtype=np.float64).reshape(-1, 3)
    n = len(I)
    n1 = np.ascontiguousarray(np.broadcast_to(n1, n), dtype=np.float64)
    n2 = np.ascontiguousarray(np.broadcast_to(n2, n), dtype=np.float64)
    u = np.ascontiguousarray(np.broadcast_to(u, n), dtype=np.float64)
    out = np.empty_like(I)
    refl = np.empty(n, dtype=np.int32)
    assert lib().oracle_reflect_refract(abi.FP32 if precision == "fp32" else abi.FP64, abi.dptr(I), abi.dptr(N),
                                        abi.dptr(n1), abi.dptr(n2), abi.dptr(u), n, abi.dptr(out),
                                        abi.i32ptr(refl)) == 0
    return out, refl.astype(bool)


def scatter_dir(dirs, g, u, precision: str = "fp64") -> np.ndarray:
    dirs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
    n = len(dirs)
    g = np.ascontiguousarray(np.broadcast_to(g, n), dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(n, 3)
    out = np.empty_like(dirs)
    assert lib().oracle_scatter_dir(abi.FP32 if precision == "fp32" else abi.FP64, abi.dptr(dirs), abi.dptr(g),
                                    abi.dptr(u), n, abi.dptr(out)) == 0
    return out


def philox(key, ctr) -> np.ndarray:
    key = np.ascontiguousarray(key, dtype=np.uint32).reshape(-1, 2)
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
    out = np.empty_like(ctr)
    assert lib().oracle_philox(abi.u32ptr(key), abi.u32ptr(ctr), len(ctr), abi.u32ptr(out)) == 0
    return out


def emit(flat: FlatScene, st: Settings, n: int, seed: int, precision: str = "fp64", first: int = 0):
    grid, src = st.grid_c(), st.source_c()
    pos = np.empty((n, 3))
    d = np.empty((n, 3))
    layer = np.empty(n, dtype=np.int32)
    assert lib().oracle_emit(flat.ptr(), C.byref(grid), C.byref(src), abi.FP32 if precision == "fp32" else abi.FP64,
                             first, n, seed, abi.dptr(pos), abi.dptr(d), abi.i32ptr(layer)) == 0
    return pos, d, layer


def detector_bin(st: Settings, det: int, pos, dirv, value: float, layer1: int) -> int:
    dets = st.detectors_c()
    darr = (abi.Detector * max(1, len(dets)))(*dets)
    p = np.ascontiguousarray(pos, dtype=np.float64)
    l = np.ascontiguousarray(dirv, dtype=np.float64)
    return int(lib().oracle_detector_bin(darr, len(dets), det, abi.dptr(p), abi.dptr(l), value, layer1))


def max_threads() -> int:
    return int(lib().oracle_max_threads())
