"""Python view of the C ABI: one `Transport` per simulation (smcrt_create), with
host-buffer runs (smcrt_run), device-resident runs (smcrt_run_device, e.g. into
torch tensors), stream replay (smcrt_replay) and batched runs.

Fluence arrays come back as (nxg, nyg, nzg) float64 views in Fortran order, so
`jmean[i-1, j-1, k-1]` is the reference's `jmean(i, j, k)`.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi
from ._lib import check, lib
from .config import Settings
from .scene import FlatScene

KERNELS = {"pathlength": abi.KERNEL_PATHLENGTH, "weight": abi.KERNEL_WEIGHT, "test": abi.KERNEL_TEST}
PRECISIONS = {"fp32": abi.FP32, "fp64": abi.FP64}


@dataclass
class RunResult:
    jmean: np.ndarray | None      # (nxg, nyg, nzg) float64, Fortran order
    bins: np.ndarray | None       # concatenated detector bins
    stats: dict
    jmean2: np.ndarray | None = None  # second moment: sum over packets of each packet's score squared

    @property
    def nscatt(self) -> float:
        return self.stats["nscatt"]


class Transport:
    def __init__(self, array, settings: Settings, *, kernel: str = "pathlength", precision: str = "fp32",
                 end_early: bool = False, stream: int | None = None, block_size: int = 0, blocks_per_sm: int = 0,
                 eps: float = 0.0, normal_h: float = 0.0, max_trace_steps: int = 0, timeout_ms: int = 0,
                 instance: int = 0, tally_copies: int = 0, scene_memory: int = 0, variance: bool = False,
                 nearest_cache: int = 0, shared_fluence: int = 0, group_order: int = 0):
        self.settings = settings
        self.flat = array if isinstance(array, FlatScene) else FlatScene(array)
        self.grid = settings.grid_c()
        self.source = settings.source_c()
        dets = settings.detectors_c()
        self._dets = (abi.Detector * max(1, len(dets)))(*dets)
        self.ndet = len(dets)
        o = abi.Options()
        o.kernel = KERNELS[kernel]
        o.precision = PRECISIONS[precision]
        o.end_early = int(bool(end_early))
        o.block_size, o.blocks_per_sm = block_size, blocks_per_sm
        o.max_trace_steps = max_trace_steps
        o.eps, o.normal_h = eps, normal_h
        o.instance = instance
        o.timeout_ms = timeout_ms
        o.tally_copies = tally_copies  # 0: library choice; 1: a single fluence grid
        o.scene_memory = scene_memory  # 1: the scene from device memory even when it fits the parameter block
        o.variance = int(bool(variance))  # keep the per-voxel second moment (run_moments)
        o.nearest_cache = nearest_cache  # 0: library choice; 1: on where allowed; 2: off
        o.shared_fluence = shared_fluence  # 0: library choice (autotuned); 1: on (FP32 pencil); 2: off
        o.group_order = group_order  # 0: library choice; abi.ORDER_WALK_LAST / abi.ORDER_INTERACT_LAST
        # stream=None: a stream private to this context; an int: that cudaStream_t (0 = default)
        o.stream = stream if stream is not None else None
        o.private_stream = int(stream is None)
        self.options = o
        self.kernel, self.precision = kernel, precision
        self._ctx = C.c_void_p()
        check(lib().smcrt_create(self.flat.ptr(), C.byref(self.grid), C.byref(self.source), self._dets,
                                 self.ndet, C.byref(o), C.byref(self._ctx)))
        self.nbins = int(lib().smcrt_detector_bins(self._ctx))
        g = settings.grid
        self.shape = (g.nxg, g.nyg, g.nzg)
        self.ncell = g.nxg * g.nyg * g.nzg

    # ------------------------------------------------------------------
    def close(self) -> None:
        if self._ctx:
            lib().smcrt_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _grid_view(self, flat: np.ndarray) -> np.ndarray:
        return flat.reshape(self.shape, order="F")

    # ------------------------------------------------------------------
    def run(self, nphotons: int, seed: int, *, jmean_out: np.ndarray | None = None,
            bins_out: np.ndarray | None = None, want_jmean: bool = True) -> RunResult:
        """Packets [0, nphotons) of stream `seed`; tallies copied to host buffers
        (pass pinned buffers as jmean_out/bins_out to reuse them)."""
        jm = None
        if want_jmean:
            jm = jmean_out if jmean_out is not None else np.empty(self.ncell, dtype=np.float64)
        bins = bins_out if bins_out is not None else np.zeros(max(self.nbins, 0), dtype=np.float64)
        st = abi.Stats()
        check(lib().smcrt_run(self._ctx, int(nphotons), int(seed), abi.dptr(jm),
                              abi.dptr(bins) if self.nbins else None, C.byref(st)))
        return RunResult(self._grid_view(jm) if jm is not None else None, bins, st.to_dict())

    def run_moments(self, nphotons: int, seed: int) -> RunResult:
        """smcrt_run_moments (a context made with variance=True): the run of
        run(nphotons, seed) plus jmean2, per voxel the sum over packets of the
        packet's own path length there squared.  The per-packet variance of voxel v
        is jmean2/N - (jmean/N)^2, the standard error of jmean/N its root over N."""
        jm = np.empty(self.ncell, dtype=np.float64)
        j2 = np.empty(self.ncell, dtype=np.float64)
        bins = np.zeros(max(self.nbins, 0), dtype=np.float64)
        st = abi.Stats()
        check(lib().smcrt_run_moments(self._ctx, int(nphotons), int(seed), abi.dptr(jm), abi.dptr(j2),
                                      abi.dptr(bins) if self.nbins else None, C.byref(st)))
        return RunResult(self._grid_view(jm), bins, st.to_dict(), self._grid_view(j2))

    def run_device_moments(self, first: int, count: int, seed: int, jmean_dev: int, jmean2_dev: int,
                           bins_dev: int | None, stats: bool = False) -> dict | None:
        """smcrt_run_device_moments: adds the tallies and the second moment of packets
        [first, first+count) into caller-owned device buffers."""
        st = abi.Stats() if stats else None
        check(lib().smcrt_run_device_moments(self._ctx, int(first), int(count), int(seed), C.c_void_p(jmean_dev),
                                             C.c_void_p(jmean2_dev), C.c_void_p(bins_dev) if bins_dev else None,
                                             C.byref(st) if st is not None else None))
        return st.to_dict() if st is not None else None

    def adjoint(self, nphotons: int, seed: int, w_dev: int, gbins_dev: int | None, region_group,
                ngroups: int) -> tuple[np.ndarray, dict]:
        """smcrt_adjoint: d/d(mua, mus, g) of each region group of
        L = sum_v w[v] jmean[v] + sum_b h[b] bins[b] for the packets of run(nphotons, seed).
        w_dev / gbins_dev: device pointers (FP32 voxel weights, FP64 bin weights or None).
        Returns (grad (3, ngroups): rows d/d mua, d/d mus, d/d g, summed over packets; stats)."""
        rg = np.ascontiguousarray(region_group, dtype=np.int32)
        if len(rg) != self.flat.nregions:
            raise ValueError("region_group needs one entry per region")
        out = np.zeros(3 * ngroups, dtype=np.float64)
        st = abi.Stats()
        check(lib().smcrt_adjoint(self._ctx, int(nphotons), int(seed), C.c_void_p(w_dev),
                                  C.c_void_p(gbins_dev) if gbins_dev else None, abi.i32ptr(rg), int(ngroups),
                                  abi.dptr(out), C.byref(st)))
        return out.reshape(3, ngroups), st.to_dict()

    def autotune(self, trial_packets: int = 200000, seed: int = 0) -> dict:
        """smcrt_autotune: times trial runs of each launch configuration (fluence-grid
        copies, detector-bin privatisation, the nearest-region cache, the shared
        fluence sub-box, the group order) and keeps the fastest for later runs."""
        t = abi.Tuning()
        check(lib().smcrt_autotune(self._ctx, int(trial_packets), int(seed), C.byref(t)))
        return {"tally_copies": t.tally_copies, "shared_bins": bool(t.shared_bins),
                "packets_per_s": t.packets_per_s, "trials": t.trials, "block_size": t.block_size,
                "slots_per_thread": t.slots_per_thread, "ctas_per_sm": t.ctas_per_sm,
                "nearest_cache": bool(t.nearest_cache), "shared_fluence": bool(t.shared_fluence),
                "group_order": int(t.group_order)}

    def run_device(self, first: int, count: int, seed: int, jmean_dev: int, bins_dev: int | None,
                   stats: bool = False) -> dict | None:
        """Adds the tallies of packets [first, first+count) into caller-owned device
        buffers (raw pointers, e.g. tensor.data_ptr()), asynchronously on the
        context stream; with stats=True it synchronises and returns counters."""
        st = abi.Stats() if stats else None
        check(lib().smcrt_run_device(self._ctx, int(first), int(count), int(seed), C.c_void_p(jmean_dev),
                                     C.c_void_p(bins_dev) if bins_dev else None,
                                     C.byref(st) if st is not None else None))
        return st.to_dict() if st is not None else None

    def replay(self, uniforms: np.ndarray, offsets: np.ndarray):
        """Runs packets from injected uniform streams; returns (RunResult, states)."""
        uniforms = np.ascontiguousarray(uniforms, dtype=np.float64)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        n = len(offsets) - 1
        jm = np.empty(self.ncell, dtype=np.float64)
        bins = np.zeros(max(self.nbins, 0), dtype=np.float64)
        states = np.zeros(max(n, 1), dtype=abi.PACKET_STATE_DTYPE)
        st = abi.Stats()
        check(lib().smcrt_replay(self._ctx, abi.dptr(uniforms), abi.i64ptr(offsets), n, abi.dptr(jm),
                                 abi.dptr(bins) if self.nbins else None, states.ctypes.data_as(C.c_void_p),
                                 C.byref(st)))
        return RunResult(self._grid_view(jm), bins, st.to_dict()), states[:n]


class Batch:
    """Many instances of one scene (smcrt_batch_*): shared geometry, grid, source and
    detectors; per-instance region optics, packet counts and seeds; one persistent
    launch.  Instance i runs the packets `Transport.run(nphotons[i], seeds[i])` would
    run with its optics."""

    def __init__(self, array, settings: Settings, ninst: int, *, kernel: str = "pathlength",
                 precision: str = "fp32", optics=None, timeout_ms: int = 0, instance: int = 0):
        self.settings = settings
        self.flat = array if isinstance(array, FlatScene) else FlatScene(array)
        self.grid = settings.grid_c()
        self.source = settings.source_c()
        dets = settings.detectors_c()
        self._dets = (abi.Detector * max(1, len(dets)))(*dets)
        o = abi.Options()
        o.kernel = KERNELS[kernel]
        o.precision = PRECISIONS[precision]
        o.timeout_ms = timeout_ms
        o.instance = instance
        self.options = o
        self.ninst = int(ninst)
        self._b = C.c_void_p()
        check(lib().smcrt_batch_create(self.flat.ptr(), C.byref(self.grid), C.byref(self.source), self._dets,
                                       len(dets), C.byref(o), self.ninst, C.byref(self._b)))
        g = settings.grid
        self.shape = (g.nxg, g.nyg, g.nzg)
        self.ncell = g.nxg * g.nyg * g.nzg
        self.nregions = self.flat.nregions
        self.nbins = sum((d.nbins + 1) ** (2 if d.type == "camera" else 1) for d in settings.detectors)
        if optics is not None:
            self.set_optics(optics)

    def set_optics(self, optics) -> None:
        """optics: (ninst, nregions, 4) array of (mus, mua, hgg, n) per instance and region."""
        a = np.ascontiguousarray(optics, dtype=np.float64).reshape(self.ninst, self.nregions, 4)
        check(lib().smcrt_batch_set_optics(self._b, a.ctypes.data_as(C.POINTER(abi.RegionOptics))))

    def launch(self, nphotons, seeds, use_graph: bool = False) -> None:
        n = np.ascontiguousarray(nphotons, dtype=np.int64).reshape(self.ninst)
        sd = np.ascontiguousarray(seeds, dtype=np.uint64).reshape(self.ninst)
        check(lib().smcrt_batch_launch(self._b, abi.i64ptr(n), sd.ctypes.data_as(C.POINTER(C.c_uint64)),
                                       int(bool(use_graph))))

    def wait(self, want_jmean: bool = True, jmean_out: np.ndarray | None = None):
        """(jmean (ninst, nxg, nyg, nzg) Fortran order per instance or None, bins (ninst, nbins),
        per-instance stats dicts, launch totals).  jmean_out: a flat float64 buffer of
        ninst * ncell (e.g. pinned) to copy the tallies into."""
        jm = None
        if want_jmean:
            jm = jmean_out if jmean_out is not None else np.empty(self.ninst * self.ncell, dtype=np.float64)
        bins = np.zeros(max(self.ninst * self.nbins, 1), dtype=np.float64)
        per = (abi.Stats * self.ninst)()
        tot = abi.Stats()
        check(lib().smcrt_batch_wait(self._b, abi.dptr(jm), abi.dptr(bins) if self.nbins else None, per,
                                     C.byref(tot)))
        if jm is not None:
            jm = jm.reshape((self.ninst,) + self.shape[::-1]).transpose(0, 3, 2, 1)
        return jm, bins[: self.ninst * self.nbins].reshape(self.ninst, self.nbins), \
            [per[i].to_dict() for i in range(self.ninst)], tot.to_dict()

    def run(self, nphotons, seeds, use_graph: bool = False, want_jmean: bool = True):
        self.launch(nphotons, seeds, use_graph)
        return self.wait(want_jmean)

    def device_tallies(self) -> tuple[int, int]:
        jm, bins = C.c_void_p(), C.c_void_p()
        check(lib().smcrt_batch_device_tallies(self._b, C.byref(jm), C.byref(bins)))
        return jm.value, bins.value

    @property
    def stream(self) -> int:
        return int(lib().smcrt_batch_stream(self._b))

    def close(self) -> None:
        if self._b:
            lib().smcrt_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_batched(transports: list, nphotons, seeds):
    """smcrt_run_batched over Transport contexts: one launch when their scenes share
    the geometry.  Returns a RunResult per context (stats: packets, rng_draws, nscatt)."""
    n = len(transports)
    nph = np.ascontiguousarray(nphotons, dtype=np.int64).reshape(n)
    sd = np.ascontiguousarray(seeds, dtype=np.uint64).reshape(n)
    ctxs = (C.c_void_p * n)(*[t._ctx.value for t in transports])
    jms = [np.empty(t.ncell, dtype=np.float64) for t in transports]
    bins = [np.zeros(max(t.nbins, 1), dtype=np.float64) for t in transports]
    jp = (C.POINTER(C.c_double) * n)(*[abi.dptr(a) for a in jms])
    bp = (C.POINTER(C.c_double) * n)(*[abi.dptr(b) for b in bins])
    st = (abi.Stats * n)()
    check(lib().smcrt_run_batched(C.cast(ctxs, C.POINTER(C.c_void_p)), n, abi.i64ptr(nph),
                                  sd.ctypes.data_as(C.POINTER(C.c_uint64)), jp, bp, st))
    return [RunResult(t._grid_view(j), b[: t.nbins], st[i].to_dict())
            for i, (t, j, b) in enumerate(zip(transports, jms, bins))]


# ---------------------------------------------------------------------- render
def _render_args(samples, extent):
    ns = np.ascontiguousarray([int(x) for x in samples], dtype=np.int32)
    ext = np.ascontiguousarray([float(x) for x in extent], dtype=np.float64)
    if ns.shape != (3,) or ext.shape != (3,):
        raise ValueError("render: samples and extent need 3 entries")
    return ns, ext


def render(array, samples, extent, precision: str = "fp64") -> np.ndarray:
    """render_sub (src/sdfs/sdf_base.f90:302-346) on the device: the minimum over
    regions of the signed distance on a samples[0] x samples[1] x samples[2] voxel
    grid spanning [-extent, extent] (voxel i at (i - nint(n/2)) * extent / nint(n/2)),
    FP32, shape `samples`, Fortran order."""
    flat = array if isinstance(array, FlatScene) else FlatScene(array)
    ns, ext = _render_args(samples, extent)
    img = np.empty(int(np.prod(ns, dtype=np.int64)), dtype=np.float32)
    check(lib().smcrt_render(flat.ptr(), PRECISIONS[precision], ns.ctypes.data_as(C.POINTER(C.c_int32)),
                             abi.dptr(ext), img.ctypes.data_as(C.POINTER(C.c_float))))
    return img.reshape(tuple(int(x) for x in ns), order="F")


def render_device(array, samples, extent, image_ptr: int, precision: str = "fp64", stream: int = 0) -> None:
    """The render into caller device memory (a float buffer of prod(samples)
    entries, Fortran order), asynchronously on `stream`."""
    flat = array if isinstance(array, FlatScene) else FlatScene(array)
    ns, ext = _render_args(samples, extent)
    check(lib().smcrt_render_device(flat.ptr(), PRECISIONS[precision], ns.ctypes.data_as(C.POINTER(C.c_int32)),
                                    abi.dptr(ext), C.c_void_p(image_ptr), C.c_void_p(stream or None)))


# ---------------------------------------------------------------------- probes
def eval_sdf(flat: FlatScene, pts: np.ndarray, precision: str = "fp32") -> np.ndarray:
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.empty((len(pts), flat.nregions), dtype=np.float64)
    check(lib().smcrt_eval_sdf(flat.ptr(), PRECISIONS[precision], abi.dptr(pts), len(pts), abi.dptr(out)))
    return out


def calc_normal(flat: FlatScene, region0: int, pts: np.ndarray, h: float = 1e-6) -> np.ndarray:
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.empty_like(pts)
    check(lib().smcrt_calc_normal(flat.ptr(), region0, h, abi.dptr(pts), len(pts), abi.dptr(out)))
    return out


def fresnel(I, N, n1, n2, precision: str = "fp32") -> np.ndarray:
    I = np.ascontiguousarray(I, dtype=np.float64).reshape(-1, 3)
    N = np.ascontiguousarray(N, dtype=np.float64).reshape(-1, 3)
    n1 = np.ascontiguousarray(np.broadcast_to(n1, len(I)), dtype=np.float64)
    n2 = np.ascontiguousarray(np.broadcast_to(n2, len(I)), dtype=np.float64)
    R = np.empty(len(I), dtype=np.float64)
    check(lib().smcrt_fresnel(PRECISIONS[precision], abi.dptr(I), abi.dptr(N), abi.dptr(n1), abi.dptr(n2),
                              len(I), abi.dptr(R)))
    return R


def reflect_refract(I, N, n1, n2, u, precision: str = "fp32"):
    I = np.ascontiguousarray(I, dtype=np.float64).reshape(-1, 3)
    N = np.ascontiguousarray(N, dtype=np.float64).reshape(-1, 3)
    n = len(I)
    n1 = np.ascontiguousarray(np.broadcast_to(n1, n), dtype=np.float64)
    n2 = np.ascontiguousarray(np.broadcast_to(n2, n), dtype=np.float64)
    u = np.ascontiguousarray(np.broadcast_to(u, n), dtype=np.float64)
    out = np.empty_like(I)
    refl = np.empty(n, dtype=np.int32)
    check(lib().smcrt_reflect_refract(PRECISIONS[precision], abi.dptr(I), abi.dptr(N), abi.dptr(n1),
                                      abi.dptr(n2), abi.dptr(u), n, abi.dptr(out), abi.i32ptr(refl)))
    return out, refl.astype(bool)


def scatter_dir(dirs, g, u, precision: str = "fp32") -> np.ndarray:
    dirs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
    n = len(dirs)
    g = np.ascontiguousarray(np.broadcast_to(g, n), dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(n, 3)
    out = np.empty_like(dirs)
    check(lib().smcrt_scatter_dir(PRECISIONS[precision], abi.dptr(dirs), abi.dptr(g), abi.dptr(u), n,
                                  abi.dptr(out)))
    return out


def emit(flat: FlatScene, settings: Settings, first: int, npk: int, seed: int, precision: str = "fp32"):
    """smcrt_emit: launch positions, directions (npk, 3) and 1-based launch layers of
    packets [first, first + npk) of stream `seed`, as the transport kernel emits them."""
    grid, src = settings.grid_c(), settings.source_c()
    pos = np.empty((npk, 3), dtype=np.float64)
    dirs = np.empty((npk, 3), dtype=np.float64)
    layer = np.empty(npk, dtype=np.int32)
    check(lib().smcrt_emit(flat.ptr(), C.byref(grid), C.byref(src), PRECISIONS[precision], int(first), int(npk),
                           int(seed), abi.dptr(pos), abi.dptr(dirs), abi.i32ptr(layer)))
    return pos, dirs, layer


def philox(key: np.ndarray, ctr: np.ndarray) -> np.ndarray:
    key = np.ascontiguousarray(key, dtype=np.uint32).reshape(-1, 2)
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
    out = np.empty_like(ctr)
    check(lib().smcrt_philox(abi.u32ptr(key), abi.u32ptr(ctr), len(ctr), abi.u32ptr(out)))
    return out
