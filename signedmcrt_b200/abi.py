"""ctypes mirror of include/smcrt.h (the C ABI of libsmcrt_b200.so).

Only plain C types cross this boundary; numpy arrays are passed as pointers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

ABI_VERSION = 5

# status
OK, ERR_ARG, ERR_SCENE, ERR_CUDA, ERR_DEVICE, ERR_TIMEOUT, ERR_NO_DEVICE = range(7)

# primitives (src/sdfs/sdfs.f90)
SPHERE, BOX, TORUS, CYLINDER, TRIPRISM, SEGMENT, CAPSULE, CONE, EGG, PLANE = range(1, 11)
# CSG ops (src/sdfs/sdfModifiers.f90:412-475)
OP_NONE, OP_UNION, OP_SMOOTH_UNION, OP_SUBTRACTION, OP_INTERSECTION = range(5)
# sources (src/photon.f90)
SRC_POINT, SRC_PENCIL, SRC_UNIFORM, SRC_CIRCULAR, SRC_ANNULUS, SRC_FOCUS = range(1, 7)
ANNULUS_TOPHAT, ANNULUS_GAUSSIAN = 0, 1
# detectors (src/detectors/detectors.f90)
DET_CIRCLE, DET_ANNULUS, DET_CAMERA = 1, 2, 3
# kernels / precision
KERNEL_PATHLENGTH, KERNEL_WEIGHT, KERNEL_TEST = 0, 1, 2
FP32, FP64 = 0, 1
# order of the action groups in the kernel's per-round packet list (options.group_order)
ORDER_WALK_LAST, ORDER_INTERACT_LAST = 1, 2

D3 = C.c_double * 3


class Prim(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nmods", C.c_int32),
                ("transform", (C.c_double * 3) * 4), ("params", C.c_double * 8),
                ("mods", C.c_int32 * 2), ("mod_params", (C.c_double * 3) * 2)]


class Region(C.Structure):
    _fields_ = [("first_prim", C.c_int32), ("nprims", C.c_int32), ("op", C.c_int32),
                ("layer_id", C.c_int32), ("k", C.c_double), ("mus", C.c_double),
                ("mua", C.c_double), ("hgg", C.c_double), ("n", C.c_double)]


class Scene(C.Structure):
    _fields_ = [("nregions", C.c_int32), ("nprims", C.c_int32),
                ("regions", C.POINTER(Region)), ("prims", C.POINTER(Prim))]


class Grid(C.Structure):
    _fields_ = [("nxg", C.c_int32), ("nyg", C.c_int32), ("nzg", C.c_int32), ("reserved", C.c_int32),
                ("xmax", C.c_double), ("ymax", C.c_double), ("zmax", C.c_double)]


class Source(C.Structure):
    _fields_ = [("kind", C.c_int32), ("annulus_type", C.c_int32), ("pos", D3), ("dir", D3),
                ("point1", D3), ("point2", D3), ("point3", D3), ("radius", C.c_double),
                ("radius_hi", C.c_double), ("beta", C.c_double), ("z_inset", C.c_double)]


class Detector(C.Structure):
    _fields_ = [("kind", C.c_int32), ("layer", C.c_int32), ("nbins", C.c_int32), ("reserved", C.c_int32),
                ("pos", D3), ("dir", D3), ("r1", C.c_double), ("r2", C.c_double),
                ("maxval", C.c_double), ("p2", D3), ("p3", D3)]


class Options(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("precision", C.c_int32), ("end_early", C.c_int32),
                ("block_size", C.c_int32), ("blocks_per_sm", C.c_int32), ("max_trace_steps", C.c_int32),
                ("eps", C.c_double), ("normal_h", C.c_double), ("instance", C.c_uint32),
                ("timeout_ms", C.c_int32), ("stream", C.c_void_p), ("private_stream", C.c_int32),
                ("tally_copies", C.c_int32), ("scene_memory", C.c_int32), ("variance", C.c_int32),
                ("nearest_cache", C.c_int32), ("shared_fluence", C.c_int32), ("group_order", C.c_int32),
                ("reserved", C.c_int32 * 3)]


class Stats(C.Structure):
    _fields_ = [("nscatt", C.c_double), ("packets", C.c_uint64), ("sdf_evals", C.c_uint64),
                ("voxel_segments", C.c_uint64), ("trace_steps", C.c_uint64), ("scatters", C.c_uint64),
                ("fresnel_events", C.c_uint64), ("reflections", C.c_uint64),
                ("kills_step_cap", C.c_uint64), ("kills_error", C.c_uint64), ("rng_draws", C.c_uint64),
                ("moments", C.c_double * 24), ("kernel_ms", C.c_double), ("device_status", C.c_int32),
                ("reserved", C.c_int32), ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("variance_overflows", C.c_uint64), ("reserved2", C.c_uint64 * 5)]

    def to_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_
             if name not in ("moments", "reserved", "reserved2")}
        d["moments"] = np.array(self.moments[:], dtype=np.float64)
        return d


class PacketState(C.Structure):
    _fields_ = [("pos", D3), ("dir", D3), ("weight", C.c_double), ("layer", C.c_int32),
                ("nscatt", C.c_int32), ("ndraws", C.c_int32), ("flags", C.c_int32)]


PACKET_STATE_DTYPE = np.dtype([("pos", "<f8", 3), ("dir", "<f8", 3), ("weight", "<f8"), ("layer", "<i4"),
                               ("nscatt", "<i4"), ("ndraws", "<i4"), ("flags", "<i4")])
assert PACKET_STATE_DTYPE.itemsize == C.sizeof(PacketState)


def dptr(a: np.ndarray | None):
    """double* of a C-contiguous float64 array (or NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def i64ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def u32ptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def i32ptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_int32))


MOD_NONE, MOD_ONION, MOD_REVOLUTION, MOD_EXTRUDE, MOD_ELONGATE, MOD_TWIST, MOD_BEND = range(7)


class RegionOptics(C.Structure):
    _fields_ = [("mus", C.c_double), ("mua", C.c_double), ("hgg", C.c_double), ("n", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("tally_copies", C.c_int32), ("shared_bins", C.c_int32), ("packets_per_s", C.c_double),
                ("trials", C.c_int32), ("block_size", C.c_int32), ("slots_per_thread", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("nearest_cache", C.c_int32), ("shared_fluence", C.c_int32),
                ("group_order", C.c_int32), ("reserved", C.c_int32)]


# Exported symbols of include/smcrt.h with their argtypes/restype.
SIGNATURES = {
    "smcrt_abi_version": ([], C.c_int32),
    "smcrt_last_error": ([], C.c_char_p),
    "smcrt_create": ([C.POINTER(Scene), C.POINTER(Grid), C.POINTER(Source), C.POINTER(Detector), C.c_int32,
                      C.POINTER(Options), C.POINTER(C.c_void_p)], C.c_int32),
    "smcrt_destroy": ([C.c_void_p], None),
    "smcrt_detector_bins": ([C.c_void_p], C.c_int64),
    "smcrt_run": ([C.c_void_p, C.c_int64, C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double),
                   C.POINTER(Stats)], C.c_int32),
    "smcrt_run_device": ([C.c_void_p, C.c_int64, C.c_int64, C.c_uint64, C.c_void_p, C.c_void_p,
                          C.POINTER(Stats)], C.c_int32),
    "smcrt_run_moments": ([C.c_void_p, C.c_int64, C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double),
                           C.POINTER(C.c_double), C.POINTER(Stats)], C.c_int32),
    "smcrt_run_device_moments": ([C.c_void_p, C.c_int64, C.c_int64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(Stats)], C.c_int32),
    "smcrt_replay": ([C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_int64, C.POINTER(C.c_double),
                      C.POINTER(C.c_double), C.c_void_p, C.POINTER(Stats)], C.c_int32),
    "smcrt_run_batched": ([C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_uint64),
                           C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.POINTER(C.c_double)), C.POINTER(Stats)],
                          C.c_int32),
    "smcrt_adjoint": ([C.c_void_p, C.c_int64, C.c_uint64, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.c_int32,
                       C.POINTER(C.c_double), C.POINTER(Stats)], C.c_int32),
    "smcrt_autotune": ([C.c_void_p, C.c_int64, C.c_uint64, C.POINTER(Tuning)], C.c_int32),
    "smcrt_batch_create": ([C.POINTER(Scene), C.POINTER(Grid), C.POINTER(Source), C.POINTER(Detector), C.c_int32,
                            C.POINTER(Options), C.c_int32, C.POINTER(C.c_void_p)], C.c_int32),
    "smcrt_batch_set_optics": ([C.c_void_p, C.POINTER(RegionOptics)], C.c_int32),
    "smcrt_batch_launch": ([C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_uint64), C.c_int32], C.c_int32),
    "smcrt_batch_wait": ([C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(Stats),
                          C.POINTER(Stats)], C.c_int32),
    "smcrt_batch_device_tallies": ([C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)], C.c_int32),
    "smcrt_batch_stream": ([C.c_void_p], C.c_int64),
    "smcrt_batch_destroy": ([C.c_void_p], None),
    "smcrt_run_device_static": ([C.POINTER(Scene), C.POINTER(Grid), C.POINTER(Source), C.POINTER(Detector),
                                 C.c_int32, C.POINTER(Options), C.c_int64, C.c_int64, C.c_uint64, C.c_void_p,
                                 C.c_void_p, C.POINTER(Stats)], C.c_int32),
    "smcrt_static_scratch_bytes": ([], C.c_int64),
    "smcrt_eval_sdf": ([C.POINTER(Scene), C.c_int32, C.POINTER(C.c_double), C.c_int64, C.POINTER(C.c_double)],
                       C.c_int32),
    "smcrt_calc_normal": ([C.POINTER(Scene), C.c_int32, C.c_double, C.POINTER(C.c_double), C.c_int64,
                           C.POINTER(C.c_double)], C.c_int32),
    "smcrt_render": ([C.POINTER(Scene), C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                      C.POINTER(C.c_float)], C.c_int32),
    "smcrt_render_device": ([C.POINTER(Scene), C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                             C.c_void_p, C.c_void_p], C.c_int32),
    "smcrt_fresnel": ([C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                       C.POINTER(C.c_double), C.c_int64, C.POINTER(C.c_double)], C.c_int32),
    "smcrt_reflect_refract": ([C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64, C.POINTER(C.c_double),
                               C.POINTER(C.c_int32)], C.c_int32),
    "smcrt_scatter_dir": ([C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                           C.c_int64, C.POINTER(C.c_double)], C.c_int32),
    "smcrt_emit": ([C.POINTER(Scene), C.POINTER(Grid), C.POINTER(Source), C.c_int32, C.c_int64, C.c_int64,
                    C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int32)], C.c_int32),
    "smcrt_philox": ([C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_int64, C.POINTER(C.c_uint32)], C.c_int32),
}


def bind(lib: C.CDLL, signatures: dict = SIGNATURES) -> C.CDLL:
    for name, (args, res) in signatures.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib
