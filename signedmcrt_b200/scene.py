"""SDF scene description mirroring signedMCRT's geometry types, flattened into
the C ABI's region/primitive tables.

Reference: src/sdfs/sdfs.f90 (primitives and their initialisers),
src/sdfs/sdf_base.f90 (sdf container, model), src/sdfs/sdfHelpers.f90
(transforms), src/opticalProps/opticalProperties.f90 (mono).  Transforms are
4x4 arrays in the reference's layout: M[i, j] is the Fortran M(i+1, j+1) and a
point transforms as the row vector [x, y, z, 1] @ M (src/vector_class.f90:292).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import abi

PI = 4.0 * math.atan(1.0)  # constants.f90:22


# ---------------------------------------------------------------- optics
@dataclass(frozen=True)
class Mono:
    """init_mono (opticalProperties.f90:107-125); kappa and albedo are derived
    by the library with the same rule (albedo = 1 when mua < 1e-9)."""
    mus: float
    mua: float
    hgg: float
    n: float

    @property
    def kappa(self) -> float:
        return self.mus + self.mua

    @property
    def albedo(self) -> float:
        return 1.0 if self.mua < 1e-9 else self.mus / self.kappa


def mono(mus: float, mua: float, hgg: float, n: float) -> Mono:
    return Mono(float(mus), float(mua), float(hgg), float(n))


# ---------------------------------------------------------------- transforms (sdfHelpers.f90)
def _cols(*cols) -> np.ndarray:
    """Builds M from its columns, as the reference's `r(:, j) = [...]`."""
    return np.array(cols, dtype=np.float64).T.copy()


def deg2rad(deg: float) -> float:
    return deg * PI / 180.0


def identity() -> np.ndarray:  # :142-152
    return np.eye(4)


def translate(o: Sequence[float]) -> np.ndarray:  # :169-182
    return _cols([1, 0, 0, o[0]], [0, 1, 0, o[1]], [0, 0, 1, o[2]], [0, 0, 0, 1])


def rotate_x(angle: float) -> np.ndarray:  # :23-41
    a = deg2rad(angle)
    c, s = math.cos(a), math.sin(a)
    return _cols([1, 0, 0, 0], [0, c, -s, 0], [0, s, c, 0], [0, 0, 0, 1])


def rotate_y(angle: float) -> np.ndarray:  # :43-62
    a = deg2rad(angle)
    c, s = math.cos(a), math.sin(a)
    return _cols([c, 0, s, 0], [0, 1, 0, 0], [-s, 0, c, 0], [0, 0, 0, 1])


def rotate_z(angle: float) -> np.ndarray:  # :64-83
    a = deg2rad(angle)
    c, s = math.cos(a), math.sin(a)
    return _cols([c, -s, 0, 0], [s, c, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1])


def rotmat(axis: Sequence[float], angle: float) -> np.ndarray:  # :85-112
    ax = np.asarray(axis, dtype=np.float64)
    x, y, z = ax / math.sqrt(float(ax @ ax))
    a = deg2rad(angle)
    s, c = math.sin(a), math.cos(a)
    oc = 1.0 - c
    return _cols([oc * x * x + c, oc * x * y - z * s, oc * z * x + y * s, 0.0],
                 [oc * x * y + z * s, oc * y * y + c, oc * y * z - x * s, 0.0],
                 [oc * z * x - y * s, oc * y * z + x * s, oc * z * z + c, 0.0],
                 [0.0, 0.0, 0.0, 1.0])


def skew_symm(a: Sequence[float]) -> np.ndarray:  # :155-167
    return _cols([0, -a[2], a[1], 0], [a[2], 0, -a[0], 0], [-a[1], a[0], 0, 0], [0, 0, 0, 0])


def rotation_align(a: Sequence[float], b: Sequence[float]) -> np.ndarray:  # :114-140
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    v = np.array([a[1] * b[2] - a[2] * b[1], -a[0] * b[2] + a[2] * b[0], a[0] * b[1] - a[1] * b[0]])
    c = float(a @ b)
    k = 1.0 / (1.0 + c)
    vx = skew_symm(v)
    return identity() + vx + (vx @ vx) * k


def invert(m: np.ndarray) -> np.ndarray:
    """4x4 inverse (mat_class.f90:154-207 computes it by cofactors)."""
    return np.linalg.inv(np.asarray(m, dtype=np.float64))


def apply(m: np.ndarray, p: Sequence[float]) -> np.ndarray:
    """pos .dot. M (vector_class.f90:292-304)."""
    p = np.asarray(p, dtype=np.float64)
    return p @ m[:3, :3] + m[3, :3]


# ---------------------------------------------------------------- primitives (sdfs.f90)
@dataclass
class Sdf:
    kind: int
    params: tuple
    opt: Mono
    layer: int
    transform: np.ndarray = field(default_factory=identity)
    mods: tuple = ()  # ((modifier kind, params), ...), innermost first


# ---------------------------------------------------------------- modifiers (sdfModifiers.f90:114-375)
# Each wraps an Sdf (a primitive, possibly already modified) and keeps its optics
# and layer, like the *_init functions; the modifier has no transform of its own.
MAX_MODIFIERS = 2


def _wrap(prim: Sdf, kind: int, params) -> Sdf:
    if len(prim.mods) >= MAX_MODIFIERS:
        raise ValueError(f"at most {MAX_MODIFIERS} modifiers per primitive")
    return Sdf(prim.kind, prim.params, prim.opt, prim.layer, prim.transform,
               prim.mods + ((kind, tuple(float(x) for x in params)),))


def onion(prim: Sdf, thickness: float) -> Sdf:  # onion_init, eval_onion
    return _wrap(prim, abi.MOD_ONION, (thickness,))


def revolution(prim: Sdf, o: float) -> Sdf:  # revolution_init, eval_revolution
    return _wrap(prim, abi.MOD_REVOLUTION, (o,))


def extrude(prim: Sdf, h: float) -> Sdf:  # extrude_init, eval_extrude
    return _wrap(prim, abi.MOD_EXTRUDE, (h,))


def elongate(prim: Sdf, size) -> Sdf:  # elongate_init, eval_elongate
    return _wrap(prim, abi.MOD_ELONGATE, tuple(size))


def twist(prim: Sdf, k: float) -> Sdf:
    """twist_init takes k as a default (single precision) real: k is rounded to FP32."""
    return _wrap(prim, abi.MOD_TWIST, (float(np.float32(k)),))


def bend(prim: Sdf, k: float) -> Sdf:  # bend_init, eval_bend
    return _wrap(prim, abi.MOD_BEND, (k,))


def _t(transform) -> np.ndarray:
    return identity() if transform is None else np.asarray(transform, dtype=np.float64)


def _v(a) -> tuple:
    return tuple(float(x) for x in a)


def sphere(radius, opt, layer, transform=None) -> Sdf:  # :463-492
    return Sdf(abi.SPHERE, (float(radius),), opt, layer, _t(transform))


def box(lengths, opt, layer, transform=None) -> Sdf:  # :433-461 (stores half lengths)
    return Sdf(abi.BOX, tuple(0.5 * float(x) for x in lengths), opt, layer, _t(transform))


def torus(oradius, iradius, opt, layer, transform=None) -> Sdf:  # :401-431
    return Sdf(abi.TORUS, (float(oradius), float(iradius)), opt, layer, _t(transform))


def cylinder(a, b, radius, opt, layer, transform=None) -> Sdf:  # :365-399
    return Sdf(abi.CYLINDER, _v(a) + _v(b) + (float(radius),), opt, layer, _t(transform))


def triprism(h1, h2, opt, layer, transform=None) -> Sdf:  # :295-325
    return Sdf(abi.TRIPRISM, (float(h1), float(h2)), opt, layer, _t(transform))


def segment(a, b, opt, layer, transform=None) -> Sdf:  # :158-191
    return Sdf(abi.SEGMENT, _v(a) + _v(b), opt, layer, _t(transform))


def capsule(a, b, r, opt, layer, transform=None) -> Sdf:  # :259-293
    return Sdf(abi.CAPSULE, _v(a) + _v(b) + (float(r),), opt, layer, _t(transform))


def cone(a, b, ra, rb, opt, layer, transform=None) -> Sdf:  # :327-363
    return Sdf(abi.CONE, _v(a) + _v(b) + (float(ra), float(rb)), opt, layer, _t(transform))


def egg(r1, r2, h, opt, layer, transform=None) -> Sdf:  # :193-227
    return Sdf(abi.EGG, (float(r1), float(r2), float(h)), opt, layer, _t(transform))


def plane(a, opt, layer, transform=None) -> Sdf:  # :229-257
    return Sdf(abi.PLANE, _v(a), opt, layer, _t(transform))


@dataclass
class Model:
    """model (sdf_base.f90:42-51, model_init :100-143): children folded with op;
    optics and layer come from the first child."""
    children: list
    op: int
    k: float = 0.0

    @property
    def opt(self) -> Mono:
        return self.children[0].opt

    @property
    def layer(self) -> int:
        return self.children[0].layer


def model(children, op: int, k: float | None = None) -> Model:
    if op not in (abi.OP_UNION, abi.OP_SMOOTH_UNION, abi.OP_SUBTRACTION, abi.OP_INTERSECTION):
        raise ValueError(f"unknown CSG op {op}")
    return Model(list(children), op, 0.0 if k is None else float(k))


union, smooth_union, subtraction, intersection = (abi.OP_UNION, abi.OP_SMOOTH_UNION,
                                                  abi.OP_SUBTRACTION, abi.OP_INTERSECTION)


# ---------------------------------------------------------------- flattening
class FlatScene:
    """The C-ABI region/primitive tables of an sdf array (array order kept)."""

    def __init__(self, array: Sequence):
        if len(array) == 0:
            raise ValueError("empty sdf array")
        prims, regions = [], []
        for ent in array:
            kids = ent.children if isinstance(ent, Model) else [ent]
            first = len(prims)
            for s in kids:
                p = abi.Prim()
                p.kind = s.kind
                m = np.asarray(s.transform, dtype=np.float64)
                for i in range(4):
                    for j in range(3):
                        p.transform[i][j] = float(m[i, j])
                for i, v in enumerate(s.params):
                    p.params[i] = v
                p.nmods = len(s.mods)
                for j, (mk, mp) in enumerate(s.mods):
                    p.mods[j] = mk
                    for i, v in enumerate(mp):
                        p.mod_params[j][i] = v
                prims.append(p)
            r = abi.Region()
            r.first_prim = first
            r.nprims = len(kids)
            r.op = ent.op if isinstance(ent, Model) else abi.OP_NONE
            r.layer_id = int(ent.layer)
            r.k = ent.k if isinstance(ent, Model) else 0.0
            o = ent.opt
            r.mus, r.mua, r.hgg, r.n = o.mus, o.mua, o.hgg, o.n
            regions.append(r)
        self.array = list(array)
        self._prims = (abi.Prim * len(prims))(*prims)
        self._regions = (abi.Region * len(regions))(*regions)
        self.c = abi.Scene(len(regions), len(prims), self._regions, self._prims)

    @property
    def nregions(self) -> int:
        return self.c.nregions

    @property
    def nprims(self) -> int:
        return self.c.nprims

    def ptr(self):
        return C.byref(self.c)

    def optics(self) -> list[Mono]:
        return [ent.opt for ent in self.array]
