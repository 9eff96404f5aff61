"""TOML input parsing, mirroring signedMCRT's parse_params.

Reference: src/parse/parse.f90:19-215, src/parse/parse_source.f90:17-201,
src/parse/parse_detectors.f90:17-246, src/parse/parse_helpers.f90:15-53,
src/parse/parse_spectrum.f90.  Defaults and error messages follow those files.
Differences (documented): a [source] `direction` given as a 3-vector is used as
the direction (the reference returns from parse_source early in that case,
parse_source.f90:99-108, leaving the emitter unset); the optional [source]
`z_inset` (default 1e-8, the value hard-coded at photon.f90:686) sets how far
below the grid top the annulus and focus sources start.
"""
from __future__ import annotations

import math
import tomllib
from dataclasses import dataclass, field
from pathlib import Path

from . import abi


class ConfigError(ValueError):
    pass


@dataclass
class SourceCfg:
    name: str = "point"
    nphotons: int = 1000000
    position: tuple = (0.0, 0.0, 0.0)
    direction: tuple = (0.0, 0.0, 0.0)
    point1: tuple = (-1.0, -1.0, 1.0)
    point2: tuple = (2.0, 0.0, 0.0)
    point3: tuple = (0.0, 2.0, 0.0)
    radius: float = 0.5
    beta: float = 5.0
    radius_hi: float = 0.6
    annulus_type: str = "gaussian"
    spectrum_type: str = "constant"
    wavelength: float = 500.0
    z_inset: float = 1e-8


@dataclass
class GridCfg:
    nxg: int = 200
    nyg: int = 200
    nzg: int = 200
    xmax: float = 1.0
    ymax: float = 1.0
    zmax: float = 1.0
    units: str = "cm"


@dataclass
class GeometryCfg:
    geom_name: str = "sphere"
    tau: float = 10.0
    num_spheres: int = 10
    musb: float = 0.0
    muab: float = 0.01
    musc: float = 0.0
    muac: float = 0.01
    hgg: float = 0.7


@dataclass
class DetectorCfg:
    type: str
    position: tuple = (0.0, 0.0, 0.0)
    direction: tuple = (0.0, 0.0, -1.0)
    layer: int = 1
    radius1: float = 0.0
    radius2: float = 0.0
    nbins: int = 100
    maxval: float = 100.0
    trackHistory: bool = False
    p1: tuple = (-1.0, -1.0, -1.0)
    p2: tuple = (2.0, 0.0, 0.0)
    p3: tuple = (0.0, 2.0, 0.0)


@dataclass
class OutputCfg:
    fluence: str = "fluence.nrrd"
    absorb: str = "absorb.nrrd"
    render: str = "geom_render.nrrd"
    render_geom: bool = False
    render_size: tuple = (200, 200, 200)
    overwrite: bool = False


@dataclass
class SimulationCfg:
    iseed: int = 123456789
    tev: bool = False
    absorb: bool = False
    load_checkpoint: bool = False
    checkpoint_file: str = "check.ckpt"
    checkpoint_every_n: int = 1000000


@dataclass
class Settings:
    source: SourceCfg = field(default_factory=SourceCfg)
    grid: GridCfg = field(default_factory=GridCfg)
    geometry: GeometryCfg = field(default_factory=GeometryCfg)
    detectors: list = field(default_factory=list)
    output: OutputCfg = field(default_factory=OutputCfg)
    simulation: SimulationCfg = field(default_factory=SimulationCfg)
    dict: dict = field(default_factory=dict)  # metadata written to output headers

    # ---- C-ABI views
    def grid_c(self) -> abi.Grid:
        g = self.grid
        return abi.Grid(g.nxg, g.nyg, g.nzg, 0, g.xmax, g.ymax, g.zmax)

    def source_c(self) -> abi.Source:
        s = self.source
        kinds = {"point": abi.SRC_POINT, "pencil": abi.SRC_PENCIL, "uniform": abi.SRC_UNIFORM,
                 "circular": abi.SRC_CIRCULAR, "annulus": abi.SRC_ANNULUS, "focus": abi.SRC_FOCUS}
        if s.name not in kinds:
            if s.name in ("slm", "dslit", "aperture"):
                raise ConfigError(f"source '{s.name}' (phase/diffraction source) is not supported by this transport")
            raise ConfigError("No such source!")  # photon.f90:153
        c = abi.Source()
        c.kind = kinds[s.name]
        if s.annulus_type not in ("tophat", "gaussian"):
            if s.name == "annulus":
                raise ConfigError("No such beam type!")  # photon.f90:675
        c.annulus_type = abi.ANNULUS_TOPHAT if s.annulus_type == "tophat" else abi.ANNULUS_GAUSSIAN
        for name in ("pos", "dir", "point1", "point2", "point3"):
            src = {"pos": s.position, "dir": s.direction}.get(name, getattr(s, name, None))
            for i in range(3):
                getattr(c, name)[i] = float(src[i])
        c.radius, c.radius_hi, c.beta, c.z_inset = s.radius, s.radius_hi, s.beta, s.z_inset
        return c

    def detectors_c(self) -> list:
        out = []
        for d in self.detectors:
            c = abi.Detector()
            c.kind = {"circle": abi.DET_CIRCLE, "annulus": abi.DET_ANNULUS, "camera": abi.DET_CAMERA}[d.type]
            c.layer, c.nbins, c.maxval = d.layer, d.nbins, d.maxval
            if d.type == "camera":
                for i in range(3):
                    c.pos[i], c.p2[i], c.p3[i] = d.p1[i], d.p2[i], d.p3[i]
            else:
                dirv = d.direction
                if d.type == "circle":  # handle_circle_dect normalises (parse_detectors.f90:180)
                    n = math.sqrt(sum(x * x for x in dirv))
                    dirv = tuple(x / n for x in dirv)
                for i in range(3):
                    c.pos[i], c.dir[i] = d.position[i], dirv[i]
                c.r1 = d.radius1
                c.r2 = d.radius2
            out.append(c)
        return out


_CARDINAL = {"x": (1.0, 0.0, 0.0), "-x": (-1.0, 0.0, 0.0), "y": (0.0, 1.0, 0.0), "-y": (0.0, -1.0, 0.0),
             "z": (0.0, 0.0, 1.0), "-z": (0.0, 0.0, -1.0)}


def _vec(tbl: dict, key: str, default=None, what: str = "") -> tuple:
    """get_vector (parse_helpers.f90:15-53)."""
    v = tbl.get(key)
    if v is None:
        if default is not None:
            return tuple(float(x) for x in default)
        raise ConfigError(f"Expected vector of size 3 for {key}")
    if not isinstance(v, list) or len(v) != 3:
        raise ConfigError(f"Expected vector of size 3 for {key}")
    return tuple(float(x) for x in v)


def parse_source(table: dict, st: Settings) -> None:
    """parse_source.f90:17-201."""
    child = table.get("source")
    if child is None:
        raise ConfigError("Simulation needs Source table")
    s = st.source
    s.name = child.get("name", "point")
    s.nphotons = int(child.get("nphotons", 1000000))
    if s.name != "uniform":
        s.position = _vec(child, "position")
    d = child.get("direction")
    if isinstance(d, list):
        s.direction = _vec(child, "direction")
    elif isinstance(d, str):
        if d not in _CARDINAL:
            raise ConfigError("Direction needs a cardinal direction i.e x, y, or z")
        s.direction = _CARDINAL[d]
    elif s.name != "point":
        raise ConfigError("Need to specify direction for source type!")
    for i, key in enumerate(("point1", "point2", "point3")):
        if key in child:
            v = child[key]
            if not isinstance(v, list) or len(v) < 3:
                raise ConfigError("Need a matrix row for points")
            setattr(s, key, tuple(float(x) for x in v[:3]))
            for ax, val in zip("xyz", v[:3]):
                st.dict[f"pos{i + 1}%{ax}"] = float(val)
        elif s.name == "uniform":
            raise ConfigError(f"Uniform source requires {key} variable")
    s.radius = float(child.get("radius", 0.5))
    s.beta = float(child.get("beta", 5.0))
    s.radius_hi = float(child.get("radius_hi", 0.6))
    s.annulus_type = child.get("annulus_type", "gaussian")
    s.z_inset = float(child.get("z_inset", 1e-8))
    s.spectrum_type = child.get("spectrum_type", "constant")
    s.wavelength = float(child.get("wavelength", 500.0))
    if s.spectrum_type not in ("constant", "1D", "2D"):
        raise ConfigError("Invalid spectrum type")
    st.dict.update(radius=s.radius, beta=s.beta, rhi=s.radius_hi, annulus_type=s.annulus_type)


def parse_grid(table: dict, st: Settings) -> None:
    """parse.f90:66-101."""
    child = table.get("grid")
    if child is None:
        raise ConfigError("Need grid table in input param file")
    g = st.grid
    g.nxg, g.nyg, g.nzg = (int(child.get(k, 200)) for k in ("nxg", "nyg", "nzg"))
    g.xmax, g.ymax, g.zmax = (float(child.get(k, 1.0)) for k in ("xmax", "ymax", "zmax"))
    g.units = child.get("units", "cm")
    st.dict["units"] = g.units


def parse_geometry(table: dict, st: Settings) -> None:
    """parse.f90:103-143."""
    child = table.get("geometry")
    if child is None:
        raise ConfigError("Need geometry table in input param file")
    g = st.geometry
    g.geom_name = child.get("geom_name", "sphere")
    g.tau = float(child.get("tau", 10.0))
    g.num_spheres = int(child.get("num_spheres", 10))
    g.musb = float(child.get("musb", 0.0))
    g.muab = float(child.get("muab", 0.01))
    g.musc = float(child.get("musc", 0.0))
    g.muac = float(child.get("muac", 0.01))
    g.hgg = float(child.get("hgg", 0.7))
    st.dict.update(tau=g.tau, num_spheres=g.num_spheres, musb=g.musb, muab=g.muab, musc=g.musc,
                   muac=g.muac, hgg=g.hgg)


def parse_detectors(table: dict, st: Settings) -> None:
    """parse_detectors.f90:17-114 (circles, then annuli, then cameras, as the reference orders them)."""
    arr = table.get("detectors", [])
    circ, ann, cam = [], [], []
    for child in arr:
        t = child.get("type")
        if t not in ("circle", "annulus", "camera"):
            raise ConfigError("Invalid detector type. Valid types are [circle, annulus, camera]")
        common = dict(layer=int(child.get("layer", 1)), nbins=int(child.get("nbins", 100)),
                      maxval=float(child.get("maxval", 100.0)), trackHistory=bool(child.get("trackHistory", False)))
        if t == "camera":
            cam.append(DetectorCfg("camera", p1=_vec(child, "p1", (-1.0, -1.0, -1.0)),
                                   p2=_vec(child, "p2", (2.0, 0.0, 0.0)), p3=_vec(child, "p3", (0.0, 2.0, 0.0)),
                                   **common))
        elif t == "circle":
            circ.append(DetectorCfg("circle", position=_vec(child, "position"),
                                    direction=_vec(child, "direction", (0.0, 0.0, -1.0)),
                                    radius1=float(child["radius1"]), **common))
        else:
            r1, r2 = float(child["radius1"]), float(child["radius2"])
            if r2 <= r1:
                raise ConfigError(f"Radii are invalid: expected radius2 ({r2}) > radius 1 ({r1})")
            ann.append(DetectorCfg("annulus", position=_vec(child, "position"),
                                   direction=_vec(child, "direction", (0.0, 0.0, -1.0)), radius1=r1, radius2=r2,
                                   **common))
        if common["trackHistory"]:
            raise ConfigError("Track history currently incompatable with OpenMP!")
    st.detectors = circ + ann + cam


def parse_output(table: dict, st: Settings) -> None:
    """parse.f90:145-186."""
    child = table.get("output")
    if child is None:
        raise ConfigError("Need output table in input param file")
    o = st.output
    o.fluence = child.get("fluence", "fluence.nrrd")
    o.absorb = child.get("absorb", "absorb.nrrd")
    o.render = child.get("render", "geom_render.nrrd")
    o.render_geom = bool(child.get("render_geom", False))
    rs = child.get("render_size")
    if rs is not None:
        if len(rs) < 3:
            raise ConfigError("Need a vector of size 3 for render_size.")
        o.render_size = tuple(int(x) for x in rs[:3])
    o.overwrite = bool(child.get("overwrite", False))


def parse_simulation(table: dict, st: Settings) -> None:
    """parse.f90:188-215."""
    child = table.get("simulation")
    if child is None:
        raise ConfigError("Need simulation table in input param file")
    s = st.simulation
    s.iseed = int(child.get("iseed", 123456789))
    s.tev = bool(child.get("tev", False))
    s.absorb = bool(child.get("absorb", False))
    s.load_checkpoint = bool(child.get("load_checkpoint", False))
    s.checkpoint_file = child.get("checkpoint_file", "check.ckpt")
    s.checkpoint_every_n = int(child.get("checkpoint_every_n", 1000000))


def parse_params(filename: str | Path) -> Settings:
    """Entry point (parse.f90:19-63): parses every table in the reference's order."""
    with open(filename, "rb") as f:
        try:
            table = tomllib.load(f)
        except tomllib.TOMLDecodeError as e:
            raise ConfigError(f"{filename}: {e}") from e
    return parse_table(table)


def parse_table(table: dict) -> Settings:
    st = Settings()
    parse_source(table, st)
    parse_grid(table, st)
    parse_geometry(table, st)
    parse_detectors(table, st)
    parse_output(table, st)
    parse_simulation(table, st)
    return st
