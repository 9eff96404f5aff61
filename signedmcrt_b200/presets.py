"""Geometry presets selected by [geometry] geom_name, mirroring
setup_simulation (src/setup.f90:14-54) and src/setupGeometry.f90, plus the
synthetic benchmark scenes `box_slab`, `sphere_water` and `layered_vessels`
added in the same style (array order = priority at crossings).
"""
from __future__ import annotations

import math

import numpy as np

from . import scene as S
from .config import ConfigError, Settings

AMBIENT = S.mono(0.0, 0.0, 0.0, 1.0)


def setup_scat_test(tau: float) -> list:
    """setupGeometry.f90:221-247: sphere r=1 (mus=tau, albedo 1) inside a 2 cm box."""
    return [S.sphere(1.0, S.mono(tau, 0.0, 0.0, 1.0), 1),
            S.box((2.0, 2.0, 2.0), S.mono(0.0, 0.0, 0.0, 1.0), 2)]


def setup_scat_test2(tau: float, hgg: float) -> list:
    """setupGeometry.f90:249-274: a 200 cm box, mus=tau, mua=1e-17."""
    return [S.box((200.0, 200.0, 200.0), S.mono(tau, 1e-17, hgg, 1.0), 2)]


def setup_sphere() -> list:
    """setupGeometry.f90:147-175 ("aptran"): sphere r=0.5 (n=1.33) in a 2 cm box in an absorbing shell."""
    return [S.sphere(0.5, S.mono(0.0, 1e-17, 0.0, 1.33), 1, transform=S.invert(S.translate((0.0, 0.0, 0.0)))),
            S.box((2.0, 2.0, 2.0), S.mono(0.0, 1e-17, 0.0, 1.0), 2),
            S.box((2.01, 2.01, 2.01), S.mono(0.0, 10000000.0, 0.0, 1.0), 3)]


def setup_omg_sdf() -> list:
    """setupGeometry.f90:276-359: the letters OMG (torus + 9 cylinders, smooth union k=0.09) in a 2 cm box."""
    o1 = S.mono(10.0, 0.16, 0.0, 2.65)
    L = 1
    c = [S.torus(0.2, 0.05, o1, L, transform=S.invert(S.translate((0.0, 0.0, -0.7))))]
    c.append(S.cylinder((-.25, 0, -.25), (-.25, 0, .25), .05, o1, L, transform=S.invert(S.rotate_y(90.0))))
    for a, b in [((-.25, 0, -.25), (.25, 0, 0)), ((.25, 0, 0), (-.25, 0, .25)), ((-.25, 0, .25), (.25, 0, .25)),
                 ((-.25, 0, .5), (.25, 0, .5)), ((-.25, 0, .5), (-.25, 0, .75)), ((.25, 0, .5), (.25, 0, .75)),
                 ((.25, 0, .75), (0, 0, .75)), ((0, 0, .625), (0, 0, .75))]:
        c.append(S.cylinder(a, b, .05, o1, L))
    return [S.model(c, S.smooth_union, 0.09), S.box((2.0, 2.0, 2.0), S.mono(0.0, 0.0, 0.0, 1.0), 2)]


def setup_egg() -> list:
    """setupGeometry.f90:10-61 ("test_egg"): a sphere yolk (r 1.5), the albumen as a
    revolved egg and the shell as the onion of a revolved egg, in a 40 cm box."""
    r1 = 3.0
    r2 = 3.0 * math.sqrt(2.0 - math.sqrt(2.0))
    h = r2
    shell = S.onion(S.revolution(S.egg(r1, r2, h, S.mono(100.0, 10.0, 0.0, 1.37), 2), 0.2), 0.2)
    albumen = S.revolution(S.egg(r1 - 0.2, r2, h, S.mono(1.0, 0.0, 0.0, 1.37), 3), 0.2)
    yolk = S.sphere(1.5, S.mono(10.0, 1.0, 0.9, 1.37), 1)
    bbox = S.box((20.001, 20.001, 20.001), S.mono(0.0, 0.0, 0.0, 1.0), 4)
    return [yolk, albumen, shell, bbox]


def setup_sphere_scene(num_spheres: int, seed: int) -> list:
    """setupGeometry.f90:62-106: random non-scattering spheres in a 2 cm box.  The
    reference draws radii/positions from the gfortran stream; here from a seeded
    numpy generator (same distributions)."""
    rng = np.random.default_rng(seed)
    o1 = S.mono(0.0, 0.0, 0.9, 1.37)
    arr = []
    for i in range(num_spheres):
        r = 0.001 + rng.random() * (0.25 - 0.001)
        pos = [-1 + r + rng.random() * (2 - 2 * r) for _ in range(3)]
        arr.append(S.sphere(r, o1, i + 1, transform=S.invert(S.translate(pos))))
    arr.append(S.box((2.0, 2.0, 2.0), S.mono(1e-17, 1e-17, 0.0, 1.0), num_spheres + 1))
    return arr


# ---------------------------------------------------------------- benchmark scenes
def box_slab(mua=0.1, mus=10.0, g=0.9, n=1.38, half=1.0) -> list:
    """Plain method, small: 2x2x2 cm box (mua 0.1, mus 10, g 0.9, n 1.38) in air;
    the ambient box is 1e-3 larger than the grid so exiting packets end on it."""
    return [S.box((2 * half, 2 * half, 2 * half), S.mono(mus, mua, g, n), 1),
            S.box((2 * half + 0.002,) * 3, AMBIENT, 2)]


def sphere_water() -> list:
    """Curved-surface refraction: sphere r=1 (mua .05, mus 50, g .85, n 1.45) centred in
    a 4x4x4 cm water box (mua .01, mus .001, g 0, n 1.33), in air."""
    return [S.sphere(1.0, S.mono(50.0, 0.05, 0.85, 1.45), 1),
            S.box((4.0, 4.0, 4.0), S.mono(0.001, 0.01, 0.0, 1.33), 2),
            S.box((4.004, 4.004, 4.004), AMBIENT, 3)]


LAYER_THICK = (0.01, 0.2, 1.0)
LAYER_OPT = ((100.0, 1.0, 0.8, 1.4), (50.0, 0.3, 0.9, 1.38), (30.0, 0.1, 0.9, 1.36))  # (mus, mua, g, n)
VESSEL_SEED = 20231203


def vessel_layout(seed: int = VESSEL_SEED, n: int = 4):
    """Depths U(0.1, 0.5) cm and lateral offsets U(-0.5, 0.5) cm of the 4 vessels."""
    rng = np.random.default_rng(seed)
    depth = 0.1 + 0.4 * rng.random(n)
    yoff = -0.5 + rng.random(n)
    return depth, yoff


def layered_vessels(optics=None, seed: int = VESSEL_SEED) -> list:
    """Layered tissue with vessels: 3 planar layers 0.01/0.2/1.0 cm (lateral half-width
    1 cm) and 4 capsule vessels r=0.05 along x at seeded depths 0.1-0.5 cm (mua 5,
    mus 50, g 0.9, n of the host layer).  The top surface is z = +0.605.
    `optics` optionally overrides the 5 tissue regions [(mus, mua, g, n)] x
    (vessel, layer1, layer2, layer3, ambient)."""
    top = 0.5 * sum(LAYER_THICK)
    depth, yoff = vessel_layout(seed)
    lay = list(LAYER_OPT)
    ves = (50.0, 5.0, 0.9)
    amb = (0.0, 0.0, 0.0, 1.0)
    if optics is not None:
        ves = tuple(optics[0][:3])
        lay = [tuple(o) for o in optics[1:4]]
        amb = tuple(optics[4])
    arr = []
    bounds = np.cumsum((0.0,) + LAYER_THICK)
    for i in range(4):
        host = int(np.searchsorted(bounds, depth[i], side="right") - 1)
        zc = top - depth[i]
        arr.append(S.capsule((-0.9, yoff[i], zc), (0.9, yoff[i], zc), 0.05,
                             S.mono(ves[0], ves[1], ves[2], lay[host][3]), i + 1))
    z = top
    for k, t in enumerate(LAYER_THICK):
        zc = z - 0.5 * t
        mus, mua, g, n = lay[k]
        arr.append(S.box((2.0, 2.0, t), S.mono(mus, mua, g, n), 5 + k,
                         transform=S.invert(S.translate((0.0, 0.0, zc)))))
        z -= t
    arr.append(S.box((2.002, 2.002, 2 * top + 0.002), S.mono(*amb), 8))
    return arr


def setup_simulation(st: Settings) -> list:
    """The geom_name switch of src/setup.f90:33-52 (plus the benchmark scenes)."""
    g = st.geometry
    name = g.geom_name
    if name == "scat_test":
        return setup_scat_test(g.tau)
    if name == "scat_test2":
        return setup_scat_test2(g.tau, g.hgg)
    if name == "aptran":
        return setup_sphere()
    if name == "omg":
        return setup_omg_sdf()
    if name == "sphere_scene":
        return setup_sphere_scene(g.num_spheres, st.simulation.iseed)
    if name == "box_slab":
        return box_slab()
    if name == "sphere_water":
        return sphere_water()
    if name == "layered_vessels":
        return layered_vessels()
    if name == "test_egg":
        return setup_egg()
    if name in ("logo", "vessels"):
        raise ConfigError(f"preset '{name}' needs geometry this transport does not model "
                          "(an svg include or external vessel files)")
    raise ConfigError("no such routine")  # setup.f90:51


# ---------------------------------------------------------------- benchmark configurations
def benchmark_settings(name: str) -> Settings:
    """Settings of the synthetic benchmark configurations (scene, grid, source,
    detectors, packet count, seed)."""
    from .config import DetectorCfg
    st = Settings()
    st.output.overwrite = True
    if name == "box_slab":
        st.geometry.geom_name = "box_slab"
        st.grid.nxg = st.grid.nyg = st.grid.nzg = 100
        st.grid.xmax = st.grid.ymax = st.grid.zmax = 1.0
        st.source.name = "pencil"
        st.source.position = (0.0, 0.0, 1.0 - 1e-5)
        st.source.direction = (0.0, 0.0, -1.0)
        st.source.nphotons = 1000000
        st.simulation.iseed = 1
    elif name == "sphere_water":
        st.geometry.geom_name = "sphere_water"
        st.grid.nxg = st.grid.nyg = st.grid.nzg = 200
        st.grid.xmax = st.grid.ymax = st.grid.zmax = 2.0
        st.source.name = "annulus"
        st.source.annulus_type = "tophat"
        st.source.radius, st.source.radius_hi, st.source.beta = 0.0, 0.5, 0.0
        st.source.z_inset = 1e-5
        st.source.direction = (0.0, 0.0, -1.0)
        st.source.nphotons = 100000000
        st.simulation.iseed = 2
    elif name == "layered_vessels":
        top = 0.5 * sum(LAYER_THICK)
        st.geometry.geom_name = "layered_vessels"
        st.grid.nxg = st.grid.nyg = st.grid.nzg = 150
        st.grid.xmax = st.grid.ymax = 1.0
        st.grid.zmax = top
        st.source.name = "pencil"
        st.source.position = (0.0, 0.0, top - 1e-5)
        st.source.direction = (0.0, 0.0, -1.0)
        st.source.nphotons = 100000000
        st.simulation.iseed = 3
        st.detectors = [DetectorCfg("annulus", position=(0.0, 0.0, top), direction=(0.0, 0.0, 1.0), layer=8,
                                    radius1=0.1 * k, radius2=0.1 * (k + 1), nbins=10, maxval=1.0)
                        for k in range(10)]
    elif name == "sphere_scene":
        sphere_scene_settings(st)
    else:
        raise ConfigError(f"unknown benchmark configuration {name}")
    return st


def sphere_scene_settings(st: Settings | None = None, num_spheres: int = 40) -> Settings:
    """The reference's res/sphere.toml (the input of its runtime-vs-number-of-SDFs
    harness, tools/run_sphere_scene.py): `num_spheres` random spheres (n 1.37, no
    scattering) in a 2 cm box, a uniform source over the top face going -z, a 200^3
    grid, 1e6 packets, iseed 123456789."""
    st = st if st is not None else Settings()
    st.output.overwrite = True
    st.geometry.geom_name = "sphere_scene"
    st.geometry.num_spheres = int(num_spheres)
    st.grid.nxg = st.grid.nyg = st.grid.nzg = 200
    st.grid.xmax = st.grid.ymax = st.grid.zmax = 1.0
    st.source.name = "uniform"
    st.source.direction = (0.0, 0.0, -1.0)
    st.source.point1 = (-1.0, -1.0, 0.9999999)
    st.source.point2 = (2.0, 0.0, 0.0)
    st.source.point3 = (0.0, 2.0, 0.0)
    st.source.nphotons = 1000000
    st.simulation.iseed = 123456789
    return st


BATCH_SEED = 20240256


def batch_instances(ninst: int = 256, seed: int = BATCH_SEED, scale: float = 1.0):
    """The batched configuration: `ninst` instances of the box_slab geometry on a
    64^3 grid, each with mu_a ~ U(0.01, 1), mu_s ~ U(1, 100), g ~ U(0.7, 0.95),
    n ~ U(1.33, 1.45) for the box (the ambient region keeps AMBIENT) and
    round(10^U(4, 6) * scale) packets, drawn from numpy's PCG64 with `seed`;
    instance i uses packet stream seed + i.  Returns (settings, optics (ninst, 2, 4)
    as (mus, mua, hgg, n), packet counts, stream seeds)."""
    import numpy as np
    st = benchmark_settings("box_slab")
    st.grid.nxg = st.grid.nyg = st.grid.nzg = 64
    rng = np.random.default_rng(seed)
    mua = rng.uniform(0.01, 1.0, ninst)
    mus = rng.uniform(1.0, 100.0, ninst)
    g = rng.uniform(0.7, 0.95, ninst)
    n = rng.uniform(1.33, 1.45, ninst)
    counts = np.maximum(1, np.round(10.0 ** rng.uniform(4.0, 6.0, ninst) * scale)).astype(np.int64)
    optics = np.zeros((ninst, 2, 4))
    optics[:, 0] = np.stack([mus, mua, g, n], axis=1)
    optics[:, 1] = (AMBIENT.mus, AMBIENT.mua, AMBIENT.hgg, AMBIENT.n)
    seeds = (seed + np.arange(ninst)).astype(np.uint64)
    return st, optics, counts, seeds
