"""Pins the CPU oracle against the known answers of signedMCRT's own tests
(tests/reference_kats.py) before it is used as the checker of the GPU path."""
import math

import numpy as np
import pytest

from signedmcrt_b200 import abi, presets as P, scene as S
from signedmcrt_b200.config import parse_table
from tests import reference_kats as K

EPS64 = np.finfo(np.float64).eps
OPT0 = S.mono(0.0, 0.0, 0.0, 0.0)


def make_prim(name, args):
    return getattr(S, name)(**args, opt=OPT0, layer=1)


@pytest.mark.parametrize("name,args,cases", K.SDF_KATS, ids=[k[0] for k in K.SDF_KATS])
def test_sdf_primitives_fp64(oracle, name, args, cases):
    flat = S.FlatScene([make_prim(name, args)])
    pts = np.array([c[0] for c in cases], dtype=np.float64)
    got = oracle.eval_sdf(flat, pts)[:, 0]
    for (p, want, thr), g in zip(cases, got):
        assert abs(g - want) <= (thr if thr is not None else EPS64), (name, p, g, want)


@pytest.mark.parametrize("name,args,cases", K.SDF_KATS, ids=[k[0] for k in K.SDF_KATS])
def test_sdf_primitives_fp32_within_1e5(oracle, name, args, cases):
    """The FP32 evaluation of the same primitives stays within 1e-5 (scale 1)."""
    flat = S.FlatScene([make_prim(name, args)])
    rng = np.random.default_rng(1)
    pts = np.concatenate([np.array([c[0] for c in cases], dtype=np.float64), rng.uniform(-3, 3, (200, 3))])
    d64 = oracle.eval_sdf(flat, pts, "fp64")[:, 0]
    d32 = oracle.eval_sdf(flat, pts, "fp32")[:, 0]
    assert np.all(np.abs(d32 - d64) <= 1e-5 * np.maximum(1.0, np.abs(d64)))


def test_calc_normal_unit_sphere(oracle):
    flat = S.FlatScene([S.sphere(1.0, OPT0, 1)])
    for p, n in K.NORMAL_KATS:
        got = oracle.calc_normal(flat, 0, [p])[0]
        assert np.allclose(got, n, atol=1e-9), (p, got)


@pytest.mark.parametrize("op,p,want", K.CSG_KATS)
def test_csg_models(oracle, op, p, want):
    kids = [S.sphere(0.25, OPT0, 1), S.box((1.0, 1.0, 1.0), OPT0, 1)]
    m = S.model(kids, {"intersection": S.intersection, "subtraction": S.subtraction}[op], 1.0)
    got = oracle.eval_sdf(S.FlatScene([m]), [p])[0, 0]
    if want == ">0":
        assert got > 0
    else:
        assert abs(got - want) <= EPS64


def test_transform_helpers():
    """sdfHelpers KATs (test/SDF/test_SDF.f90:301-674)."""
    for ang in (45.0, 90.0, 0.0, 64.45):
        a = S.deg2rad(ang)
        rx = S.rotate_x(ang)
        assert rx[0, 0] == 1 and rx[1, 1] == math.cos(a) and rx[2, 1] == -math.sin(a) and rx[1, 2] == math.sin(a)
        ry = S.rotate_y(ang)
        assert ry[0, 0] == math.cos(a) and ry[2, 0] == math.sin(a) and ry[0, 2] == -math.sin(a)
    rz = S.rotate_z(45.0)
    assert rz[1, 0] == -math.sin(S.deg2rad(45.0)) and rz[0, 1] == math.sin(S.deg2rad(45.0))
    for axis, fn in (((0, 0, 1), S.rotate_z), ((0, 1, 0), S.rotate_y), ((1, 0, 0), S.rotate_x)):
        assert np.array_equal(S.rotmat(axis, 45.0), fn(45.0))
    t = S.translate((1.0, 2.0, 3.0))
    assert tuple(t[3, :3]) == (1.0, 2.0, 3.0)
    assert np.array_equal(S.identity(), np.eye(4))
    sk = S.skew_symm((1.0, 2.0, 3.0))
    assert np.array_equal(sk, -sk.T)
    for a, b in (((0, 0, 1), (1, 0, 0)), ((1, 2, 1), (1, 4, 5))):
        a = np.array(a, float) / np.linalg.norm(a)
        b = np.array(b, float) / np.linalg.norm(b)
        assert np.allclose(S.apply(S.rotation_align(a, b), a), b, atol=1e-14)
    # invert(translate(c)) moves c to the origin (how presets place primitives)
    c = (0.3, -0.2, 0.7)
    assert np.allclose(S.apply(S.invert(S.translate(c)), c), 0.0, atol=1e-15)


def test_fresnel_simple(oracle):
    """Normal incidence refracts straight through; reflection mirrors z (test_fresnel.f90:118-189)."""
    I = np.array([[0.0, 0.0, -1.0]])
    N = np.array([[0.0, 0.0, 1.0]])
    out, refl = oracle.reflect_refract(I, N, 1.0, 1.33, 0.5)
    assert not refl[0] and abs(math.pi - math.acos(out[0, 2])) <= 1e-10
    th = S.deg2rad(50.0)
    I = np.array([[math.sin(th), 0.0, math.cos(th)]])
    out, refl = oracle.reflect_refract(I, N, 1.33, 1.0, 0.5)
    assert refl[0] and np.allclose(out[0], [I[0, 0], I[0, 1], -I[0, 2]], atol=EPS64)


@pytest.mark.parametrize("n1,n2,mode", [(1.0, 1.33, "refract"), (1.33, 1.0, "reflect")])
def test_fresnel_statistical(oracle, n1, n2, mode):
    """Fraction refracted (reflected) at 45 deg over 1e6 trials equals 1-R (R) within 5e-4
    (test_fresnel.f90:34-116)."""
    th = S.deg2rad(45.0)
    n = K.FRESNEL_STAT_TRIALS
    I = np.tile([math.sin(th), 0.0, -math.cos(th)] if mode == "refract" else
                [math.sin(th), 0.0, math.cos(th)], (n, 1))
    N = np.tile([0.0, 0.0, 1.0], (n, 1))
    u = np.random.default_rng(123456789).random(n)
    R = oracle.fresnel(I[:1], N[:1], n1, n2)[0]
    out, refl = oracle.reflect_refract(I, N, n1, n2, u)
    if mode == "refract":
        want_theta = math.asin(n1 / n2 * math.sin(th))
        got = np.abs(np.pi - np.arccos(out[:, 2]) - want_theta) < 1e-10
        assert abs(got.mean() - (1.0 - R)) <= K.FRESNEL_STAT_THR
    else:
        got = (out[:, 2] == -I[:, 2]) & refl
        assert abs(got.mean() - R) <= K.FRESNEL_STAT_THR


def test_fresnel_tir_and_normal_incidence(oracle):
    I = np.array([[math.sin(1.2), 0.0, math.cos(1.2)], [0.0, 0.0, 1.0]])
    N = np.array([[0.0, 0.0, 1.0], [0.0, 0.0, 1.0]])
    R = oracle.fresnel(I, N, 1.45, 1.0)
    assert R[0] == 1.0 and R[1] == 0.0  # TIR -> 1, exact normal incidence -> 0 (surfaces.f90:104-109)


def test_philox_known_answers(oracle):
    for key, ctr, want in K.PHILOX_KATS:
        assert tuple(int(x) for x in oracle.philox(key, ctr)[0]) == want


def scat_test_settings():
    return parse_table({"source": {"name": "point", "nphotons": 100000, "position": [0.0, 0.0, 0.0]},
                        "grid": {"nxg": 200, "nyg": 200, "nzg": 200, "xmax": 1.0, "ymax": 1.0, "zmax": 1.0},
                        "geometry": {"geom_name": "scat_test", "tau": 10.0}, "output": {},
                        "simulation": {"iseed": 123456789}})


def scat_test2_settings():
    return parse_table({"source": {"name": "pencil", "nphotons": 10000000, "position": [0.0, 0.0, 0.0],
                                   "direction": "z"},
                        "grid": {"nxg": 200, "nyg": 200, "nzg": 200, "xmax": 100.0, "ymax": 100.0, "zmax": 100.0},
                        "geometry": {"geom_name": "scat_test2", "tau": 10.0, "hgg": 0.9}, "output": {},
                        "simulation": {"iseed": 123456789}})


def test_scatter_test1_mean_scatters(oracle):
    """Sphere r=1, tau=10, albedo 1: mean scatters 57.5 +- 0.5 (test_scat.f90:23-41)."""
    st = scat_test_settings()
    r = oracle.run(P.setup_simulation(st), st, nphotons=100000, seed=123456789, kernel="test")
    assert abs(r.nscatt / 1e5 - K.SCAT_TEST1_NSCATT) <= K.SCAT_TEST1_THR


def test_scatter_test2_moments(oracle):
    """Pencil beam in a ~infinite g=0.9 medium: scatter-order position moments
    (test_scat.f90:43-86), 1e7 packets as the reference runs."""
    st = scat_test2_settings()
    N = 10_000_000
    r = oracle.run(P.setup_simulation(st), st, nphotons=N, seed=123456789, kernel="test", end_early=True,
                   want_jmean=False)
    m = r.stats["moments"]
    got = np.concatenate([10.0 * m[:12].reshape(4, 3), 100.0 * m[12:].reshape(4, 3)]) / N
    for row, want in zip(got, K.SCAT_TEST2_MOMENTS):
        for ax in range(3):
            assert abs(row[ax] - want[ax]) <= K.SCAT_TEST2_THR[ax], (row, want)
    # sharper: the first-moment z of order k follows 1 + E|mu| (1 + g + ... ), the
    # reference's sign(cost, nzp) making the first scatter off the vertical beam forward-only
    g = 0.9
    mu = np.linspace(-1, 1, 2000001)
    p = (1 - g * g) / (2 * (1 + g * g - 2 * g * mu) ** 1.5)
    e_abs = np.trapezoid(np.abs(mu) * p, mu)
    pred = [1.0, 1 + e_abs, 1 + e_abs * (1 + g), 1 + e_abs * (1 + g + g * g)]
    assert np.allclose(got[:4, 2], pred, atol=4e-3)


def test_reference_and_device_fp64_semantics_agree(oracle):
    """The integer voxel walk (GPU algorithm) and the reference's snapping walk give
    identical event counters and total path length; per voxel they differ only by
    the reference's 1e-8 face snap (update_pos, inttau2.f90:239,369-393) moved
    between neighbours at each crossing (~1e-6 relative on the beam axis)."""
    st = P.benchmark_settings("box_slab")
    arr = P.setup_simulation(st)
    a = oracle.run(arr, st, nphotons=20000, seed=5, policy=oracle.reference_policy())
    b = oracle.run(arr, st, nphotons=20000, seed=5, policy=oracle.device_policy("fp64", st.grid_c()))
    for k in ("nscatt", "sdf_evals", "trace_steps", "fresnel_events", "reflections", "rng_draws"):
        assert a.stats[k] == b.stats[k], k
    assert abs(a.jmean.sum() - b.jmean.sum()) <= 1e-12 * a.jmean.sum()
    assert np.allclose(a.jmean, b.jmean, rtol=1e-5, atol=1e-7 * a.jmean.max())


def test_detector_kats(oracle):
    """Circle / annulus / camera hit tests (test/detector/test_detector.f90:27-167)."""
    from signedmcrt_b200.config import DetectorCfg, Settings
    st = Settings()
    st.geometry.geom_name = "scat_test"
    st.detectors = [DetectorCfg("circle", position=(0, 0, 0), direction=(1, 0, 0), layer=1, radius1=0.5,
                                nbins=100, maxval=100.0),
                    DetectorCfg("annulus", position=(0, 0, 0), direction=(1, 0, 0), layer=1, radius1=0.5,
                                radius2=1.0, nbins=100, maxval=100.0),
                    DetectorCfg("camera", p1=(-1, -1, -1), p2=(0, 2, 0), p3=(0, 0, 2), layer=1, nbins=100,
                                maxval=100.0)]
    assert oracle.detector_bin(st, 0, (0, 0, 0), (1, 0, 0), 1.0, 1) >= 0
    assert oracle.detector_bin(st, 1, (0.75, 0, 0), (-1, 0, 0), 1.0, 1) >= 0
    assert oracle.detector_bin(st, 1, (0, 0, 0), (1, 0, 0), 1.0, 1) < 0
    assert oracle.detector_bin(st, 2, (10, 0, 0), (-1, 0, 0), 1.0, 1) >= 0
    assert oracle.detector_bin(st, 2, (10, 0, 0), (1, 0, 0), 1.0, 1) < 0
    assert oracle.detector_bin(st, 0, (0, 0, 0), (1, 0, 0), 1.0, 2) < 0  # wrong layer


# ---------------------------------------------------------------- SDF modifiers
def _sph(r):
    return S.sphere(r, S.mono(0.0, 0.0, 0.0, 1.0), 1)


def test_bend_known_answers(oracle):
    """test/SDF/test_SDF.f90:265-299 (test_bend): box(1,1,1) bent with k = 10."""
    bbox = S.box((1.0, 1.0, 1.0), S.mono(0.0, 0.0, 0.0, 0.0), 1)
    bent = S.FlatScene([S.bend(bbox, 10.0)])
    plain = S.FlatScene([bbox])
    d = oracle.eval_sdf(bent, [(0.0, 0.0, 0.0), (0.6, 0.0, 0.0), (0.4, -0.4, -0.4)])[:, 0]
    assert d[0] < 0 and d[1] > 0 and d[2] > 0
    assert oracle.eval_sdf(plain, [(0.4, -0.4, -0.4)])[0, 0] < 0


def _points(n=200, seed=3, scale=2.0):
    return np.random.default_rng(seed).uniform(-scale, scale, (n, 3))


def test_revolution_of_sphere_is_torus(oracle):
    pts = _points()
    rev = oracle.eval_sdf(S.FlatScene([S.revolution(_sph(0.3), 1.1)]), pts)[:, 0]
    tor = oracle.eval_sdf(S.FlatScene([S.torus(1.1, 0.3, S.mono(0, 0, 0, 1), 1)]), pts)[:, 0]
    np.testing.assert_allclose(rev, tor, rtol=0, atol=1e-14)


def test_onion_extrude_elongate_twist_formulas(oracle):
    pts = _points()
    r = np.linalg.norm(pts, axis=1)
    got = oracle.eval_sdf(S.FlatScene([S.onion(_sph(0.8), 0.1)]), pts)[:, 0]
    np.testing.assert_allclose(got, np.abs(r - 0.8) - 0.1, atol=1e-14)
    got = oracle.eval_sdf(S.FlatScene([S.extrude(_sph(0.8), 0.3)]), pts)[:, 0]
    d, wy = r - 0.8, np.abs(pts[:, 2]) - 0.3
    want = np.minimum(np.maximum(d, wy), 0) + np.hypot(np.maximum(d, 0), np.maximum(wy, 0))
    np.testing.assert_allclose(got, want, atol=1e-14)
    # elongating a sphere along x gives a capsule (off the axis segment)
    got = oracle.eval_sdf(S.FlatScene([S.elongate(_sph(0.3), (0.7, 0.0, 0.0))]), pts)[:, 0]
    cap = oracle.eval_sdf(S.FlatScene([S.capsule((-0.7, 0, 0), (0.7, 0, 0), 0.3, S.mono(0, 0, 0, 1), 1)]), pts)[:, 0]
    np.testing.assert_allclose(got, cap, atol=1e-14)
    # zero twist / bend leave the primitive unchanged; a twist turns the point about z
    box = S.box((1.0, 0.4, 2.0), S.mono(0, 0, 0, 1), 1)
    base = oracle.eval_sdf(S.FlatScene([box]), pts)[:, 0]
    for f in (S.twist, S.bend):
        np.testing.assert_allclose(oracle.eval_sdf(S.FlatScene([f(box, 0.0)]), pts)[:, 0], base, atol=1e-15)
    k = float(np.float32(0.7))
    a = k * pts[:, 2]
    rot = np.stack([np.cos(a) * pts[:, 0] - np.sin(a) * pts[:, 1], np.sin(a) * pts[:, 0] + np.cos(a) * pts[:, 1],
                    pts[:, 2]], axis=1)
    np.testing.assert_allclose(oracle.eval_sdf(S.FlatScene([S.twist(box, 0.7)]), pts)[:, 0],
                               oracle.eval_sdf(S.FlatScene([box]), rot)[:, 0], atol=1e-14)


def test_nested_modifiers_and_egg_preset(oracle):
    """onion(revolution(egg)) is the reference's egg shell (setupGeometry.f90:37-38):
    the outer modifier maps the point first, the inner one the value first."""
    from signedmcrt_b200 import presets as P
    arr = P.setup_egg()
    pts = _points(100, 5, 4.0)
    got = oracle.eval_sdf(S.FlatScene(arr), pts)
    egg = S.egg(3.0, 3.0 * np.sqrt(2 - np.sqrt(2)), 3.0 * np.sqrt(2 - np.sqrt(2)), S.mono(0, 0, 0, 1), 1)
    q = np.stack([np.hypot(pts[:, 0], pts[:, 2]) - 0.2, pts[:, 1], np.zeros(len(pts))], axis=1)
    inner = oracle.eval_sdf(S.FlatScene([egg]), q)[:, 0]
    np.testing.assert_allclose(got[:, 2], np.abs(inner) - 0.2, atol=1e-14)
    with pytest.raises(ValueError):
        S.onion(S.onion(S.onion(_sph(1.0), 0.1), 0.1), 0.1)


def _render_restated(oracle, flat, samples, extent, precision="fp64"):
    """render_sub (src/sdfs/sdf_base.f90:319-336) with numpy building the voxel
    centres and the oracle evaluating them, image(i, j, k) in Fortran order."""
    ns = np.floor(np.asarray(samples) / 2.0 + 0.5)  # nint, half away from zero
    w = np.asarray(extent, dtype=np.float64) / ns
    axes = [(np.arange(1, n + 1, dtype=np.float64) - ns[a]) * w[a] for a, n in enumerate(samples)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    pts = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    d = oracle.eval_sdf(flat, pts, precision).min(axis=1).astype(np.float32)
    return d.reshape(tuple(samples), order="F")


def test_render_voxel_centres_known_answers(oracle):
    """A unit sphere on a 3^3 render of half-width 1: nint(3/2) = 2 puts the voxels
    at -0.5, 0, 0.5 (sdf_base.f90:320-331)."""
    img = oracle.render(S.FlatScene([_sph(1.0)]), (3, 3, 3), (1.0, 1.0, 1.0))
    assert img.dtype == np.float32 and img.shape == (3, 3, 3)
    assert img[1, 1, 1] == np.float32(-1.0)
    assert img[2, 1, 1] == np.float32(-0.5)
    assert img[0, 0, 0] == np.float32(np.sqrt(0.75) - 1.0)
    # even sizes: nint(4/2) = 2, voxels at -0.5, 0, 0.5, 1.0
    img = oracle.render(S.FlatScene([_sph(1.0)]), (4, 1, 1), (1.0, 1.0, 1.0))
    np.testing.assert_array_equal(img[:, 0, 0], np.float32([-0.5, -1.0, -0.5, 0.0]))


@pytest.mark.parametrize("scene", ["sphere_water", "layered_vessels", "test_egg"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_render_matches_restatement(oracle, scene, precision):
    """The oracle's render loop against the restatement above, ragged sizes, bit for bit."""
    arr = P.setup_egg() if scene == "test_egg" else P.setup_simulation(P.benchmark_settings(scene))
    flat = S.FlatScene(arr)
    for samples in ((9, 6, 5), (7, 1, 4)):
        want = _render_restated(oracle, flat, samples, (2.0, 1.5, 1.0), precision)
        got = oracle.render(flat, samples, (2.0, 1.5, 1.0), precision)
        np.testing.assert_array_equal(got, want)


def test_intersection_known_answers(oracle):
    """test/geometry/test_geometry.f90 test_plane and test_circle: a ray from
    (0,0,-10) along +z meets the z = 0 plane (and the r = 10 disc) at the origin; a
    ray from (0,0,-20) along -z meets neither.  These are the circle detector's hit
    test (check_hit_circle, src/detectors/detectors.f90:110-127)."""
    n, c = (0.0, 0.0, 1.0), (0.0, 0.0, 0.0)
    for hit_fn in (lambda o, d: oracle.intersect_plane(n, c, o, d),
                   lambda o, d: oracle.intersect_circle(n, c, 10.0, o, d)):
        hit, t = hit_fn((0.0, 0.0, -10.0), (0.0, 0.0, 1.0))
        assert hit and np.allclose(np.array([0.0, 0.0, -10.0]) + t * np.array([0.0, 0.0, 1.0]), 0.0)
        hit, _ = hit_fn((0.0, 0.0, -20.0), (0.0, 0.0, -1.0))
        assert not hit
    # beyond the radius the plane is hit but the disc is not
    assert oracle.intersect_plane(n, c, (11.0, 0.0, -1.0), (0.0, 0.0, 1.0))[0]
    assert not oracle.intersect_circle(n, c, 10.0, (11.0, 0.0, -1.0), (0.0, 0.0, 1.0))[0]
