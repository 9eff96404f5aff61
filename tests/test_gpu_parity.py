"""GPU parity: the sm_100a path through the C ABI against the CPU oracle.

(a) building blocks (SDF values, normals, Fresnel, reflect/refract, HG scatter,
    Philox) -- FP32 within 1e-5 (relative to max(1, |value|)), FP64 to rounding;
(b) per-packet histories replayed from injected uniform streams -- FP64 identical
    to the oracle's device semantics, FP32 within 1e-5 of the reference semantics;
(c) whole runs on the counter RNG -- FP64 event counters identical to the oracle,
    FP32 fluence and detector totals statistically equal (chi-square per voxel
    block, totals within 3 sigma) to the reference-semantics oracle.
"""
import math

import numpy as np
import pytest

from signedmcrt_b200 import abi, presets as P, scene as S
from tests import fluence_stats as FS
from tests import reference_kats as K
from tests.test_oracle_kats import make_prim, scat_test2_settings, scat_test_settings

pytestmark = pytest.mark.gpu
OPT0 = S.mono(0.0, 0.0, 0.0, 0.0)
TOL32 = 1e-5


def fluence_agrees(a, b, rtol_voxel=1e-6):
    """FP64 tallies of the same histories: total to 1e-12, 10^3-voxel blocks to 1e-7,
    and at least 99.9% of voxels to rtol_voxel.  Individual voxels may differ more
    where a ~1e-9 position difference (libm ulps amplified along a long history)
    moves a voxel-face crossing."""
    assert abs(a.sum() - b.sum()) <= 1e-12 * abs(b.sum())
    ba, bb = block_sums(a), block_sums(b)
    assert np.allclose(ba, bb, rtol=1e-7, atol=1e-10 * bb.max())
    bad = np.abs(a - b) > rtol_voxel * np.abs(b) + 1e-12 * b.max()
    assert bad.mean() <= 1e-3, bad.sum()


def all_primitives_scene():
    arr = [make_prim(name, args) for name, args, _ in K.SDF_KATS]
    t = S.invert(S.translate((0.1, -0.2, 0.3))) @ np.eye(4)
    arr.append(S.box((1.0, 0.5, 0.8), OPT0, 1, transform=S.invert(S.rotate_y(30.0)) @ S.invert(S.translate((0.2, 0, 0)))))
    arr.append(S.capsule((-0.5, 0, 0), (0.5, 0.2, 0), 0.3, OPT0, 1, transform=t))
    kids = [S.sphere(0.25, OPT0, 1), S.box((1.0, 1.0, 1.0), OPT0, 1)]
    for op in (S.union, S.smooth_union, S.subtraction, S.intersection):
        arr.append(S.model(kids, op, 0.1))
    return S.FlatScene(arr[:16])


def test_sdf_values(gpu, oracle):
    flat = all_primitives_scene()
    rng = np.random.default_rng(0)
    pts = np.concatenate([rng.uniform(-3, 3, (4000, 3)), rng.uniform(-0.3, 0.3, (1000, 3))])
    ref = oracle.eval_sdf(flat, pts, "fp64")
    g64 = gpu.eval_sdf(flat, pts, "fp64")
    g32 = gpu.eval_sdf(flat, pts, "fp32")
    assert np.allclose(g64, ref, rtol=0, atol=1e-13)
    assert np.all(np.abs(g32 - ref) <= TOL32 * np.maximum(1.0, np.abs(ref)))


def test_sdf_known_answers_on_device(gpu):
    for name, args, cases in K.SDF_KATS:
        flat = S.FlatScene([make_prim(name, args)])
        pts = np.array([c[0] for c in cases], dtype=np.float64)
        got = gpu.eval_sdf(flat, pts, "fp64")[:, 0]
        for (p, want, thr), g in zip(cases, got):
            assert abs(g - want) <= (thr if thr is not None else 4e-16), (name, p, g)


def test_normals(gpu, oracle):
    flat = all_primitives_scene()
    rng = np.random.default_rng(1)
    pts = rng.uniform(-1.5, 1.5, (500, 3))
    for r in range(flat.nregions):
        a = gpu.calc_normal(flat, r, pts)
        b = oracle.calc_normal(flat, r, pts)
        ok = np.isfinite(b).all(axis=1)
        assert np.allclose(a[ok], b[ok], atol=1e-9), r
    sph = S.FlatScene([S.sphere(1.0, OPT0, 1)])
    for p, n in K.NORMAL_KATS:
        assert np.allclose(gpu.calc_normal(sph, 0, [p])[0], n, atol=1e-9)


def random_incidence(n, seed):
    rng = np.random.default_rng(seed)
    I = rng.normal(size=(n, 3))
    I /= np.linalg.norm(I, axis=1, keepdims=True)
    N = rng.normal(size=(n, 3))
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    n1 = rng.choice([1.0, 1.33, 1.38, 1.45], n)
    n2 = rng.choice([1.0, 1.33, 1.36, 1.4], n)
    return I, N, n1, n2


def well_conditioned(I, N, n1, n2, margin=0.05):
    """Away from the critical angle, where R and the refracted direction have
    unbounded sensitivity to cos(theta): the transmitted cos^2 = 1 - sin^2 must
    exceed `margin` (or total internal reflection must hold by that margin)."""
    c = np.abs(np.einsum("ij,ij->i", I, N))
    s2 = n1 / n2 * np.sqrt(np.maximum(0.0, 1 - c * c))
    return np.abs(1.0 - s2 * s2) > margin


def test_fresnel_and_reflect_refract(gpu, oracle):
    """The transport evaluates boundary events in FP64 (identical to the oracle);
    the FP32 form of the same functions is checked on well-conditioned inputs."""
    I, N, n1, n2 = random_incidence(20000, 2)
    ok = well_conditioned(I, N, n1, n2)
    assert ok.mean() > 0.85
    R64 = oracle.fresnel(I, N, n1, n2)
    assert np.allclose(gpu.fresnel(I, N, n1, n2, "fp64"), R64, atol=1e-14)
    assert np.all(np.abs(gpu.fresnel(I, N, n1, n2, "fp32") - R64)[ok] <= TOL32)
    u = np.random.default_rng(3).random(len(I))
    o64, r64 = oracle.reflect_refract(I, N, n1, n2, u)
    g64, gr64 = gpu.reflect_refract(I, N, n1, n2, u, "fp64")
    assert np.array_equal(r64, gr64) and np.allclose(g64, o64, atol=1e-13)
    g32, gr32 = gpu.reflect_refract(I, N, n1, n2, u, "fp32")
    same = (gr32 == r64) & ok   # a draw within FP32 rounding of R may fall either side
    assert same.mean() > 0.85
    assert np.all(np.abs(g32[same] - o64[same]) <= TOL32)
    # normal incidence and total internal reflection (surfaces.f90:104-109)
    Ik = np.array([[0, 0, -1.0], [math.sin(1.2), 0, math.cos(1.2)]])
    Nk = np.array([[0, 0, 1.0], [0, 0, 1.0]])
    for prec in ("fp32", "fp64"):
        Rk = gpu.fresnel(Ik, Nk, np.array([1.0, 1.45]), np.array([1.33, 1.0]), prec)
        assert Rk[0] == 0.0 and Rk[1] == 1.0


def test_hg_scatter(gpu, oracle):
    rng = np.random.default_rng(4)
    n = 20000
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:50] = (0, 0, 1.0)
    d[50:100] = (0, 0, -1.0)
    g = rng.choice([0.0, 0.8, 0.9, 0.85], n)
    u = rng.random((n, 3))
    ref = oracle.scatter_dir(d, g, u, "fp64")
    assert np.allclose(gpu.scatter_dir(d, g, u, "fp64"), ref, atol=1e-13)
    assert np.all(np.abs(gpu.scatter_dir(d, g, u, "fp32") - ref) <= TOL32)


def test_philox_on_device(gpu):
    for key, ctr, want in K.PHILOX_KATS:
        assert tuple(int(x) for x in gpu.philox(key, ctr)[0]) == want
    rng = np.random.default_rng(5)
    key = rng.integers(0, 2**32, (1000, 2), dtype=np.uint64).astype(np.uint32)
    ctr = rng.integers(0, 2**32, (1000, 4), dtype=np.uint64).astype(np.uint32)
    from oracle import binding
    assert np.array_equal(gpu.philox(key, ctr), binding.philox(key, ctr))


# ---------------------------------------------------------------- replay
SCENES = ["box_slab", "sphere_water", "layered_vessels"]


def streams(npk, per, seed):
    u = np.random.default_rng(seed).random(npk * per)
    u = np.where(u == 0.0, 0.5, u)
    return u, np.arange(0, npk * per + 1, per, dtype=np.int64)


@pytest.mark.parametrize("cfg", SCENES)
def test_replay_fp64_matches_oracle(gpu, oracle, cfg):
    """FP64 replay: every discrete decision identical to the oracle (draw count,
    scatter count, final layer, detector bins); positions agree to 1e-9 after
    tens of boundary events (libm-ulp differences amplified by curved refraction)."""
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    u, off = streams(512, 6000, 11)
    with gpu.Transport(arr, st, precision="fp64") as tr:
        res, states = tr.replay(u, off)
    ref = oracle.run(arr, st, nphotons=512, seed=0, policy=oracle.device_policy("fp64", st.grid_c()),
                     uniforms=u, offsets=off, want_states=True)
    assert not np.any(states["flags"] & 4), "a packet exhausted its stream"
    assert np.array_equal(states["layer"], ref.states["layer"])
    assert np.array_equal(states["nscatt"], ref.states["nscatt"])
    assert np.array_equal(states["ndraws"], ref.states["ndraws"])
    assert np.allclose(states["pos"], ref.states["pos"], atol=1e-9)
    assert np.allclose(states["dir"], ref.states["dir"], atol=1e-9)
    fluence_agrees(res.jmean, ref.jmean)
    assert np.array_equal(res.bins, ref.bins)


def short_history(cfg):
    """The scene with absorbing optics (mua = max(mua, mus)): about two interactions
    per packet, so one history is a well-conditioned function of its stream."""
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)

    def absorb(o):
        return S.mono(o.mus, max(o.mua, o.mus), o.hgg, o.n)
    out = []
    for ent in arr:
        if isinstance(ent, S.Model):
            for k in ent.children:
                k.opt = absorb(k.opt)
        else:
            ent.opt = absorb(ent.opt)
        out.append(ent)
    return out, st


def history_close(a, b, tol=TOL32):
    same = (a["ndraws"] == b["ndraws"]) & (a["layer"] == b["layer"]) & (a["nscatt"] == b["nscatt"])
    return same & np.all(np.abs(a["pos"] - b["pos"]) <= tol * np.maximum(1, np.abs(b["pos"])), axis=1) \
        & np.all(np.abs(a["dir"] - b["dir"]) <= 10 * tol, axis=1)


@pytest.mark.parametrize("cfg", SCENES)
def test_replay_fp32_single_histories_within_1e5(gpu, oracle, cfg):
    """FP32 histories replayed from the same uniforms as the FP64 reference algorithm
    end within 1e-5 (positions, cm scale) of it.  A history may differ only where a
    discrete decision lands within rounding of its threshold."""
    arr, st = short_history(cfg)
    u, off = streams(4096, 400, 12)
    with gpu.Transport(arr, st, precision="fp32") as tr:
        _, states = tr.replay(u, off)
    ref = oracle.run(arr, st, nphotons=4096, seed=0, policy=oracle.reference_policy(), uniforms=u, offsets=off,
                     want_states=True, want_jmean=False)
    assert not np.any(states["flags"] & 4)
    assert history_close(states, ref.states).mean() >= 0.99


@pytest.mark.parametrize("cfg", SCENES)
def test_replay_fp32_full_scenes_track_oracle(gpu, oracle, cfg):
    """Full-length FP32 histories (tens of events) against the oracle's FP32 device
    semantics: the large majority stay within 1e-5; the rest diverge through
    ulp-level differences (FMA, libm) amplified at curved refracting surfaces."""
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    u, off = streams(1024, 6000, 13)
    with gpu.Transport(arr, st, precision="fp32") as tr:
        _, states = tr.replay(u, off)
    ref = oracle.run(arr, st, nphotons=1024, seed=0, policy=oracle.device_policy("fp32", st.grid_c()),
                     uniforms=u, offsets=off, want_states=True, want_jmean=False)
    assert history_close(states, ref.states).mean() >= 0.9


# ---------------------------------------------------------------- counter RNG runs
COUNT_KEYS = ("nscatt", "sdf_evals", "voxel_segments", "trace_steps", "scatters", "fresnel_events", "reflections",
              "rng_draws", "kills_error", "kills_step_cap")


@pytest.mark.parametrize("cfg", SCENES)
@pytest.mark.parametrize("kernel", ["pathlength", "weight"])
def test_fp64_run_matches_oracle_exactly(gpu, oracle, cfg, kernel):
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    n = 20000
    with gpu.Transport(arr, st, precision="fp64", kernel=kernel) as tr:
        g = tr.run(n, 99)
    o = oracle.run(arr, st, nphotons=n, seed=99, kernel=kernel, policy=oracle.device_policy("fp64", st.grid_c()))
    diff = {k: (g.stats[k], o.stats[k]) for k in COUNT_KEYS if g.stats[k] != o.stats[k]}
    assert not diff, diff
    fluence_agrees(g.jmean, o.jmean)
    assert np.array_equal(g.bins, o.bins)


def block_sums(j, b=10):
    nx, ny, nz = j.shape
    return j.reshape(nx // b, b, ny // b, b, nz // b, b).sum(axis=(1, 3, 5))


@pytest.mark.parametrize("cfg,n_or,batches,bsz", [("box_slab", 200000, 32, 100000),
                                                  ("sphere_water", 400000, 32, 100000),
                                                  ("layered_vessels", 100000, 32, 50000)])
def test_fp32_fluence_statistical_parity(gpu, oracle, cfg, n_or, batches, bsz):
    """FP32 GPU fluence vs the reference-semantics FP64 oracle (eps 1e-8, snapping
    voxel walk) on independent seeds: chi-square per degree of freedom over 10^3-voxel
    blocks, the per-voxel chi-square (mean z^2) over voxels above 1e-2 of the
    maximum, the total path length within 3 sigma, and every detector bin within
    4 sigma (tests/fluence_stats.py)."""
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    o = oracle.run(arr, st, nphotons=n_or, seed=424242, policy=oracle.reference_policy())
    acc = FS.Accumulator(bsz)
    bins = []
    with gpu.Transport(arr, st, precision="fp32") as tr:
        for b in range(batches):
            r = tr.run(bsz, 1000 + b)
            acc.add(r.jmean)
            bins.append(r.bins / bsz)
    res = FS.compare(acc, o.jmean, n_or)
    print(cfg, res)
    FS.assert_agree(res)
    ng = batches * bsz
    if st.detectors:
        bins = np.array(bins)
        gb, obn = bins.mean(axis=0), o.bins / n_or
        seb = bins.std(axis=0, ddof=1) * math.sqrt(bsz) * math.sqrt(1 / ng + 1 / n_or)
        ok = seb > 0
        assert np.all(np.abs(gb - obn)[ok] <= 4 * seb[ok])
        assert abs(gb.sum() - obn.sum()) <= 3 * math.sqrt((seb ** 2).sum())


def test_scatter_test1_on_device(gpu, tmp_path):
    """Scatter_test1 (test/end_to_end/test_scat.f90:23-41) as the reference runs it:
    test_kernel, then the mean scatter count read back from nscatt.dat."""
    from signedmcrt_b200 import kernels, writer
    st = scat_test_settings()
    kernels.run_kernel(st, "test", root=tmp_path, verbose=False)
    val = writer.read_table(tmp_path / "nscatt.dat")[0, 0]
    assert abs(val - K.SCAT_TEST1_NSCATT) <= K.SCAT_TEST1_THR


def test_scatter_test2_on_device(gpu, tmp_path):
    """Scatter_test2 (test/end_to_end/test_scat.f90:43-86) as the reference runs it:
    test_kernel(end_early), then the 8 moment rows read back from positions.dat."""
    from signedmcrt_b200 import kernels, writer
    st = scat_test2_settings()
    N = 10_000_000
    st.source.nphotons = N
    kernels.run_kernel(st, "test", end_early=True, root=tmp_path, verbose=False)
    got = writer.read_table(tmp_path / "positions.dat")
    assert got.shape == (8, 3)
    for row, want in zip(got, K.SCAT_TEST2_MOMENTS):
        for ax in range(3):
            assert abs(row[ax] - want[ax]) <= K.SCAT_TEST2_THR[ax], (row, want)


def test_run_device_into_torch_tensors_equals_run(gpu):
    import torch
    st = P.benchmark_settings("layered_vessels")
    arr = P.setup_simulation(st)
    with gpu.Transport(arr, st, precision="fp64") as tr:
        ref = tr.run(30000, 5)
        jm = torch.zeros(tr.ncell, dtype=torch.float64, device="cuda")
        bins = torch.zeros(tr.nbins, dtype=torch.float64, device="cuda")
        # two shards of the packet range add up to the whole run
        tr.run_device(0, 10000, 5, jm.data_ptr(), bins.data_ptr())
        tr.run_device(10000, 20000, 5, jm.data_ptr(), bins.data_ptr(), stats=True)
    got = jm.cpu().numpy().reshape(tr.shape, order="F")
    assert np.allclose(got, ref.jmean, rtol=1e-11, atol=1e-12 * ref.jmean.max())
    assert np.array_equal(bins.cpu().numpy(), ref.bins)


def test_time_budget_stops_the_kernel_and_context_stays_usable(gpu):
    """A run past its time limit returns SMCRT_ERR_TIMEOUT (device-side budget, no
    fault) and the same context runs normally afterwards."""
    from signedmcrt_b200 import _lib
    st = P.benchmark_settings("sphere_water")
    arr = P.setup_simulation(st)
    with gpu.Transport(arr, st, timeout_ms=20) as tr:
        with pytest.raises(_lib.SmcrtError) as e:
            tr.run(2_000_000_000, 1)
        assert e.value.code == abi.ERR_TIMEOUT
        r = tr.run(1000, 2)
        assert r.stats["packets"] == 1000 and r.stats["device_status"] == 0


def test_invalid_inputs_are_errors(gpu):
    from signedmcrt_b200 import _lib
    st = P.benchmark_settings("box_slab")
    bad = [S.box((2, 2, 2), S.mono(-1.0, 0.1, 0.9, 1.38), 1)]
    with pytest.raises(_lib.SmcrtError) as e:
        gpu.Transport(bad, st)
    assert e.value.code == abi.ERR_SCENE
    too_many = [S.sphere(0.01 * (i + 1), S.mono(1, 0, 0, 1), i) for i in range(300)]  # > 255 regions
    with pytest.raises(_lib.SmcrtError) as e:
        gpu.Transport(too_many, st)
    assert e.value.code == abi.ERR_SCENE
    st.grid.nxg = 0
    with pytest.raises(_lib.SmcrtError) as e:
        gpu.Transport(P.setup_simulation(st), st)
    assert e.value.code == abi.ERR_ARG


def test_tally_copies_sum_to_the_single_grid(gpu):
    """Fluence-grid copies only spread the atomic adds: the same FP64 histories
    tallied into 1 or 8 copies give the same counters, bins and fluence."""
    st = P.benchmark_settings("box_slab")
    arr = P.setup_simulation(st)
    out = []
    for copies in (1, 8):
        with gpu.Transport(arr, st, precision="fp64", tally_copies=copies) as tr:
            out.append(tr.run(50000, 17))
    a, b = out
    assert all(a.stats[k] == b.stats[k] for k in COUNT_KEYS)
    # FP64 atomics add in a different order: agreement to accumulated rounding
    assert np.allclose(a.jmean, b.jmean, rtol=1e-10, atol=1e-12 * a.jmean.max())
    assert np.array_equal(a.bins, b.bins)


@pytest.mark.parametrize("nbins", [40, 70])
def test_camera_bins_shared_and_global(gpu, oracle, nbins):
    """A camera of 41^2 bins is counted in shared memory, one of 71^2 bins (above
    the 4096-bin limit) in the global bins: both equal the oracle's FP64 bins."""
    from signedmcrt_b200.config import DetectorCfg
    st = P.benchmark_settings("box_slab")
    st.detectors = [DetectorCfg("camera", p1=(-1.0, -1.0, -1.0), p2=(1.0, -1.0, -1.0), p3=(-1.0, 1.0, -1.0),
                                layer=1, nbins=nbins, maxval=2.0)]
    arr = P.setup_simulation(st)
    n = 20000
    with gpu.Transport(arr, st, precision="fp64") as tr:
        g = tr.run(n, 31)
    o = oracle.run(arr, st, nphotons=n, seed=31, policy=oracle.device_policy("fp64", st.grid_c()))
    assert g.bins.size == (nbins + 1) ** 2
    assert g.bins.sum() > 0
    assert np.array_equal(g.bins, o.bins)


@pytest.mark.parametrize("cfg", SCENES)
def test_fp32_total_path_is_unbiased(gpu, cfg):
    """The FP32 transport's mean path length per packet equals the FP64
    transport's within 4 standard errors (8 batches each, independent seeds).
    Sensitive to ~0.2%: FP32 surface decisions once lost 0.8% here."""
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    n, B = 500000, 8
    means = {}
    for prec, base in (("fp32", 100), ("fp64", 200)):
        with gpu.Transport(arr, st, precision=prec) as tr:
            means[prec] = np.array([tr.run(n, base + b).jmean.sum() / n for b in range(B)])
    m32, m64 = means["fp32"], means["fp64"]
    se = np.sqrt(m32.var(ddof=1) / B + m64.var(ddof=1) / B)
    assert abs(m32.mean() - m64.mean()) < 4 * se, (m32.mean(), m64.mean(), se)


def modifier_scene():
    o = OPT0
    box = S.box((1.0, 0.4, 2.0), o, 1)
    sph = S.sphere(0.8, o, 1)
    egg = S.egg(3.0, 2.3, 2.3, o, 1)
    return S.FlatScene([S.onion(sph, 0.1), S.revolution(S.sphere(0.3, o, 1), 1.1), S.extrude(sph, 0.3),
                        S.elongate(S.sphere(0.3, o, 1), (0.7, 0.2, 0.0)), S.twist(box, 0.7), S.bend(box, 0.9),
                        S.onion(S.revolution(egg, 0.2), 0.2)])


def test_modified_primitives_on_device(gpu, oracle):
    flat = modifier_scene()
    pts = np.random.default_rng(11).uniform(-3, 3, (4000, 3))
    want = oracle.eval_sdf(flat, pts, "fp64")
    got64 = gpu.eval_sdf(flat, pts, "fp64")
    np.testing.assert_allclose(got64, want, rtol=1e-12, atol=1e-12)
    got32 = gpu.eval_sdf(flat, pts, "fp32")
    assert np.all(np.abs(got32 - want) <= TOL32 * np.maximum(1.0, np.abs(want)))


def test_egg_preset_fp64_transport_matches_oracle(gpu, oracle):
    """The reference's test_egg scene (onion and revolution modifiers): FP64 event
    counters identical to the oracle's."""
    st = P.benchmark_settings("box_slab")
    st.grid.nxg = st.grid.nyg = st.grid.nzg = 40
    st.grid.xmax = st.grid.ymax = st.grid.zmax = 4.0
    st.source.position = (0.0, 0.0, 3.9)
    arr = P.setup_egg()
    with gpu.Transport(arr, st, precision="fp64") as tr:
        g = tr.run(20000, 8)
    o = oracle.run(arr, st, nphotons=20000, seed=8, policy=oracle.device_policy("fp64", st.grid_c()))
    diff = {k: (g.stats[k], o.stats[k]) for k in COUNT_KEYS if g.stats[k] != o.stats[k]}
    assert not diff, diff
    assert g.stats["fresnel_events"] > 0
    fluence_agrees(g.jmean, o.jmean)


@pytest.mark.parametrize("cfg", ["box_slab", "layered_vessels"])
def test_shared_fluence_sub_box_equals_global_tally(gpu, cfg):
    """The privatised beam-axis sub-box (options.shared_fluence) only changes where
    segments are summed: FP32 runs with it on and off follow identical histories
    (identical counters and detector bins), and the fluence agrees to the
    fixed-point rounding of the shared sums (2^-32 cm a segment)."""
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    out = []
    for mode in (1, 2):
        with gpu.Transport(arr, st, precision="fp32", shared_fluence=mode) as tr:
            out.append(tr.run(200000, 21))
    on, off = out
    for k in COUNT_KEYS:
        assert on.stats[k] == off.stats[k], (k, on.stats[k], off.stats[k])
    assert np.array_equal(on.bins, off.bins)
    np.testing.assert_allclose(on.jmean, off.jmean, rtol=1e-7, atol=1e-9 * off.jmean.max())
    assert abs(on.jmean.sum() - off.jmean.sum()) <= 1e-8 * off.jmean.sum()
