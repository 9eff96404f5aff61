"""Scenes beyond the launch's parameter block: the reference's own res/sphere.toml
(setup_sphere_scene, src/setupGeometry.f90:62-106: 40 spheres + the bounding box
= 41 regions) runs on the device from scene tables in device memory, with the
sweep's bounding-sphere cull.  FP64 event counters equal the oracle's exactly
(the cull skips only regions that cannot change the sweep's outputs), FP32
transport agrees with the reference-semantics oracle in total path length, and a
small scene gives the same FP64 histories from device memory as from the
parameter block."""
import math

import numpy as np
import pytest

from signedmcrt_b200 import abi, presets as P
from tests.test_gpu_parity import COUNT_KEYS, fluence_agrees

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("num_spheres", [17, 40, 120])
def test_sphere_scene_fp64_matches_oracle_exactly(gpu, oracle, num_spheres):
    st = P.sphere_scene_settings(num_spheres=num_spheres)
    arr = P.setup_simulation(st)
    assert len(arr) == num_spheres + 1
    n = 20000
    with gpu.Transport(arr, st, precision="fp64") as tr:
        g = tr.run(n, 31)
    o = oracle.run(arr, st, nphotons=n, seed=31, policy=oracle.device_policy("fp64", st.grid_c()))
    diff = {k: (g.stats[k], o.stats[k]) for k in COUNT_KEYS if g.stats[k] != o.stats[k]}
    assert not diff, diff
    assert g.stats["fresnel_events"] > 0.2 * n  # many packets do cross the spheres
    fluence_agrees(g.jmean, o.jmean)


def test_sphere_scene_fp32_total_path_matches_reference_semantics(gpu, oracle):
    st = P.sphere_scene_settings(num_spheres=40)
    arr = P.setup_simulation(st)
    n_or, batches, bsz = 200000, 16, 100000
    o = oracle.run(arr, st, nphotons=n_or, seed=4242, policy=oracle.reference_policy())
    tot = []
    with gpu.Transport(arr, st, precision="fp32") as tr:
        for b in range(batches):
            tot.append(tr.run(bsz, 500 + b).jmean.sum() / bsz)
    tot = np.array(tot)
    ng = batches * bsz
    se = tot.std(ddof=1) * math.sqrt(bsz) * math.sqrt(1 / ng + 1 / n_or)
    assert abs(tot.mean() - o.jmean.sum() / n_or) <= 3 * se, (tot.mean(), o.jmean.sum() / n_or, se)


@pytest.mark.parametrize("cfg", ["layered_vessels", "sphere_water"])
def test_device_memory_scene_equals_parameter_block(gpu, cfg):
    """The same FP64 packets from the parameter-block scene and from device-memory
    tables with the cull (layered_vessels: 4 cullable capsules): identical events."""
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    n = 20000
    with gpu.Transport(arr, st, precision="fp64") as a, \
            gpu.Transport(arr, st, precision="fp64", scene_memory=1) as b:
        ra, rb = a.run(n, 5), b.run(n, 5)
    diff = {k: (ra.stats[k], rb.stats[k]) for k in COUNT_KEYS if ra.stats[k] != rb.stats[k]}
    assert not diff, diff
    fluence_agrees(rb.jmean, ra.jmean)
    assert np.array_equal(ra.bins, rb.bins)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("cfg,n", [("sphere_scene", 40), ("layered_vessels", 0), ("sphere_water", 0)])
def test_nearest_region_cache_changes_nothing(gpu, cfg, n, precision):
    """The nearest-region cache only skips regions that cannot be the nearest, and
    the region it keeps is evaluated by the same code: runs with it on and off
    follow identical histories -- identical event counters, the same fluence (up
    to the order of the FP64 atomic adds) -- in FP64 and in FP32."""
    st = P.sphere_scene_settings(num_spheres=n) if cfg == "sphere_scene" else P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    out = []
    for mode in (1, 2):
        with gpu.Transport(arr, st, precision=precision, nearest_cache=mode) as tr:
            out.append(tr.run(20000, 5))
    on, off = out
    for k in ("sdf_evals", "voxel_segments", "trace_steps", "scatters", "fresnel_events", "reflections"):
        assert on.stats[k] == off.stats[k], (k, on.stats[k], off.stats[k])
    np.testing.assert_allclose(on.jmean, off.jmean, rtol=1e-9, atol=1e-12 * off.jmean.max())


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("cfg", ["sphere_water", "layered_vessels"])
def test_group_order_changes_nothing(gpu, cfg, precision):
    """The group order only decides which chunks of a round's sorted list the
    warps take first: each packet's history is the same under either order --
    identical event counters and detector bins, the same fluence up to the order
    of the FP64 atomic adds -- and the autotuner reports the order it keeps."""
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    out = []
    for order in (abi.ORDER_WALK_LAST, abi.ORDER_INTERACT_LAST):
        with gpu.Transport(arr, st, precision=precision, group_order=order) as tr:
            out.append(tr.run(20000, 5))
    a, b = out
    for k in ("sdf_evals", "voxel_segments", "trace_steps", "scatters", "fresnel_events", "reflections"):
        assert a.stats[k] == b.stats[k], (k, a.stats[k], b.stats[k])
    np.testing.assert_allclose(a.jmean, b.jmean, rtol=1e-9, atol=1e-12 * b.jmean.max())
    assert np.array_equal(a.bins, b.bins)
    with gpu.Transport(arr, st, precision=precision) as tr:
        t = tr.autotune(20000, 3)
        assert t["group_order"] in (abi.ORDER_WALK_LAST, abi.ORDER_INTERACT_LAST)
