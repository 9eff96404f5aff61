"""Batches on the GPU: instances of one geometry with their own optics, packet
counts and seeds in one launch equal the same instances run one by one (the same
packets: event counts identical, tallies to FP64 rounding), with and without a
CUDA graph, and the context form falls back to one launch per context when the
geometry differs."""
import numpy as np
import pytest

from signedmcrt_b200 import presets as P
from signedmcrt_b200.transport import Batch, Transport, run_batched

pytestmark = pytest.mark.gpu

OPTICS = [(10.0, 0.1, 0.9, 1.38), (50.0, 0.5, 0.8, 1.45), (2.0, 1.0, 0.95, 1.33), (80.0, 0.01, 0.7, 1.40)]
AMB = (0.0, 0.0, 0.0, 1.0)


def settings(nxg=32):
    st = P.benchmark_settings("box_slab")
    st.grid.nxg = st.grid.nyg = st.grid.nzg = nxg
    return st


def plain(st, kernel, precision, opt, n, seed):
    mus, mua, g, nidx = opt
    with Transport(P.box_slab(mua=mua, mus=mus, g=g, n=nidx), st, kernel=kernel, precision=precision) as tr:
        return tr.run(n, seed)


@pytest.mark.parametrize("kernel", ["pathlength", "weight"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_equals_instances_run_alone(kernel, precision):
    st = settings()
    counts = [3000, 0, 7000, 1500]
    seeds = [5, 6, 7, 8]
    optics = np.array([[o, AMB] for o in OPTICS])
    with Batch(P.box_slab(), st, 4, kernel=kernel, precision=precision, optics=optics) as b:
        jm, bins, per, tot = b.run(counts, seeds)
    assert tot["packets"] == sum(counts)
    for i in range(4):
        ref = plain(st, kernel, precision, OPTICS[i], counts[i], seeds[i])
        assert per[i]["packets"] == ref.stats["packets"] == counts[i]
        assert per[i]["rng_draws"] == ref.stats["rng_draws"]
        if kernel == "pathlength":
            assert per[i]["nscatt"] == ref.stats["nscatt"]
        np.testing.assert_allclose(jm[i], ref.jmean, rtol=1e-9, atol=1e-12 * max(ref.jmean.max(), 1e-30))


def test_graph_replays_with_new_counts_and_seeds():
    st = settings()
    optics = np.array([[o, AMB] for o in OPTICS])
    with Batch(P.box_slab(), st, 4, precision="fp64", optics=optics) as b:
        direct = [b.run([2000, 1000, 500, 4000], [1, 2, 3, 4]), b.run([100, 3000, 0, 2500], [9, 8, 7, 6])]
        graph = [b.run([2000, 1000, 500, 4000], [1, 2, 3, 4], use_graph=True),
                 b.run([100, 3000, 0, 2500], [9, 8, 7, 6], use_graph=True)]
    for (j1, _, p1, t1), (j2, _, p2, t2) in zip(direct, graph):
        assert [p["rng_draws"] for p in p1] == [p["rng_draws"] for p in p2]
        assert t1["voxel_segments"] == t2["voxel_segments"]
        np.testing.assert_allclose(j1, j2, rtol=1e-9, atol=1e-12 * j1.max())


def test_run_batched_over_contexts():
    st = settings()
    trs = [Transport(P.box_slab(mua=o[1], mus=o[0], g=o[2], n=o[3]), st, precision="fp64") for o in OPTICS]
    res = run_batched(trs, [2000, 2500, 1000, 3000], [3, 4, 5, 6])
    for tr, r, n, sd in zip(trs, res, [2000, 2500, 1000, 3000], [3, 4, 5, 6]):
        ref = tr.run(n, sd)
        assert r.stats["rng_draws"] == ref.stats["rng_draws"]
        np.testing.assert_allclose(r.jmean, ref.jmean, rtol=1e-9, atol=1e-12 * ref.jmean.max())
    # a context with another geometry: every context runs alone, results unchanged
    other = Transport(P.box_slab(half=0.5), st, precision="fp64")
    res2 = run_batched(trs[:2] + [other], [2000, 2500, 1000], [3, 4, 5])
    np.testing.assert_allclose(res2[0].jmean, res[0].jmean, rtol=1e-9, atol=1e-12 * res[0].jmean.max())
    assert res2[2].stats["packets"] == 1000
    for t in trs + [other]:
        t.close()


@pytest.mark.parametrize("cfg", ["box_slab", "layered_vessels"])
def test_autotune_keeps_results(cfg):
    """The autotuner only changes how tallies are accumulated: FP64 event counts
    and tallies of a run are the same before and after tuning."""
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    with Transport(arr, st, precision="fp64") as tr:
        before = tr.run(20000, 4)
        t = tr.autotune(trial_packets=50000)
        after = tr.run(20000, 4)
    assert t["tally_copies"] in (1, 2, 4, 8) and t["packets_per_s"] > 0 and t["trials"] >= 2
    assert t["block_size"] == 640 and t["slots_per_thread"] == 1 and t["ctas_per_sm"] >= 1
    assert before.stats["voxel_segments"] == after.stats["voxel_segments"]
    assert np.array_equal(before.bins, after.bins)
    np.testing.assert_allclose(after.jmean, before.jmean, rtol=1e-9, atol=1e-12 * before.jmean.max())


def test_fp32_error_matches_fp64_error():
    """At matched packet counts the FP32 transport's fluence error against a 10x
    FP64 reference equals the FP64 transport's (its bias is below the noise)."""
    from signedmcrt_b200.accuracy import error_table
    t = error_table("box_slab", 200000)
    assert 0.85 < t["ratio"] < 1.15, t
    # per voxel, with standard errors from the second moments
    assert t["variance_overflows"] == 0, t
    for tag in ("fp32", "fp64"):
        assert t["chi2_" + tag]["voxels"] > 1000 and t["chi2_" + tag]["chi2_per_voxel"] < 1.15, t
        assert t["chi2_" + tag]["frac_z_gt_4"] < 2e-3, t
