"""FP64 per-voxel variance sums (smcrt_run_moments): the history-based second
moment jmean2[v] = sum over packets of (the packet's own path length in voxel v)^2.

(1) FP64 transport against the oracle's exact second moment (each packet's
    scores merged per voxel in a hash map, then squared): identical event
    counters, the same jmean, jmean2 equal to the FP32 rounding of the
    per-packet score sums, and no crowded score table;
(2) FP32 transport: the standard errors the second moment gives agree with the
    spread of independent batches, voxel by voxel on average;
(3) the per-voxel chi-square of FP32 GPU fluence against the reference-semantics
    oracle, with each voxel's standard error from the second moments alone.
"""
import numpy as np
import pytest

from signedmcrt_b200 import presets as P
from tests.test_gpu_parity import COUNT_KEYS, fluence_agrees

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg", ["box_slab", "sphere_water", "layered_vessels"])
def test_fp64_second_moment_matches_oracle(gpu, oracle, cfg):
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    n = 20000
    with gpu.Transport(arr, st, precision="fp64", variance=True) as tr:
        g = tr.run_moments(n, 17)
    o = oracle.run(arr, st, nphotons=n, seed=17, policy=oracle.device_policy("fp64", st.grid_c()),
                   want_moments=True)
    diff = {k: (g.stats[k], o.stats[k]) for k in COUNT_KEYS if g.stats[k] != o.stats[k]}
    assert not diff, diff
    assert g.stats["variance_overflows"] == 0
    fluence_agrees(g.jmean, o.jmean)
    a, b = g.jmean2, o.jmean2
    assert abs(a.sum() - b.sum()) <= 1e-6 * b.sum()
    bad = np.abs(a - b) > 1e-5 * np.abs(b) + 1e-12 * b.max()
    assert bad.mean() <= 1e-3, bad.sum()
    # a packet's merged score squared is at least the sum of its segments squared, and
    # the second moment bounds the first: jmean^2 / N <= jmean2 (Cauchy-Schwarz)
    assert np.all(g.jmean ** 2 / n <= g.jmean2 * (1 + 1e-6) + 1e-300)


def test_fp32_second_moment_standard_errors_match_batch_spread(gpu):
    st = P.benchmark_settings("box_slab")
    arr = P.setup_simulation(st)
    B, bsz = 24, 50000
    means, j2 = [], 0.0
    with gpu.Transport(arr, st, precision="fp32", variance=True) as tr:
        for b in range(B):
            r = tr.run_moments(bsz, 300 + b)
            means.append(r.jmean / bsz)
            j2 = j2 + r.jmean2
            assert r.stats["variance_overflows"] == 0
    m = np.array(means)
    n = B * bsz
    mean = m.mean(axis=0)
    var_hist = j2 / n - mean ** 2                       # per-packet variance, history-based
    var_batch = m.var(axis=0, ddof=1) * bsz             # per-packet variance, from the batches
    mask = mean > 1e-2 * mean.max()
    ratio = var_batch[mask] / var_hist[mask]
    assert mask.sum() > 100
    # the batch estimate has B-1 degrees of freedom per voxel: its mean ratio over
    # the voxels is 1 within a few percent
    assert abs(ratio.mean() - 1.0) < 0.05, (ratio.mean(), mask.sum())


def test_fp32_per_voxel_chi_square_from_second_moments(gpu, oracle):
    st = P.benchmark_settings("box_slab")
    arr = P.setup_simulation(st)
    n_g, n_o = 2_000_000, 200000
    with gpu.Transport(arr, st, precision="fp32", variance=True) as tr:
        g = tr.run_moments(n_g, 99)
    o = oracle.run(arr, st, nphotons=n_o, seed=4321, policy=oracle.reference_policy(), want_moments=True)
    mg, mo = g.jmean / n_g, o.jmean / n_o
    vg = g.jmean2 / n_g - mg ** 2
    vo = o.jmean2 / n_o - mo ** 2
    se = np.sqrt(np.maximum(vg, 0) / n_g + np.maximum(vo, 0) / n_o)
    mask = (mg > 1e-2 * mg.max()) & (se > 0)
    z = (mg - mo)[mask] / se[mask]
    assert mask.sum() > 100
    assert np.mean(z * z) < 1.15, (np.mean(z * z), mask.sum())
    assert np.mean(np.abs(z) > 4) < 2e-3
