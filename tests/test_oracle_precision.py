"""The FP32 device semantics (the GPU's FP32 kernels' algorithm: the reference's
epsilon 1e-8, integer voxel walk, FP64 boundary events, and sweeps within 16 FP32
ulps of a surface or after a crossing step in FP64) against the reference
semantics (FP64, eps 1e-8, the snapping voxel walk of src/inttau2.f90:213-441),
both in the CPU oracle, on the curved refracting surface of sphere_water: the
epsilon policy must not move the fluence, the total path length, or the rates
of Fresnel events and reflections (src/inttau2.f90:44,58-61,104-136;
src/surfaces.f90:14-40)."""
import math

import numpy as np

from oracle import binding as O
from signedmcrt_b200 import presets as P
from tests import fluence_stats as FS


def test_fp32_eps_policy_matches_reference_at_a_curved_surface():
    st = P.benchmark_settings("sphere_water")
    arr = P.setup_simulation(st)
    n_ref, B, bsz = 160000, 16, 20000
    ref = O.run(arr, st, nphotons=n_ref, seed=424242, policy=O.reference_policy())
    pol = O.device_policy("fp32", st.grid_c())
    acc = FS.Accumulator(bsz)
    rates = []
    for b in range(B):
        r = O.run(arr, st, nphotons=bsz, seed=7000 + b, policy=pol)
        acc.add(r.jmean)
        rates.append([r.stats["fresnel_events"] / bsz, r.stats["reflections"] / bsz, r.nscatt / bsz])
    res = FS.compare(acc, ref.jmean, n_ref)
    FS.assert_agree(res)
    rates = np.array(rates)
    want = np.array([ref.stats["fresnel_events"], ref.stats["reflections"], ref.nscatt]) / n_ref
    se = rates.std(axis=0, ddof=1) * math.sqrt(bsz) * math.sqrt(1 / (B * bsz) + 1 / n_ref)
    assert np.all(np.abs(rates.mean(axis=0) - want) <= 3.5 * se), (rates.mean(axis=0), want, se)


def test_without_fp64_near_surface_sweeps_fp32_is_biased():
    """The same comparison with every sweep in FP32 (the rule switched off) shows the
    bias the rule removes: FP32 coordinate rounding near the surface changes how
    many refracted packets the eps rule kills, and the total path drops by ~1%.
    With and without the rule run on the same streams (common random numbers)."""
    st = P.benchmark_settings("sphere_water")
    arr = P.setup_simulation(st)
    B, bsz = 8, 15000
    ref = O.run(arr, st, nphotons=B * bsz, seed=11, policy=O.reference_policy())
    pol = O.device_policy("fp32", st.grid_c())
    with_rule, without = [], []
    for b in range(B):
        pol.near_surface_f64 = 1
        with_rule.append(O.run(arr, st, nphotons=bsz, seed=20 + b, policy=pol).jmean.sum() / bsz)
        pol.near_surface_f64 = 0
        without.append(O.run(arr, st, nphotons=bsz, seed=20 + b, policy=pol).jmean.sum() / bsz)
    with_rule, without = np.array(with_rule), np.array(without)
    t_ref = ref.jmean.sum() / (B * bsz)
    se = with_rule.std(ddof=1) / math.sqrt(B) * math.sqrt(2.0)  # both runs of B x bsz packets
    assert abs(with_rule.mean() - t_ref) <= 3 * se, (with_rule.mean(), t_ref, se)
    d = with_rule - without  # paired: the streams are shared
    assert d.mean() / t_ref > 0.005 and d.mean() > 3 * d.std(ddof=1) / math.sqrt(B), d
