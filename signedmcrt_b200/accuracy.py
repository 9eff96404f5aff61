"""Fluence accuracy: the relative RMS error of a fluence map against a reference
map, over the voxels the reference fills (fluence above 1e-3 of its maximum).

The transport's FP32 arithmetic is judged by running the same configuration in
FP32 and in FP64 with the same packet count against a high-count FP64 reference
(other seeds): equal errors mean the FP32 bias lies below the Monte Carlo noise,
so packets/s compare at matched fluence error.  The runs also keep the
history-based second moment (smcrt_run_moments), which gives every voxel's
standard error of the mean and, per voxel, the chi-square of each test map
against the reference.
"""
from __future__ import annotations

import numpy as np


def rms_rel_error(test: np.ndarray, ref: np.ndarray, threshold: float = 1e-3) -> float:
    """sqrt(mean(((test - ref) / ref)^2)) over voxels with ref > threshold * max(ref);
    both maps per packet (tally / packets)."""
    ref = np.asarray(ref, dtype=np.float64)
    test = np.asarray(test, dtype=np.float64)
    mask = ref > threshold * ref.max()
    r = (test[mask] - ref[mask]) / ref[mask]
    return float(np.sqrt(np.mean(r * r)))


def voxel_chi2(jm_a, j2_a, n_a, jm_b, j2_b, n_b, threshold: float = 1e-3) -> dict:
    """Per-voxel z = (mean_a - mean_b) / sqrt(var_a/n_a + var_b/n_b), each voxel's
    per-packet variance from its second moment (jmean2/N - (jmean/N)^2); the mean
    of z^2 (1 when the maps agree) and the fraction |z| > 4, over voxels whose
    mean b is above threshold x its maximum."""
    ma, mb = jm_a / n_a, jm_b / n_b
    va = np.maximum(j2_a / n_a - ma * ma, 0.0)
    vb = np.maximum(j2_b / n_b - mb * mb, 0.0)
    se = np.sqrt(va / n_a + vb / n_b)
    mask = (mb > threshold * mb.max()) & (se > 0)
    z = (ma - mb)[mask] / se[mask]
    return {"chi2_per_voxel": float(np.mean(z * z)), "frac_z_gt_4": float(np.mean(np.abs(z) > 4)),
            "voxels": int(mask.sum())}


def error_table(cfg: str, n_test: int, ref_factor: int = 10, seed: int = 1000, transport_cls=None) -> dict:
    """Runs `cfg` (a benchmark configuration) on the GPU: FP64 reference with
    ref_factor x n_test packets, then FP32 and FP64 runs of n_test packets on other
    seeds; returns their RMS errors against the reference, their per-voxel
    chi-square against it (standard errors from the second moments), the median
    relative standard error of the test maps, and the run times (plain runs)."""
    from . import presets as P
    from .transport import Transport
    T = transport_cls or Transport
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    nref = ref_factor * n_test
    out = {"config": cfg, "packets": n_test, "reference_packets": nref}
    with T(arr, st, precision="fp64", timeout_ms=3_600_000, variance=True) as tr:
        ref = tr.run_moments(nref, seed)
        t64 = tr.run_moments(n_test, seed + 1)
        out["fp64_ms_per_packet"] = tr.run(n_test, seed + 3, want_jmean=False).stats["kernel_ms"] / n_test
    with T(arr, st, precision="fp32", timeout_ms=3_600_000, variance=True) as tr:
        t32 = tr.run_moments(n_test, seed + 2)
        out["fp32_ms_per_packet"] = tr.run(n_test, seed + 3, want_jmean=False).stats["kernel_ms"] / n_test
    phi_ref = ref.jmean / nref
    out["rms_fp32"] = rms_rel_error(t32.jmean / n_test, phi_ref)
    out["rms_fp64"] = rms_rel_error(t64.jmean / n_test, phi_ref)
    out["voxels"] = int((phi_ref > 1e-3 * phi_ref.max()).sum())
    out["ratio"] = out["rms_fp32"] / out["rms_fp64"]
    for tag, t in (("fp32", t32), ("fp64", t64)):
        out["chi2_" + tag] = voxel_chi2(t.jmean, t.jmean2, n_test, ref.jmean, ref.jmean2, nref)
    m = t32.jmean / n_test
    mask = phi_ref > 1e-3 * phi_ref.max()
    sem = np.sqrt(np.maximum(t32.jmean2 / n_test - m * m, 0.0) / n_test)
    out["sem_rel_median_fp32"] = float(np.median(sem[mask] / np.maximum(m[mask], 1e-300)))
    out["variance_overflows"] = int(ref.stats["variance_overflows"] + t64.stats["variance_overflows"] +
                                    t32.stats["variance_overflows"])
    return out
