"""Fluence accuracy: the relative RMS error of a fluence map against a reference
map, over the voxels the reference fills (fluence above 1e-3 of its maximum).

The transport's FP32 arithmetic is judged by running the same configuration in
FP32 and in FP64 with the same packet count against a high-count FP64 reference
(other seeds): equal errors mean the FP32 bias lies below the Monte Carlo noise,
so packets/s compare at matched fluence error.
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


def error_table(cfg: str, n_test: int, ref_factor: int = 10, seed: int = 1000, transport_cls=None) -> dict:
    """Runs `cfg` (a benchmark configuration) on the GPU: FP64 reference with
    ref_factor x n_test packets, then FP32 and FP64 runs of n_test packets on other
    seeds; returns their RMS errors against the reference and the run times."""
    from . import presets as P
    from .transport import Transport
    T = transport_cls or Transport
    st = P.benchmark_settings(cfg)
    arr = P.setup_simulation(st)
    out = {"config": cfg, "packets": n_test, "reference_packets": ref_factor * n_test}
    with T(arr, st, precision="fp64", timeout_ms=3_600_000) as tr:
        ref = tr.run(ref_factor * n_test, seed)
        out["fp64_ms_per_packet"] = ref.stats["kernel_ms"] / (ref_factor * n_test)
        phi_ref = ref.jmean / (ref_factor * n_test)
        t64 = tr.run(n_test, seed + 1)
    with T(arr, st, precision="fp32", timeout_ms=3_600_000) as tr:
        t32 = tr.run(n_test, seed + 2)
        out["fp32_ms_per_packet"] = t32.stats["kernel_ms"] / n_test
    out["rms_fp32"] = rms_rel_error(t32.jmean / n_test, phi_ref)
    out["rms_fp64"] = rms_rel_error(t64.jmean / n_test, phi_ref)
    out["voxels"] = int((phi_ref > 1e-3 * phi_ref.max()).sum())
    out["ratio"] = out["rms_fp32"] / out["rms_fp64"]
    return out
