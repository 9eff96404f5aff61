"""The fluence RMS error measure (host side, on synthetic maps)."""
import numpy as np

from signedmcrt_b200.accuracy import rms_rel_error


def test_rms_rel_error_definition():
    ref = np.array([1.0, 2.0, 4.0, 1e-4])  # the last voxel is below 1e-3 of the maximum
    test = np.array([1.1, 1.8, 4.0, 5.0])
    want = np.sqrt(np.mean([0.1 ** 2, 0.1 ** 2, 0.0]))
    assert abs(rms_rel_error(test, ref) - want) < 1e-15


def test_rms_scales_like_poisson_noise():
    rng = np.random.default_rng(0)
    ref = np.full(10000, 100.0)
    err = [rms_rel_error(rng.poisson(ref * k) / k, ref) for k in (1, 4, 16)]
    assert abs(err[0] / err[1] - 2.0) < 0.1 and abs(err[1] / err[2] - 2.0) < 0.1
