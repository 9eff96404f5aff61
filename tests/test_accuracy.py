"""The fluence RMS error measure (host side, on synthetic maps)."""
import numpy as np

from signedmcrt_b200.accuracy import rms_rel_error, voxel_chi2


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


def test_voxel_chi2_of_two_samples_of_one_distribution():
    """Two tallies of the same per-packet score distribution (exponential scores,
    a tenth of packets scoring per voxel): mean z^2 near 1; a shifted mean shows."""
    rng = np.random.default_rng(3)
    nv, na, nb = 400, 20000, 40000

    def tally(n, scale):
        hit = rng.random((n, nv)) < 0.1
        s = np.where(hit, rng.exponential(scale, (n, nv)), 0.0)
        return s.sum(axis=0), (s * s).sum(axis=0)

    a, a2 = tally(na, 1.0)
    b, b2 = tally(nb, 1.0)
    r = voxel_chi2(a, a2, na, b, b2, nb)
    assert r["voxels"] == nv and abs(r["chi2_per_voxel"] - 1.0) < 0.2
    c, c2 = tally(na, 1.1)
    assert voxel_chi2(c, c2, na, b, b2, nb)["chi2_per_voxel"] > 3.0
