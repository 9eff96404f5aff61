"""Statistical comparison of two Monte Carlo fluence tallies of the same scene.

Run A is given as B independent batches of `bsz` packets each; run B as one
tally of `n_b` packets.  The per-packet variance of every voxel (and block of
voxels) is estimated from A's batches and, since both runs transport the same
physics, used for both: the standard error of the difference of the per-packet
means is sqrt(var (1/n_a + 1/n_b)).  Reported:

* chi2_block: chi-square per degree of freedom over 10^3-voxel blocks whose mean
  is above 1e-3 of the largest block (sums of many voxels: near-Gaussian);
  expected (B - 1)/(B - 3) with the variance estimated from B batches;
* z2_voxel: the mean of z^2 over single voxels above `voxel_frac` of the largest
  voxel, and the fraction with |z| > 4 (the per-voxel chi-square per degree of
  freedom; near 1 when the runs agree, inflated by a few percent by the
  (B - 1)-dof variance estimate);
* z_total: the difference of the total path length per packet in units of its
  standard error.
"""
import math

import numpy as np


def block_sums(j, b=10):
    nx, ny, nz = j.shape
    return j.reshape(nx // b, b, ny // b, b, nz // b, b).sum(axis=(1, 3, 5))


class Accumulator:
    """Sums of per-packet batch means and their squares, voxel- and block-wise."""

    def __init__(self, bsz: int):
        self.bsz = bsz
        self.n = 0
        self.s = self.q = self.bs = self.bq = 0.0
        self.tot = []

    def add(self, jmean):
        m = np.asarray(jmean, dtype=np.float64) / self.bsz
        b = block_sums(m)
        self.s = self.s + m
        self.q = self.q + m * m
        self.bs = self.bs + b
        self.bq = self.bq + b * b
        self.tot.append(m.sum())
        self.n += 1


def compare(acc: Accumulator, ref_jmean, n_b: int, voxel_frac: float = 1e-2) -> dict:
    B, bsz = acc.n, acc.bsz
    n_a = B * bsz

    def pp_var(s, q):  # per-packet variance from the batch means
        mean = s / B
        return mean, np.maximum(q / B - mean * mean, 0.0) * B / (B - 1) * bsz

    ref = np.asarray(ref_jmean, dtype=np.float64) / n_b
    mb, vb = pp_var(acc.bs, acc.bq)
    rb = block_sums(ref)
    se = np.sqrt(vb * (1.0 / n_a + 1.0 / n_b))
    mask = (mb > 1e-3 * mb.max()) & (se > 0)
    zb = (mb[mask] - rb[mask]) / se[mask]
    mv, vv = pp_var(acc.s, acc.q)
    sev = np.sqrt(vv * (1.0 / n_a + 1.0 / n_b))
    maskv = (mv > voxel_frac * mv.max()) & (sev > 0)
    zv = (mv[maskv] - ref[maskv]) / sev[maskv]
    tot = np.array(acc.tot)
    se_tot = tot.std(ddof=1) * math.sqrt(bsz) * math.sqrt(1.0 / n_a + 1.0 / n_b)
    return {"batches": B, "chi2_block": float((zb * zb).sum() / max(mask.sum(), 1)), "dof_block": int(mask.sum()),
            "z2_voxel": float((zv * zv).mean()) if maskv.any() else float("nan"), "voxels": int(maskv.sum()),
            "frac_z_gt_4": float((np.abs(zv) > 4).mean()) if maskv.any() else 0.0,
            "z_total": float((tot.mean() - ref.sum()) / se_tot), "total_a": float(tot.mean()),
            "total_b": float(ref.sum())}


def assert_agree(r: dict, min_voxels: int = 200):
    """The acceptance used by the parity tests.  With the variance estimated from
    B batches (B - 1 degrees of freedom) the expected chi-square per degree of
    freedom is (B - 1) / (B - 3), not 1.  Accepted: the block chi-square within 5
    sigma of that, the per-voxel mean z^2 below 1.12 times it, at most 0.5% of
    voxels beyond 4 sigma, and the total within 3 sigma."""
    infl = (r["batches"] - 1) / (r["batches"] - 3)
    assert r["dof_block"] > 50, r
    assert r["chi2_block"] < infl * (1 + 5 * math.sqrt(2 / r["dof_block"])), r
    assert r["voxels"] >= min_voxels, r
    assert r["z2_voxel"] < 1.12 * infl, r
    assert r["frac_z_gt_4"] <= 5e-3, r
    assert abs(r["z_total"]) <= 3.0, r
