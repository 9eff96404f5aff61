"""The path-replay adjoint on the GPU.

(1) Known answer: in an absorbing medium the packets cannot leave, the mean
    track length per packet is 1/mu_a whatever mu_s and g are, so with unit voxel
    weights d/d mu_a = -1/mu_a^2 and d/d mu_s = d/d g = 0.
(2) The layered-vessel scene, 15 parameters (mu_a, mu_s, g of vessels, three
    layers and the bounding medium): the adjoint against common-random-number
    central finite differences of the same loss, batch means within 3 sigma.
(3) The same scene and loss: the adjoint against the oracle's perturbation Monte
    Carlo reference gradient (FP64, whole-path likelihood ratio), a different
    estimator of the same expectation.
"""
import numpy as np
import pytest
import torch

from signedmcrt_b200 import presets as P
from signedmcrt_b200.autograd import layered_groups, transport

pytestmark = pytest.mark.gpu


def absorbing_box():
    st = P.benchmark_settings("box_slab")
    st.grid.nxg = st.grid.nyg = st.grid.nzg = 40
    st.grid.xmax = st.grid.ymax = st.grid.zmax = 5.0
    st.source.position = (0.0, 0.0, 0.0)

    def scene_fn(o):
        mua, mus, g = o[0]
        return P.box_slab(mua=mua, mus=mus, g=g, n=1.0, half=5.0)
    return st, scene_fn


def test_adjoint_known_answer_absorbing_medium():
    st, scene_fn = absorbing_box()
    mua = 5.0
    grads, tracks = [], []
    for b in range(8):
        params = torch.tensor([[mua, 5.0, 0.9]], dtype=torch.float64, requires_grad=True)
        phi, det = transport(params, scene_fn, st, [0, -1], 250000, 100 + b)
        loss = phi.sum()  # mean track length per packet inside the grid
        loss.backward()
        grads.append(params.grad.numpy()[0].copy())
        tracks.append(float(loss.detach()))
    g = np.array(grads)
    m, se = g.mean(axis=0), g.std(axis=0, ddof=1) / np.sqrt(len(g))
    assert abs(np.mean(tracks) - 1 / mua) < 0.01 / mua
    assert abs(m[0] - (-1 / mua ** 2)) < 4 * se[0] + 1e-3 / mua ** 2, (m, se)
    assert abs(m[1]) < 4 * se[1] + 1e-4 and abs(m[2]) < 4 * se[2] + 1e-4, (m, se)


def layered_params():
    # (mu_a, mu_s, g) per group: vessels, layer 1..3, bounding medium (given optics
    # so that its parameters have a finite-difference neighbourhood)
    return np.array([[5.0, 50.0, 0.9], [1.0, 100.0, 0.8], [0.3, 50.0, 0.9], [0.1, 30.0, 0.9], [0.01, 0.1, 0.5]])


def layered_loss(phi, det):
    nx, ny, nz = phi.shape
    z = torch.linspace(1.0, 0.2, nz, dtype=torch.float64, device=phi.device)  # deeper voxels weigh less
    w = z.reshape(1, 1, nz).expand(nx, ny, nz)
    h = torch.linspace(1.0, 2.0, det.numel(), dtype=torch.float64, device=det.device)
    return (w * phi).sum() + (h * det).sum()


def test_adjoint_matches_crn_finite_differences():
    st = P.benchmark_settings("layered_vessels")
    scene_fn, groups = layered_groups()
    base = layered_params()
    n, rel = 200000, 0.02
    adj, fd = [], []
    for b in range(6):
        seed = 500 + b
        p = torch.tensor(base, dtype=torch.float64, requires_grad=True)
        layered_loss(*transport(p, scene_fn, st, groups, n, seed)).backward()
        adj.append(p.grad.numpy().reshape(-1).copy())
        row = []
        for k in range(base.size):
            dp = np.zeros(base.size)
            dp[k] = rel * base.flat[k]
            lp = float(layered_loss(*transport(torch.tensor(base + dp.reshape(base.shape)), scene_fn, st, groups,
                                               n, seed)))
            lm = float(layered_loss(*transport(torch.tensor(base - dp.reshape(base.shape)), scene_fn, st, groups,
                                               n, seed)))
            row.append((lp - lm) / (2 * dp[k]))
        fd.append(row)
    adj, fd = np.array(adj), np.array(fd)
    se = np.sqrt(adj.var(axis=0, ddof=1) / len(adj) + fd.var(axis=0, ddof=1) / len(fd))
    z = (adj.mean(axis=0) - fd.mean(axis=0)) / np.maximum(se, 1e-12)
    # Finite differences only see a parameter through packets whose paths change:
    # the bounding medium is a 0.001 cm shell crossed in one step, so its mu_a and
    # mu_s move the loss by much less than one packet's contribution and the CRN
    # differences are exactly zero in every batch.  Compare where they vary.
    informative = np.abs(fd).max(axis=0) > 1e-9 * np.abs(fd).max()
    assert informative.sum() >= 12
    assert np.all(np.abs(z[informative]) < 3.0), (z, adj.mean(axis=0), fd.mean(axis=0))


def test_adjoint_matches_oracle_reference_gradient(oracle):
    """GPU adjoint (FP32 transport, two-pass causal replay) against the oracle's
    perturbation Monte Carlo gradient (FP64, C times the whole path's score) of
    L = sum w jmean + sum h bins, 8 batches each.  15 parameters are compared at
    once, so each |z| must stay below 3.5 (two-sided 5e-4 per parameter, under 1%
    for the family) and the mean z^2 near 1."""
    from signedmcrt_b200.transport import Transport
    st = P.benchmark_settings("layered_vessels")
    st.grid.nxg = st.grid.nyg = st.grid.nzg = 30
    scene_fn, groups = layered_groups()
    base = layered_params()
    nz = st.grid.nzg
    w = np.broadcast_to(np.linspace(1.0, 0.2, nz, dtype=np.float32).astype(np.float64).reshape(1, 1, nz),
                        (st.grid.nxg, st.grid.nyg, nz))
    nb = sum(d.nbins + 1 for d in st.detectors)
    h = np.linspace(1.0, 2.0, nb)
    w_dev = torch.tensor(np.asfortranarray(w).reshape(-1, order="F"), dtype=torch.float32, device="cuda")
    h_dev = torch.tensor(h, dtype=torch.float64, device="cuda")
    pol = oracle.device_policy("fp64", st.grid_c())
    n, B = 100000, 8
    gpu, ref = [], []
    with Transport(scene_fn(base), st, precision="fp32") as tr:
        for b in range(B):
            g, _ = tr.adjoint(n, 900 + b, w_dev.data_ptr(), h_dev.data_ptr(), groups, 5)
            gpu.append(g.reshape(-1) / n)
            r, _ = oracle.adjoint(scene_fn(base), st, nphotons=n, seed=900 + b, w=w, h=h, region_group=groups,
                                  ngroups=5, policy=pol)
            ref.append(r.reshape(-1) / n)
    gpu, ref = np.array(gpu), np.array(ref)
    se = np.sqrt(gpu.var(axis=0, ddof=1) / B + ref.var(axis=0, ddof=1) / B)
    resolved = se > 0
    z = (gpu.mean(axis=0) - ref.mean(axis=0))[resolved] / se[resolved]
    assert resolved.sum() >= 13
    assert np.all(np.abs(z) < 3.5) and np.mean(z ** 2) < 2.5, (z, gpu.mean(axis=0), ref.mean(axis=0))


def test_adjoint_in_an_albedo_one_region(oracle):
    """An albedo-1 sphere (mu_a = 0 < 1e-9: init_mono sets albedo 1,
    src/opticalProps/opticalProperties.f90:115-119): its scatter events score the
    interaction density kappa alone (the roulette no longer depends on the
    parameters), so d/d mu_a = d/d mu_s exactly, packet by packet; and the GPU
    gradient agrees with the oracle's perturbation Monte Carlo gradient, which
    tests/test_oracle_adjoint.py pins to finite differences on this scene."""
    from signedmcrt_b200.transport import Transport
    from tests.test_oracle_adjoint import _albedo_one
    st, arr = _albedo_one(10.0)
    w = np.ones((20, 20, 20))
    w_dev = torch.ones(20 ** 3, dtype=torch.float32, device="cuda")
    pol = oracle.device_policy("fp64", st.grid_c())
    n, B = 50000, 8
    gpu, ref = [], []
    with Transport(arr, st, precision="fp32") as tr:
        for b in range(B):
            g, _ = tr.adjoint(n, 40 + b, w_dev.data_ptr(), None, [0, -1], 1)
            assert g[0, 0] == g[1, 0]  # the same terms accumulate into both rows
            gpu.append(g[:, 0] / n)
            r, _ = oracle.adjoint(arr, st, nphotons=n, seed=40 + b, w=w, h=None, region_group=[0, -1], ngroups=1,
                                  policy=pol)
            ref.append(r[:, 0] / n)
    gpu, ref = np.array(gpu), np.array(ref)
    se = np.sqrt(gpu.var(axis=0, ddof=1) / B + ref.var(axis=0, ddof=1) / B)
    z = (gpu.mean(axis=0) - ref.mean(axis=0)) / se
    assert np.all(np.abs(z[:2]) < 3.5), (z, gpu.mean(axis=0), ref.mean(axis=0))
