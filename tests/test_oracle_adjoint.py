"""The oracle's perturbation Monte Carlo reference gradient, pinned on the CPU.

The reference gradient is the likelihood-ratio estimator: each packet's
contribution C to L = sum w jmean + sum h bins times the derivative of the log
density of its whole path (survival per region, interaction density, roulette,
Henyey-Greenstein phase function).  It is a different estimator from the GPU's
two-pass causal replay, so the GPU adjoint is compared with it statistically
(tests/test_gpu_adjoint.py).  Here it is checked against
(1) a known answer: in an absorbing medium the packets cannot leave and the mean
    track length is 1/mu_a whatever mu_s and g are, so with unit voxel weights
    d/d mu_a = -1/mu_a^2 and d/d mu_s = d/d g = 0;
(2) the oracle's own common-random-number central finite differences of the same
    loss on the layered-vessel scene (15 parameters), batch means within 3 sigma.
"""
import numpy as np

from signedmcrt_b200 import presets as P
from signedmcrt_b200.autograd import layered_groups


def absorbing_settings():
    st = P.benchmark_settings("box_slab")
    st.grid.nxg = st.grid.nyg = st.grid.nzg = 20
    st.grid.xmax = st.grid.ymax = st.grid.zmax = 5.0
    st.source.position = (0.0, 0.0, 0.0)
    return st


def test_reference_gradient_known_answer_absorbing_medium(oracle):
    st = absorbing_settings()
    mua = 5.0
    arr = P.box_slab(mua=mua, mus=5.0, g=0.9, n=1.0, half=5.0)
    w = np.ones((20, 20, 20))
    pol = oracle.device_policy("fp64", st.grid_c())
    n, grads, losses = 40000, [], []
    for b in range(8):
        g, L = oracle.adjoint(arr, st, nphotons=n, seed=300 + b, w=w, h=None, region_group=[0, -1], ngroups=1,
                              policy=pol)
        grads.append(g[:, 0] / n)
        losses.append(L / n)
    g = np.array(grads)
    m, se = g.mean(axis=0), g.std(axis=0, ddof=1) / np.sqrt(len(g))
    assert abs(np.mean(losses) - 1 / mua) < 0.01 / mua
    assert abs(m[0] - (-1 / mua ** 2)) < 4 * se[0] + 1e-3 / mua ** 2, (m, se)
    assert abs(m[1]) < 4 * se[1] + 1e-4 and abs(m[2]) < 4 * se[2] + 1e-4, (m, se)


def layered_case():
    st = P.benchmark_settings("layered_vessels")
    st.grid.nxg = st.grid.nyg = st.grid.nzg = 30
    scene_fn, groups = layered_groups()
    base = np.array([[5.0, 50.0, 0.9], [1.0, 100.0, 0.8], [0.3, 50.0, 0.9], [0.1, 30.0, 0.9], [0.01, 0.1, 0.5]])
    nz = st.grid.nzg
    w = np.broadcast_to(np.linspace(1.0, 0.2, nz).reshape(1, 1, nz), (st.grid.nxg, st.grid.nyg, nz))
    return st, scene_fn, groups, base, w


def test_reference_gradient_matches_crn_finite_differences(oracle):
    st, scene_fn, groups, base, w = layered_case()
    pol = oracle.device_policy("fp64", st.grid_c())
    nb = sum(d.nbins + 1 for d in st.detectors)
    h = np.linspace(1.0, 2.0, nb)

    def loss(params, n, seed):
        r = oracle.run(scene_fn(params), st, nphotons=n, seed=seed, policy=pol)
        return float((w * r.jmean).sum() + (h * r.bins).sum())

    n, rel = 20000, 0.02
    ref, fd = [], []
    for b in range(6):
        seed = 700 + b
        g, L = oracle.adjoint(scene_fn(base), st, nphotons=n, seed=seed, w=w, h=h, region_group=groups, ngroups=5,
                              policy=pol)
        assert abs(L - loss(base, n, seed)) <= 1e-9 * abs(L)
        ref.append(g.T.reshape(-1) / n)
        row = []
        for k in range(base.size):
            dp = np.zeros(base.size)
            dp[k] = rel * base.flat[k]
            row.append((loss(base + dp.reshape(base.shape), n, seed) - loss(base - dp.reshape(base.shape), n, seed))
                       / (2 * dp[k] * n))
        fd.append(row)
    ref, fd = np.array(ref), np.array(fd)
    se = np.sqrt(ref.var(axis=0, ddof=1) / len(ref) + fd.var(axis=0, ddof=1) / len(fd))
    z = (ref.mean(axis=0) - fd.mean(axis=0)) / np.maximum(se, 1e-300)
    # the bounding medium is a 0.001 cm shell: its mu_a and mu_s move the loss by far
    # less than one packet's contribution, so the CRN differences are exactly zero
    informative = fd.std(axis=0) > 0
    assert informative.sum() >= 12
    assert np.all(np.abs(z[informative]) < 3.0), (z, ref.mean(axis=0), fd.mean(axis=0))


def _albedo_one(mus):
    from signedmcrt_b200 import scene as S
    st = P.benchmark_settings("box_slab")
    st.grid.nxg = st.grid.nyg = st.grid.nzg = 20
    st.source.name = "point"
    st.source.position = (0.0, 0.0, 0.0)
    arr = [S.sphere(0.5, S.mono(mus, 0.0, 0.0, 1.0), 1), S.box((2.0, 2.0, 2.0), S.mono(0.0, 0.0, 0.0, 1.0), 2)]
    return st, arr


def test_reference_gradient_in_an_albedo_one_region(oracle):
    """With the albedo held at 1 the loss depends on mu_a and mu_s only through
    kappa = mu_s + mu_a, so d/d mu_a = d/d mu_s, and both match common-random-number
    central finite differences in mu_s (mu_a cannot be stepped down from 0)."""
    mus, rel, B, n = 10.0, 0.02, 8, 20000
    st, arr = _albedo_one(mus)
    w = np.ones((20, 20, 20))
    pol = oracle.device_policy("fp64", st.grid_c())
    g, fd = [], []
    for b in range(B):
        gb, _ = oracle.adjoint(arr, st, nphotons=n, seed=400 + b, w=w, h=None, region_group=[0, -1], ngroups=1,
                               policy=pol)
        g.append(gb[:, 0] / n)
        lp = oracle.run(_albedo_one(mus * (1 + rel))[1], st, nphotons=n, seed=400 + b, policy=pol).jmean.sum() / n
        lm = oracle.run(_albedo_one(mus * (1 - rel))[1], st, nphotons=n, seed=400 + b, policy=pol).jmean.sum() / n
        fd.append((lp - lm) / (2 * rel * mus))
    g, fd = np.array(g), np.array(fd)
    m, se = g.mean(axis=0), g.std(axis=0, ddof=1) / np.sqrt(B)
    assert abs(m[0] - m[1]) <= 3 * np.hypot(se[0], se[1]), (m, se)
    sfd = fd.std(ddof=1) / np.sqrt(B)
    assert abs(m[1] - fd.mean()) <= 3 * np.hypot(se[1], sfd), (m[1], fd.mean(), se[1], sfd)
