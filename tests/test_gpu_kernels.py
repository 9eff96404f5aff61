"""The reference-named entry points (kernels.pathlength_scatter & co.) on the GPU:
files written as finalise writes them, and checkpoints that resume exactly."""
import numpy as np
import pytest

from signedmcrt_b200 import kernels, writer

pytestmark = pytest.mark.gpu

TOML = """
[source]
name = "pencil"
position = [0.0, 0.0, 0.99999]
direction = "-z"
nphotons = {n}
[grid]
nxg = 40
nyg = 40
nzg = 40
xmax = 1.0
ymax = 1.0
zmax = 1.0
[geometry]
geom_name = "box_slab"
[output]
fluence = "slab.nrrd"
overwrite = true
[simulation]
iseed = 11
checkpoint_file = "slab.ckpt"
checkpoint_every_n = {every}
load_checkpoint = {load}
"""

COUNTS = ("packets", "sdf_evals", "voxel_segments", "trace_steps", "scatters", "fresnel_events", "rng_draws")


def run(tmp_path, every, load=False, n=20000):
    f = tmp_path / f"in_{every}_{int(load)}.toml"
    f.write_text(TOML.format(n=n, every=every, load=str(load).lower()))
    return kernels.pathlength_scatter(f, root=tmp_path, precision="fp64", verbose=False)


def test_pathlength_scatter_writes_normalised_fluence(tmp_path):
    r = run(tmp_path, every=10**9)
    arr, fields = writer.read_nrrd(tmp_path / "data" / "jmean" / "slab.nrrd")
    assert fields["type"] == "double" and fields["nphotons"] == "20000"
    np.testing.assert_array_equal(arr, r.fluence)
    assert r.jmean.sum() > 0 and r.stats["packets"] == 20000 and np.isfinite(r.nscatt)


def test_checkpointed_and_resumed_runs_equal_one_run(tmp_path):
    whole = run(tmp_path, every=10**9)
    chunked = run(tmp_path, every=5000)          # checkpoints at 5000, 10000, 15000
    assert all(chunked.stats[k] == whole.stats[k] for k in COUNTS)
    np.testing.assert_allclose(chunked.jmean, whole.jmean, rtol=1e-10, atol=1e-12 * whole.jmean.max())
    _, done, _ = writer.load_checkpoint(tmp_path / "data" / "slab.ckpt", whole.jmean.shape)
    assert done == 15000
    resumed = run(tmp_path, every=5000, load=True)  # continues from packet 15000
    np.testing.assert_allclose(resumed.jmean, whole.jmean, rtol=1e-10, atol=1e-12 * whole.jmean.max())
