"""GPU parity of the SDF voxel render (render_sub, src/sdfs/sdf_base.f90:302-346)
through the C ABI against the CPU oracle.

The render unit is compiled without FMA contraction, so scenes built from
primitives, CSG and the onion/revolution/extrude/elongate modifiers render bit for
bit as the oracle does, FP64 and FP32.  Twist and bend call sin/cos, whose CUDA
and libm results may differ in the last place: those scenes agree to 1e-6.
"""
import numpy as np
import pytest

from signedmcrt_b200 import presets as P, scene as S, writer
from tests.test_gpu_parity import modifier_scene

pytestmark = pytest.mark.gpu


def _scene(name):
    if name == "test_egg":
        return S.FlatScene(P.setup_egg())
    return S.FlatScene(P.setup_simulation(P.benchmark_settings(name)))


@pytest.mark.parametrize("name", ["sphere_water", "box_slab", "layered_vessels", "test_egg"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_render_bit_exact(gpu, oracle, name, precision):
    flat = _scene(name)
    for samples, extent in (((37, 24, 19), (2.0, 1.5, 1.0)), ((1, 1, 1), (1.0, 1.0, 1.0)), ((64, 1, 3), (4.0, 0.5, 3.0))):
        got = gpu.render(flat, samples, extent, precision)
        want = oracle.render(flat, samples, extent, precision)
        assert got.shape == tuple(samples) and got.dtype == np.float32
        np.testing.assert_array_equal(got, want)


def test_render_reference_default_size_bit_exact(gpu, oracle):
    """The reference's default render_size (200, 200, 200; parse.f90:177) of the
    sphere_water scene, FP64."""
    flat = _scene("sphere_water")
    got = gpu.render(flat, (200, 200, 200), (2.0, 2.0, 2.0))
    np.testing.assert_array_equal(got, oracle.render(flat, (200, 200, 200), (2.0, 2.0, 2.0)))


def test_render_twist_and_bend(gpu, oracle):
    flat = modifier_scene()
    for precision in ("fp64", "fp32"):
        got = gpu.render(flat, (33, 29, 21), (3.0, 3.0, 3.0), precision)
        want = oracle.render(flat, (33, 29, 21), (3.0, 3.0, 3.0), precision)
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6)


def test_render_into_device_memory(gpu):
    import torch
    flat = _scene("layered_vessels")
    img = torch.full((23 * 17 * 9,), float("nan"), dtype=torch.float32, device="cuda")
    gpu.render_device(flat, (23, 17, 9), (1.0, 1.0, 1.5), img.data_ptr(),
                      stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    want = gpu.render(flat, (23, 17, 9), (1.0, 1.0, 1.5))
    np.testing.assert_array_equal(img.cpu().numpy().reshape((23, 17, 9), order="F"), want)


def test_render_geom_writes_the_voxel_file(gpu, tmp_path):
    """render_geom = true in the output table renders the scene at render_size over
    the grid's half-widths and writes it to data/<render> (kernelsMod.f90:531-536)."""
    from signedmcrt_b200 import kernels
    st = P.benchmark_settings("box_slab")
    st.source.nphotons = 2000
    st.output.render_geom = True
    st.output.render_size = (16, 12, 8)
    st.output.render = "geom_render.nrrd"
    run = kernels.run_kernel(st, "pathlength", root=tmp_path, verbose=False)
    path = [f for f in run.files if f.name == "geom_render.nrrd"]
    assert len(path) == 1
    img, _ = writer.read_nrrd(path[0])
    want = gpu.render(P.setup_simulation(st), (16, 12, 8), (st.grid.xmax, st.grid.ymax, st.grid.zmax))
    np.testing.assert_array_equal(np.asarray(img, dtype=np.float32).reshape(want.shape), want)
