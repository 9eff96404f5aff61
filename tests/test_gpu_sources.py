"""Every emitter of src/photon.f90 and the circle detector
(src/detectors/detectors.f90:74-127) on the device against the CPU oracle:

* launch states from smcrt_emit equal the oracle's emitter in FP64 (bit for bit)
  and within 1e-5 in FP32, on the same Philox streams;
* the reference's own source tests (test/photon/test_photon.f90) hold on the
  device's emitters;
* whole FP64 runs with each source and a circle detector give event counters and
  detector bins identical to the oracle's."""
import numpy as np
import pytest

from signedmcrt_b200.scene import FlatScene
from tests import source_cases as SC
from tests.test_gpu_parity import COUNT_KEYS, fluence_agrees

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(SC.BOX_SOURCES))
def test_device_emitters_match_oracle(gpu, oracle, name):
    st, arr = SC.box_source_settings(name)
    flat = FlatScene(arr)
    n = 4096
    gp, gd, gl = gpu.emit(flat, st, 100, n, 77, "fp64")
    op, od, ol = oracle.emit(flat, st, n, 77, "fp64", first=100)
    # the same draws and formulas; sin/cos/atan2/log of CUDA and of the host C
    # library may differ in the last bit
    assert np.abs(gp - op).max() <= 1e-13 and np.abs(gd - od).max() <= 1e-13
    assert np.array_equal(gl, ol)
    gp, gd, gl = gpu.emit(flat, st, 100, n, 77, "fp32")
    op, od, ol = oracle.emit(flat, st, n, 77, "fp32", first=100)
    assert np.abs(gp - op).max() <= 1e-5 * max(1.0, np.abs(op).max())
    assert np.abs(gd - od).max() <= 1e-5
    assert np.array_equal(gl, ol)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["uniform", "point", "pencil", "circular"])
def test_device_emitters_pass_reference_source_tests(gpu, kind, precision):
    st, arr = SC.kat_settings(kind)
    pos, _, _ = gpu.emit(FlatScene(arr), st, 0, 10000, 12345678, precision)
    SC.check_kat(kind, pos)


@pytest.mark.parametrize("name", list(SC.BOX_SOURCES))
def test_fp64_runs_with_each_source_and_a_circle_detector_match_oracle(gpu, oracle, name):
    st, arr = SC.box_source_settings(name, circle_detector=True)
    n = 20000
    with gpu.Transport(arr, st, precision="fp64") as tr:
        g = tr.run(n, 99)
    o = oracle.run(arr, st, nphotons=n, seed=99, policy=oracle.device_policy("fp64", st.grid_c()))
    diff = {k: (g.stats[k], o.stats[k]) for k in COUNT_KEYS if g.stats[k] != o.stats[k]}
    assert not diff, diff
    fluence_agrees(g.jmean, o.jmean)
    assert g.bins.sum() > 100  # the circle detector is hit
    assert np.array_equal(g.bins, o.bins)
