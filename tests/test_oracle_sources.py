"""The oracle's emitters pinned to signedMCRT's own source tests
(test/photon/test_photon.f90): uniform x fixed and y, z in range, point and pencil
positions exact, circular positions within the radius of the (moved) centre."""
import pytest

from oracle import binding as O
from signedmcrt_b200.scene import FlatScene
from tests import source_cases as SC


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["uniform", "point", "pencil", "circular"])
def test_oracle_emitters_pass_reference_source_tests(kind, precision):
    st, arr = SC.kat_settings(kind)
    pos, _, _ = O.emit(FlatScene(arr), st, 10000, 12345678, precision)
    SC.check_kat(kind, pos)


@pytest.mark.parametrize("name", list(SC.BOX_SOURCES))
def test_every_box_source_launches_inside_the_box(name):
    st, arr = SC.box_source_settings(name)
    pos, d, layer = O.emit(FlatScene(arr), st, 5000, 3, "fp64")
    assert (abs(pos) < 1.0).all() and (layer == 1).all()
    assert abs((d * d).sum(axis=1) - 1.0).max() < 1e-12
