"""Host-side logic on the CPU: TOML parsing (parse_params), presets and the
flattening of an sdf array into the C-ABI tables."""
import numpy as np
import pytest

from signedmcrt_b200 import abi, presets as P, scene as S
from signedmcrt_b200.config import ConfigError, parse_params, parse_table

MIN = {"source": {"name": "point", "position": [0.0, 0.0, 0.0]}, "grid": {}, "geometry": {"geom_name": "scat_test"},
       "output": {}, "simulation": {}}


def test_defaults_follow_parse_params():
    st = parse_table(MIN)
    assert (st.grid.nxg, st.grid.xmax) == (200, 1.0)            # parse.f90:86-91
    assert st.source.nphotons == 1000000                        # parse_source.f90:58
    assert st.simulation.iseed == 123456789                     # parse.f90:202
    assert st.source.annulus_type == "gaussian" and st.source.radius_hi == 0.6
    assert st.geometry.tau == 10.0 and st.geometry.hgg == 0.7


@pytest.mark.parametrize("drop,msg", [("grid", "Need grid table"), ("geometry", "Need geometry table"),
                                      ("output", "Need output table"), ("simulation", "Need simulation table"),
                                      ("source", "Simulation needs Source table")])
def test_missing_tables_raise(drop, msg):
    t = {k: v for k, v in MIN.items() if k != drop}
    with pytest.raises(ConfigError, match=msg):
        parse_table(t)


def test_direction_forms_and_errors():
    t = dict(MIN, source={"name": "pencil", "position": [0, 0, 0], "direction": "-z"})
    assert parse_table(t).source.direction == (0.0, 0.0, -1.0)
    t = dict(MIN, source={"name": "pencil", "position": [0, 0, 0], "direction": [0.0, 1.0, 0.0]})
    assert parse_table(t).source.direction == (0.0, 1.0, 0.0)
    with pytest.raises(ConfigError, match="cardinal"):
        parse_table(dict(MIN, source={"name": "pencil", "position": [0, 0, 0], "direction": "w"}))
    with pytest.raises(ConfigError, match="Need to specify direction"):
        parse_table(dict(MIN, source={"name": "pencil", "position": [0, 0, 0]}))
    with pytest.raises(ConfigError, match="Uniform source requires point1"):
        parse_table(dict(MIN, source={"name": "uniform", "direction": "z"}))


def test_detectors_order_and_validation():
    dets = [{"type": "camera", "layer": 2}, {"type": "annulus", "position": [0, 0, 0], "radius1": 0.1,
                                             "radius2": 0.2}, {"type": "circle", "position": [0, 0, 0],
                                                               "radius1": 0.5, "direction": [0, 0, 2.0]}]
    st = parse_table(dict(MIN, detectors=dets))
    assert [d.type for d in st.detectors] == ["circle", "annulus", "camera"]  # parse_detectors.f90:97-110
    c = st.detectors_c()
    assert tuple(c[0].dir) == (0.0, 0.0, 1.0)  # circle direction normalised
    with pytest.raises(ConfigError, match="Radii are invalid"):
        parse_table(dict(MIN, detectors=[{"type": "annulus", "position": [0, 0, 0], "radius1": 0.3,
                                          "radius2": 0.2}]))
    with pytest.raises(ConfigError, match="Invalid detector type"):
        parse_table(dict(MIN, detectors=[{"type": "square"}]))


def test_parse_file(tmp_path):
    f = tmp_path / "in.toml"
    f.write_text('[source]\nname="annulus"\nposition=[0.0,0.0,0.0]\ndirection="-z"\nannulus_type="tophat"\n'
                 'radius=0.0\nradius_hi=0.5\nbeta=0.0\n[grid]\nnxg=10\n[geometry]\ngeom_name="sphere_water"\n'
                 '[output]\n[simulation]\niseed=7\n')
    st = parse_params(f)
    src = st.source_c()
    assert src.kind == abi.SRC_ANNULUS and src.annulus_type == abi.ANNULUS_TOPHAT and src.radius_hi == 0.5
    assert st.grid.nxg == 10 and st.simulation.iseed == 7
    with pytest.raises(ConfigError, match="no such routine"):
        P.setup_simulation(parse_table(dict(MIN, geometry={"geom_name": "nope"})))


def test_flatten_regions_and_models():
    arr = P.setup_omg_sdf()
    flat = S.FlatScene(arr)
    assert flat.nregions == 2 and flat.nprims == 11
    r0 = flat.c.regions[0]
    assert (r0.first_prim, r0.nprims, r0.op, r0.k) == (0, 10, abi.OP_SMOOTH_UNION, 0.09)
    assert flat.c.prims[0].kind == abi.TORUS
    b = flat.c.prims[10]
    assert b.kind == abi.BOX and tuple(b.params[:3]) == (1.0, 1.0, 1.0)  # box_init halves the lengths
    t = flat.c.prims[0].transform
    assert (t[3][0], t[3][1], t[3][2]) == (0.0, 0.0, 0.7)  # invert(translate(0,0,-.7))


def test_benchmark_scenes_shape():
    lv = P.layered_vessels()
    assert len(lv) == 8 and [s.kind for s in lv[:4]] == [abi.CAPSULE] * 4
    depth, _ = P.vessel_layout()
    assert np.all((depth >= 0.1) & (depth <= 0.5))
    assert P.box_slab()[0].opt.albedo == pytest.approx(10 / 10.1)
    sw = P.sphere_water()
    assert sw[1].opt.n == 1.33 and sw[0].opt.hgg == 0.85
    st = P.benchmark_settings("layered_vessels")
    assert len(st.detectors) == 10 and st.detectors[0].layer == 8
