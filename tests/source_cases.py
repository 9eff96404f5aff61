"""Source and detector configurations shared by the CPU oracle tests and the GPU
tests: every emitter of src/photon.f90 on the box_slab geometry, and the source
known-answer setups of signedMCRT's own test/photon/test_photon.f90."""
from signedmcrt_b200 import presets as P
from signedmcrt_b200.config import DetectorCfg, parse_table

# name -> [source] table on the box_slab geometry (2 cm box, grid +-1 cm), every
# launch inside the box
BOX_SOURCES = {
    "pencil": {"name": "pencil", "position": [0.1, -0.2, 0.99999], "direction": "-z"},
    "point": {"name": "point", "position": [0.0, 0.1, 0.0]},
    "uniform": {"name": "uniform", "direction": "-z", "point1": [-0.5, -0.5, 0.99999], "point2": [1.0, 0.0, 0.0],
                "point3": [0.0, 1.0, 0.0]},
    # circular: the disc is rotated onto the direction and moved by MINUS the
    # position (photon.f90:262-265), so this disc is centred at z = +0.99999
    "circular": {"name": "circular", "position": [0.0, 0.0, -0.99999], "direction": "-z", "radius": 0.5},
    "annulus_tophat": {"name": "annulus", "annulus_type": "tophat", "radius": 0.1, "radius_hi": 0.5, "beta": 10.0,
                       "position": [0.0, 0.0, 0.0], "direction": "-z"},
    "annulus_gaussian": {"name": "annulus", "annulus_type": "gaussian", "radius": 0.0, "radius_hi": 0.5,
                         "beta": 0.0, "position": [0.0, 0.0, 0.0], "direction": "-z"},
    "focus": {"name": "focus", "position": [0.0, 0.0, 0.0], "direction": "-z"},
}


def box_source_settings(name: str, nphotons: int = 20000, circle_detector: bool = False):
    src = dict(BOX_SOURCES[name])
    src["nphotons"] = nphotons
    table = {"source": src,
             "grid": {"nxg": 100, "nyg": 100, "nzg": 100, "xmax": 1.0, "ymax": 1.0, "zmax": 1.0},
             "geometry": {"geom_name": "box_slab"}, "output": {}, "simulation": {"iseed": 5}}
    st = parse_table(table)
    if name.startswith("annulus") or name == "focus":
        st.source.z_inset = 1e-5  # start just inside the box top (the reference's 1e-8 is below FP32 spacing)
    if circle_detector:
        # packets leaving through the top end on the ambient box's face at z = 1.001
        st.detectors = [DetectorCfg("circle", position=(0.0, 0.0, 1.001), direction=(0.0, 0.0, 1.0), layer=2,
                                    radius1=0.6, nbins=20, maxval=0.6)]
    return st, P.setup_simulation(st)


def kat_settings(kind: str):
    """The source setups of test/photon/test_photon.f90 (Uniform_src :64-115,
    Point_src :117-156, circular_src :158-203, Pencil_src :205-244)."""
    if kind == "uniform":
        src = {"name": "uniform", "position": [0.0, 0.0, 0.0], "direction": [1.0, 0.0, 0.0],
               "point1": [-7.5, -1.0, -1.0], "point2": [0.0, 2.0, 0.0], "point3": [0.0, 0.0, 2.0]}
        half = 7.5
    elif kind in ("point", "pencil"):
        src = {"name": kind, "position": [0.0, 0.5, -0.25], "direction": [1.0, 0.0, 0.0]}
        half = 1.0
    elif kind == "circular":
        src = {"name": "circular", "position": [1.0, 1.0, 1.0], "direction": [0.0, 0.0, -1.0], "radius": 2.5}
        half = 1.0
    else:
        raise ValueError(kind)
    st = parse_table({"source": src, "grid": {"nxg": 200, "nyg": 200, "nzg": 200, "xmax": half, "ymax": half,
                                              "zmax": half},
                      "geometry": {"geom_name": "scat_test"}, "output": {}, "simulation": {"iseed": 12345678}})
    return st, P.setup_simulation(st)


def check_kat(kind: str, pos):
    """The position checks of test_photon.f90 for `kind` on (n, 3) launch positions."""
    import numpy as np
    if kind == "uniform":  # :99-113
        assert np.all(pos[:, 0] == -7.5)
        assert np.all((pos[:, 1] >= -1.0) & (pos[:, 1] <= 1.0))
        assert np.all((pos[:, 2] >= -1.0) & (pos[:, 2] <= 1.0))
    elif kind in ("point", "pencil"):  # :142-154, :230-242
        assert np.all(pos[:, 0] == 0.0) and np.all(pos[:, 1] == 0.5) and np.all(pos[:, 2] == -0.25)
    elif kind == "circular":  # :195-201
        r = np.sqrt(((pos + 1.0) ** 2).sum(axis=1))
        assert np.all((r <= 2.5) | (pos[:, 2] == -1.0)), r.max()
