"""Output formats of the writer module (src/writer.f90) on the CPU: fluence
normalisation, NRRD and raw arrays, file naming, detector dump, checkpoints."""
import numpy as np
import pytest

from signedmcrt_b200 import writer as W
from signedmcrt_b200.config import DetectorCfg, parse_table

MIN = {"source": {"name": "point", "position": [0.0, 0.0, 0.0]}, "grid": {"nxg": 4, "nyg": 5, "nzg": 6,
       "xmax": 1.0, "ymax": 2.0, "zmax": 0.5}, "geometry": {"geom_name": "scat_test"}, "output": {}, "simulation": {}}


def test_normalise_fluence_factor():
    st = parse_table(MIN)
    g = st.grid
    a = np.arange(4 * 5 * 6, dtype=np.float64).reshape(4, 5, 6, order="F")
    out = W.normalise_fluence(g, a, 1000)
    dx, dy, dz = 2 * 1.0 / 4, 2 * 2.0 / 5, 2 * 0.5 / 6
    np.testing.assert_allclose(out, a * (2 * 1.0 * 2 * 2.0) / (1000 * dx * dy * dz), rtol=1e-15)
    assert W.normalise_fluence(g, a, 1000, dtype=np.float32).dtype == np.float32


@pytest.mark.parametrize("dtype,kind", [(np.float64, "double"), (np.float32, "float")])
def test_nrrd_round_trip_and_header(tmp_path, dtype, kind):
    a = np.random.default_rng(1).random((3, 4, 5)).astype(dtype)
    meta = {"grid_data": "fluence map", "nphotons": 100, "source": "point"}
    p = W.write_nrrd(a, tmp_path / "f.nrrd", meta=meta)
    raw = p.read_bytes()
    head = raw.split(b"\n")
    assert head[:7] == [b"NRRD0004", f"type: {kind}".encode(), b"dimension: 3", b"sizes: 3 4 5",
                        b"space dimension: 3", b"encoding: raw", b"endian: little"]
    assert b'grid_data = "fluence map"' in raw and b"nphotons = 100" in raw
    # the data follow the header in column-major order
    n = a.size * a.itemsize
    assert raw[-n:] == np.asfortranarray(a).tobytes(order="F")
    b, fields = W.read_nrrd(p)
    assert np.array_equal(a, b) and fields["type"] == kind


def test_new_file_names_and_dispatch(tmp_path):
    a = np.zeros((2, 2, 2))
    p1 = W.write_data(a, tmp_path / "x.nrrd")
    p2 = W.write_data(a, tmp_path / "x.nrrd")
    assert p1.name == "x.nrrd" and p2.name == "x (1).nrrd"
    assert W.write_data(a, tmp_path / "x.nrrd", overwrite=True).name == "x.nrrd"
    r = W.write_data(np.arange(8.0).reshape(2, 2, 2, order="F"), tmp_path / "y.raw")
    assert np.array_equal(np.frombuffer(r.read_bytes(), dtype="<f8"), np.arange(8.0))
    assert W.write_data(a, tmp_path / "z.dat").stat().st_size == 64
    with pytest.raises(ValueError, match="File type not supported"):
        W.write_data(a, tmp_path / "z.png")


def test_detector_dump(tmp_path):
    st = parse_table(MIN)
    st.detectors = [DetectorCfg("circle", nbins=5, maxval=2.0), DetectorCfg("annulus", nbins=4, maxval=1.0),
                    DetectorCfg("camera", nbins=2, maxval=1.0)]
    bins = np.arange(6 + 5 + 9, dtype=np.float64)
    parts = W.split_bins(st, bins)
    assert [p.shape for p in parts] == [(6,), (5,), (3, 3)]
    assert W.detector_bin_widths(st) == [2.0 / 4, 1.0 / 4, 1.0 / 3]
    paths = W.write_detected_photons(st, bins, tmp_path / "d")
    rows = [list(map(float, line.split())) for line in paths[0].read_text().splitlines()]
    assert len(rows) == 5 and rows[0] == [0.5, 0.0] and rows[4] == [2.5, 4.0]   # j * bin_wid, data(j)
    assert paths[1].read_text() == ""                                            # the reference writes no annulus data
    paths = W.write_detected_photons(st, bins, tmp_path / "e", all_kinds=True)
    assert len(paths[1].read_text().splitlines()) == 4
    assert len(paths[2].read_text().splitlines()) == 3


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_checkpoint_round_trip(tmp_path, dtype):
    a = np.random.default_rng(2).random((4, 3, 2))
    p = W.checkpoint("in.toml", tmp_path / "c.ckpt", 12345, a, dtype=dtype)
    assert p.read_bytes().startswith(b"tomlfile=in.toml\nphotons_run=12345\n")
    toml, nrun, b = W.load_checkpoint(p, a.shape)
    assert toml == "in.toml" and nrun == 12345 and b.dtype == dtype
    np.testing.assert_array_equal(b, a.astype(dtype))


def test_positions_and_nscatt_files(tmp_path):
    """positions.dat (src/kernelsMod.f90:439-446): 8 rows, first moments x 10 / N then
    second moments x 100 / N; nscatt.dat (:596-599): mean scatters per packet."""
    m = np.arange(24, dtype=np.float64)
    p = W.write_positions(m, 1000, tmp_path / "positions.dat")
    rows = W.read_table(p)
    assert rows.shape == (8, 3)
    np.testing.assert_allclose(rows[:4], 10.0 * m[:12].reshape(4, 3) / 1000, rtol=1e-15)
    np.testing.assert_allclose(rows[4:], 100.0 * m[12:].reshape(4, 3) / 1000, rtol=1e-15)
    q = W.write_nscatt(5750000.0, 100000, tmp_path / "nscatt.dat")
    assert W.read_table(q)[0, 0] == 57.5
