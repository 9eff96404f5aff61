"""Output side of the transport path: the fluence normalisation, the NRRD / raw
array writers, the detector dump and the checkpoint file, with the file formats
of signedMCRT's writer module (src/writer.f90) so that users can compare files.

Arrays are (nxg, nyg, nzg) and written in Fortran (column-major) order, like the
reference's `write(u) array` of `jmean(nxg, nyg, nzg)`.  The transport tallies in
FP64; `normalise_fluence` and the writers keep FP64 unless `dtype=np.float32`
asks for the reference's `real(sp)` output.
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np


def data_dirs(root: str | Path | None = None) -> Path:
    """The reference's output tree (`directory`, src/setup.f90:55-100): <root>/data
    with jmean/, deposit/, detectors/ and phasor/ (root = the working directory)."""
    base = Path(root if root is not None else os.getcwd()) / "data"
    for sub in ("", "jmean", "deposit", "detectors", "phasor"):
        (base / sub).mkdir(parents=True, exist_ok=True)
    return base


def normalise_fluence(grid, array: np.ndarray, nphotons: int, dtype=None) -> np.ndarray:
    """Fluence per packet and per unit volume (normalise_fluence, src/writer.f90:25-50):
    array * (2 xmax * 2 ymax) / (nphotons * dx * dy * dz).  The factor is formed in
    FP64 as in the reference (xmax is real(wp)); `dtype=np.float32` rounds the result
    to the reference's real(sp) array.  Does not normalise by power."""
    g = grid
    dx = 2.0 * g.xmax / g.nxg
    dy = 2.0 * g.ymax / g.nyg
    dz = 2.0 * g.zmax / g.nzg
    factor = (2.0 * g.xmax * 2.0 * g.ymax) / (float(nphotons) * dx * dy * dz)
    out = np.asarray(array, dtype=np.float64) * factor
    return out.astype(dtype) if dtype is not None else out


def new_file_name(filename: str | Path) -> Path:
    """`name (i).ext` for the first i >= 1 not taken (get_new_file_name, src/writer.f90:188-205)."""
    p = str(filename)
    pos = p.rfind(".")
    i = 1
    while True:
        cand = p[:pos] + f" ({i})" + p[pos:] if pos >= 0 else p + f" ({i})"
        if not Path(cand).exists():
            return Path(cand)
        i += 1


def _target(filename: str | Path, overwrite: bool) -> Path:
    return Path(filename) if overwrite or not Path(filename).exists() else new_file_name(filename)


def _toml_value(v) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        return repr(float(v))
    return '"' + str(v).replace("\\", "\\\\").replace('"', '\\"') + '"'


def nrrd_header(shape, nrrd_type: str, meta: dict | None = None) -> bytes:
    """The header of write_hdr (src/writer.f90:215-247) followed by the metadata
    table as TOML `key = value` lines and the blank line that ends the header."""
    lines = ["NRRD0004", f"type: {nrrd_type}", f"dimension: {len(shape)}",
             "sizes: " + " ".join(str(int(n)) for n in shape), f"space dimension: {len(shape)}",
             "encoding: raw", "endian: little"]
    for k, v in (meta or {}).items():
        lines.append(f"{k} = {_toml_value(v)}")
    return ("\n".join(lines) + "\n\n\n").encode()


def write_nrrd(array: np.ndarray, filename: str | Path, overwrite: bool = False, meta: dict | None = None) -> Path:
    """write_3d_r8_nrrd / write_3d_r4_nrrd (src/writer.f90:249-334): "double" for
    FP64 arrays, "float" for FP32, raw little-endian data in column-major order."""
    a = np.asarray(array)
    if a.ndim != 3:
        raise ValueError("write_nrrd: a 3-D array is required")
    if a.dtype not in (np.float64, np.float32):
        a = a.astype(np.float64)
    path = _target(filename, overwrite)
    with open(path, "wb") as fh:
        fh.write(nrrd_header(a.shape, "double" if a.dtype == np.float64 else "float", meta))
        fh.write(np.asfortranarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes(order="F"))
    return path


def write_raw(array: np.ndarray, filename: str | Path, overwrite: bool = False) -> Path:
    """write_3d_r8_raw / write_3d_r4_raw (src/writer.f90:140-186): the bare stream."""
    a = np.asarray(array)
    path = _target(filename, overwrite)
    with open(path, "wb") as fh:
        fh.write(np.asfortranarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes(order="F"))
    return path


def write_data(array: np.ndarray, filename: str | Path, overwrite: bool = False, meta: dict | None = None) -> Path:
    """Picks the writer from the extension (write_data, src/writer.f90:86-138):
    .nrrd -> NRRD, .raw / .dat -> raw stream, anything else is an error."""
    name = str(filename)
    if ".nrrd" in name:
        return write_nrrd(array, filename, overwrite, meta)
    if ".raw" in name or ".dat" in name:
        return write_raw(array, filename, overwrite)
    raise ValueError("File type not supported!")


def read_nrrd(filename: str | Path) -> tuple[np.ndarray, dict]:
    """Reads a file written by write_nrrd: (array (nx, ny, nz), header fields)."""
    raw = Path(filename).read_bytes()
    end = raw.index(b"\n\n\n")  # last header line, the blank line, the writer's extra newline
    head = raw[:end].decode().splitlines()
    fields = {}
    for line in head[1:]:
        if ": " in line:
            k, v = line.split(": ", 1)
            fields[k] = v
        elif " = " in line:
            k, v = line.split(" = ", 1)
            fields[k] = v
    data = raw[end + 3:]
    shape = tuple(int(x) for x in fields["sizes"].split())
    dt = np.dtype("<f8") if fields["type"] == "double" else np.dtype("<f4")
    arr = np.frombuffer(data[: dt.itemsize * int(np.prod(shape))], dtype=dt).reshape(shape, order="F")
    return arr, fields


def detector_bin_widths(settings) -> list:
    """Bin width of each detector as its init routine sets it (circle maxval/(nbins-1),
    annulus maxval/nbins, camera maxval/(nbins+1); src/detectors/detectors.f90)."""
    out = []
    for d in settings.detectors:
        if d.nbins == 0:
            out.append(1.0)
        elif d.type == "circle":
            out.append(d.maxval / (d.nbins - 1))
        elif d.type == "annulus":
            out.append(d.maxval / d.nbins)
        else:
            out.append(d.maxval / (d.nbins + 1))
    return out


def split_bins(settings, bins: np.ndarray) -> list:
    """The concatenated detector bins of a run, one array per detector
    (nbins + 1 values; a camera's (nbins + 1)^2 as a column-major image)."""
    out, off = [], 0
    for d in settings.detectors:
        n = d.nbins + 1
        if d.type == "camera":
            out.append(np.asarray(bins[off:off + n * n]).reshape((n, n), order="F"))
            off += n * n
        else:
            out.append(np.asarray(bins[off:off + n]))
            off += n
    return out


def write_detected_photons(settings, bins: np.ndarray, directory: str | Path, all_kinds: bool = False) -> list:
    """detector_<i>.dat per detector (write_detected_photons, src/writer.f90:53-84):
    a circle writes `j * bin_wid, data(j)` for j = 1..nbins; the reference writes no
    data for an annulus (the file is created empty) and only warns for a camera.
    `all_kinds=True` also writes annulus bins the same way and a camera's image
    (one row of nbins + 1 counts per line)."""
    directory = Path(directory)
    directory.mkdir(parents=True, exist_ok=True)
    paths = []
    for i, (d, data, bw) in enumerate(zip(settings.detectors, split_bins(settings, bins),
                                          detector_bin_widths(settings)), start=1):
        path = directory / f"detector_{i}.dat"
        with open(path, "w") as fh:
            if d.type == "circle":
                for j in range(1, d.nbins + 1):
                    fh.write(f" {j * bw!r:>24} {float(data[j - 1])!r:>24}\n")
            elif d.type == "annulus" and all_kinds:
                for j in range(1, d.nbins + 1):
                    fh.write(f" {j * bw!r:>24} {float(data[j - 1])!r:>24}\n")
            elif d.type == "camera":
                if all_kinds:
                    for row in data:
                        fh.write(" ".join(repr(float(v)) for v in row) + "\n")
                else:
                    print("Warning not yet implmented!")
        paths.append(path)
    return paths


def checkpoint(toml_filename: str, filename: str | Path, nphotons_run: int, jmean: np.ndarray,
               overwrite: bool = True, dtype=np.float32) -> Path:
    """Checkpoint file of src/writer.f90:336-367: `tomlfile=<input>` and
    `photons_run=<n>` lines, then the raw fluence tally (the reference's real(sp)
    jmean; pass dtype=np.float64 to keep the FP64 tally exactly)."""
    path = _target(filename, overwrite)
    with open(path, "wb") as fh:
        fh.write(f"tomlfile={toml_filename}\n".encode())
        fh.write(f"photons_run={int(nphotons_run)}\n".encode())
        fh.write(np.asfortranarray(np.asarray(jmean, dtype=dtype)).tobytes(order="F"))
    return path


def load_checkpoint(filename: str | Path, shape, dtype=None) -> tuple[str, int, np.ndarray]:
    """Reads a checkpoint: (toml file name, packets run, fluence tally).  The tally
    type is taken from the data length unless given (FP32 as the reference writes
    it, or FP64).  Packet ids are the RNG counter, so a run resumes exactly from
    packet `photons_run` on."""
    raw = Path(filename).read_bytes()
    l1 = raw.index(b"\n")
    l2 = raw.index(b"\n", l1 + 1)
    toml = raw[:l1].decode().split("=", 1)[1]
    nrun = int(raw[l1 + 1:l2].decode().split("=", 1)[1])
    n = int(np.prod(shape))
    if dtype is None:
        nbytes = len(raw) - (l2 + 1)
        if nbytes not in (4 * n, 8 * n):
            raise ValueError(f"checkpoint {filename}: {nbytes} data bytes for {n} cells")
        dtype = np.float32 if nbytes == 4 * n else np.float64
    dt = np.dtype(dtype)
    arr = np.frombuffer(raw[l2 + 1:l2 + 1 + n * dt.itemsize], dtype=dt).reshape(shape, order="F")
    return toml, nrun, arr


def write_positions(moments, nphotons: int, filename: str | Path = "positions.dat") -> Path:
    """positions.dat of test_kernel (src/kernelsMod.f90:439-446): 8 lines of x y z,
    the 1st moments of the positions of scatter events 1-4 times 10 / nphotons,
    then their 2nd moments times 100 / nphotons (mean-free-path units of the
    Scatter_test2 table).  `moments` is the 24 sums of the test kernel: sum of
    positions (4 x 3) then sum of squared positions (4 x 3)."""
    m = np.asarray(moments, dtype=np.float64).reshape(2, 4, 3)
    n = float(nphotons)
    rows = [10.0 * m[0, i] / n for i in range(4)] + [100.0 * m[1, i] / n for i in range(4)]
    p = Path(filename)
    p.write_text("".join(" ".join(f"{v:.17g}" for v in r) + "\n" for r in rows))
    return p


def write_nscatt(nscatt: float, nphotons: int, filename: str | Path = "nscatt.dat") -> Path:
    """nscatt.dat of finalise (src/kernelsMod.f90:596-599): the mean number of
    scatters per packet, read back by Scatter_test1."""
    p = Path(filename)
    p.write_text(f"{float(nscatt) / float(nphotons):.17g}\n")
    return p


def read_table(filename: str | Path) -> np.ndarray:
    """The whitespace-separated numbers of positions.dat / nscatt.dat, one row per line."""
    return np.array([[float(x) for x in line.split()] for line in Path(filename).read_text().splitlines()
                     if line.strip()])
