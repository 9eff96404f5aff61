"""The reference's kernel entry points (module `kernels`, src/kernelsMod.f90:7) over
the B200 transport: `pathlength_scatter(input_file)`, `weight_scatter(input_file)`
and `test_kernel(input_file, end_early)`.

Each one does what the Fortran routine does around its packet loop -- parse the
TOML input (`setup`, :453-546), run every packet, then `finalise` (:548-633):
print the mean number of scatters, normalise the fluence, write
`data/jmean/<output.fluence>` with the run's metadata and the detector files.
Like the reference's serial build, `nscatt.dat` (mean scatters per packet,
:596-599) goes to the working directory, and `test_kernel` writes
`positions.dat` there too (:439-446): the files the reference's end-to-end
tests read.  The packet loop itself is the GPU kernel behind the C ABI.

Checkpoints (`[simulation] checkpoint_every_n`, `checkpoint_file`) are written in
the reference's layout every `checkpoint_every_n` packets, with the FP64 tally
(the reference stores its FP32 one; both load).  Unlike the reference,
`load_checkpoint = true` resumes exactly: packet ids are the RNG counter, so the
packets after the checkpoint are the ones an uninterrupted run would have made.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import writer
from .config import Settings, parse_params
from .presets import setup_simulation
from .transport import Transport, render


@dataclass
class KernelRun:
    jmean: np.ndarray          # raw FP64 path-length tally (nxg, nyg, nzg), Fortran order
    fluence: np.ndarray        # normalised fluence (normalise_fluence)
    bins: np.ndarray           # concatenated detector bins
    nscatt: float              # total scatters (the reference's reduction variable)
    stats: dict
    files: list = field(default_factory=list)


def _add_stats(total: dict | None, st: dict) -> dict:
    if total is None:
        return dict(st)
    out = {}
    for k, v in st.items():
        if k in ("device_status",):
            out[k] = total[k] | v
        else:
            out[k] = total[k] + v
    return out


def run_kernel(settings: Settings, kernel: str, *, end_early: bool = False, input_file: str = "",
               root: str | Path | None = None, precision: str = "fp32", write: bool = True,
               verbose: bool = True) -> KernelRun:
    """The body shared by the three entry points, from parsed settings."""
    st = settings
    arr = setup_simulation(st)
    nphotons = int(st.source.nphotons)
    seed = int(st.simulation.iseed)
    sim = st.simulation
    base = writer.data_dirs(root) if write else None
    files = []
    if st.output.render_geom:  # setup, src/kernelsMod.f90:531-536
        if verbose:
            print("Rendering geometry to file")
        image = render_geometry(arr, st)
        if write:
            files.append(writer.write_data(image, base / st.output.render, overwrite=True))
    with Transport(arr, st, kernel=kernel, precision=precision, end_early=end_early) as tr:
        every = int(sim.checkpoint_every_n)
        chunked = write and 0 < every < nphotons
        if not chunked and not sim.load_checkpoint:
            res = tr.run(nphotons, seed)
            jmean, bins, stats = res.jmean, res.bins, res.stats
        else:
            import torch  # device buffers for the packet-range runs
            jm = torch.zeros(tr.ncell, dtype=torch.float64, device="cuda")
            bins_t = torch.zeros(max(tr.nbins, 1), dtype=torch.float64, device="cuda")
            done = 0
            ckpt = Path(base if base is not None else ".") / sim.checkpoint_file
            if sim.load_checkpoint:
                _, done, prev = writer.load_checkpoint(ckpt, tr.shape)
                jm.copy_(torch.from_numpy(prev.reshape(-1, order="F").copy()))
            stats = None
            while done < nphotons:
                count = min(every if every > 0 else nphotons, nphotons - done)
                st_chunk = tr.run_device(done, count, seed, jm.data_ptr(), bins_t.data_ptr() if tr.nbins else None,
                                         stats=True)
                stats = _add_stats(stats, st_chunk)
                done += count
                if chunked and done % every == 0 and done < nphotons:
                    host = jm.cpu().numpy().reshape(tr.shape, order="F")
                    files.append(writer.checkpoint(input_file, ckpt, done, host, overwrite=True,
                                                   dtype=np.float64))
            torch.cuda.synchronize()
            jmean = jm.cpu().numpy().reshape(tr.shape, order="F")
            bins = bins_t.cpu().numpy()[: tr.nbins]
            stats = stats or {}
    nscatt = float(stats.get("nscatt", np.nan))
    if verbose and np.isfinite(nscatt):
        print("Average # of scatters per photon:", nscatt / nphotons)
    fluence = writer.normalise_fluence(st.grid, jmean, nphotons)
    if write:
        meta = {"grid_data": "fluence map",
                "real_size": f"{st.grid.xmax:.7g} {st.grid.ymax:.7g} {st.grid.zmax:.7g}",
                "nphotons": nphotons, "source": st.source.name,
                "experiment": st.dict.get("experiment", "")}
        files.append(writer.write_data(fluence, base / "jmean" / st.output.fluence, st.output.overwrite, meta))
        if st.detectors:
            files += writer.write_detected_photons(st, bins, base / "detectors")
        cwd = Path(root) if root is not None else Path.cwd()
        if np.isfinite(nscatt):
            files.append(writer.write_nscatt(nscatt, nphotons, cwd / "nscatt.dat"))
        if kernel == "test":
            files.append(writer.write_positions(stats["moments"], nphotons, cwd / "positions.dat"))
    return KernelRun(jmean, fluence, bins, nscatt, stats, files)


def render_geometry(array, settings: Settings) -> np.ndarray:
    """render_vec (src/sdfs/sdf_base.f90:287-299): the scene rendered on a
    render_size voxel grid spanning the fluence grid's half-widths."""
    g = settings.grid
    return render(array, settings.output.render_size, (g.xmax, g.ymax, g.zmax))


def pathlength_scatter(input_file: str | Path, **kw) -> KernelRun:
    """Analog-absorption transport with the path-length fluence tally
    (pathlength_scatter, src/kernelsMod.f90:165-333)."""
    return run_kernel(parse_params(input_file), "pathlength", input_file=str(input_file), **kw)


def weight_scatter(input_file: str | Path, **kw) -> KernelRun:
    """Implicit capture with Russian roulette, absorbed weight tallied at each
    interaction (weight_scatter, src/kernelsMod.f90:12-163)."""
    return run_kernel(parse_params(input_file), "weight", input_file=str(input_file), **kw)


def test_kernel(input_file: str | Path, end_early: bool = False, **kw) -> KernelRun:
    """Scatter-order position moments for the end-to-end tests (test_kernel,
    src/kernelsMod.f90:335-448); `end_early` kills packets after the 4th scatter."""
    return run_kernel(parse_params(input_file), "test", end_early=end_early, input_file=str(input_file), **kw)
