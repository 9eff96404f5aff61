"""The C-ABI boundary without a GPU: the library loads, exports every function
include/smcrt.h declares, and the ctypes mirror has the header's struct layout."""
import ctypes as C
import json
import os
import re
import subprocess
from pathlib import Path

import pytest

from signedmcrt_b200 import abi

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "smcrt.h"


def declared_functions(header: Path = HEADER) -> list[str]:
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:[\w\*\s]+?)\b(smcrt_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_expected_entry_points():
    names = declared_functions()
    for must in ("smcrt_create", "smcrt_run", "smcrt_run_device", "smcrt_replay", "smcrt_run_batched",
                 "smcrt_destroy", "smcrt_last_error", "smcrt_eval_sdf", "smcrt_calc_normal", "smcrt_fresnel"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from signedmcrt_b200 import _lib
    if not _lib.LIB_PATH.exists():
        from signedmcrt_b200 import build
        build.build()
    lib = C.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(abi.SIGNATURES) <= set(declared_functions())
    abi.bind(lib)
    assert lib.smcrt_abi_version() == abi.ABI_VERSION


def test_no_device_is_an_error_not_a_crash():
    """Without a visible GPU, creation reports SMCRT_ERR_NO_DEVICE (or succeeds on a GPU host)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from signedmcrt_b200 import _lib, presets as P, transport as T
    st = P.benchmark_settings("box_slab")
    with pytest.raises(_lib.SmcrtError) as e:
        T.Transport(P.setup_simulation(st), st)
    assert e.value.code == abi.ERR_NO_DEVICE


STRUCTS = {
    "smcrt_prim": (abi.Prim, ["kind", "nmods", "transform", "params", "mods", "mod_params"]),
    "smcrt_region": (abi.Region, ["first_prim", "nprims", "op", "layer_id", "k", "mus", "mua", "hgg", "n"]),
    "smcrt_scene": (abi.Scene, ["nregions", "nprims", "regions", "prims"]),
    "smcrt_grid": (abi.Grid, ["nxg", "nyg", "nzg", "xmax", "ymax", "zmax"]),
    "smcrt_source": (abi.Source, ["kind", "annulus_type", "pos", "dir", "point1", "point2", "point3", "radius",
                                  "radius_hi", "beta", "z_inset"]),
    "smcrt_detector": (abi.Detector, ["kind", "layer", "nbins", "pos", "dir", "r1", "r2", "maxval", "p2", "p3"]),
    "smcrt_options": (abi.Options, ["kernel", "precision", "end_early", "block_size", "blocks_per_sm",
                                    "max_trace_steps", "eps", "normal_h", "instance", "timeout_ms", "stream",
                                    "private_stream", "tally_copies", "scene_memory", "variance", "nearest_cache",
                                    "shared_fluence", "group_order", "reserved"]),
    "smcrt_stats": (abi.Stats, ["nscatt", "packets", "sdf_evals", "voxel_segments", "trace_steps", "scatters",
                                "fresnel_events", "reflections", "kills_step_cap", "kills_error", "rng_draws",
                                "moments", "kernel_ms", "device_status", "h2d_bytes", "d2h_bytes",
                                "variance_overflows", "reserved2"]),
    "smcrt_packet_state": (abi.PacketState, ["pos", "dir", "weight", "layer", "nscatt", "ndraws", "flags"]),
    "smcrt_region_optics": (abi.RegionOptics, ["mus", "mua", "hgg", "n"]),
    "smcrt_tuning": (abi.Tuning, ["tally_copies", "shared_bins", "packets_per_s", "trials", "block_size",
                                  "slots_per_thread", "ctas_per_sm", "nearest_cache",
                                  "shared_fluence", "group_order", "reserved"]),
}


def test_struct_layout_matches_header(tmp_path):
    """Compiles a C probe against include/smcrt.h and compares sizes/offsets with ctypes."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "smcrt.h"', "int main(void){", 'printf("{");']
    first = True
    for name, (_, fields) in STRUCTS.items():
        sep = "" if first else ","
        first = False
        lines.append(f'printf("{sep}\\"{name}\\":{{\\"size\\":%zu", sizeof({name}));')
        for f in fields:
            lines.append(f'printf(",\\"{f}\\":%zu", offsetof({name}, {f}));')
        lines.append('printf("}");')
    lines += ['printf("}\\n");', "return 0;}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    layout = json.loads(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    for name, (cls, fields) in STRUCTS.items():
        assert C.sizeof(cls) == layout[name]["size"], name
        for f in fields:
            assert getattr(cls, f).offset == layout[name][f], (name, f)


def test_render_checks_its_arguments_before_the_device():
    """smcrt_render rejects bad sizes and extents with SMCRT_ERR_ARG whether or not a
    GPU is visible; without one a valid call reports SMCRT_ERR_NO_DEVICE."""
    import torch
    from signedmcrt_b200 import _lib, presets as P, transport as T
    arr = P.setup_egg()
    for samples, extent in (((0, 4, 4), (1.0, 1.0, 1.0)), ((4, 70000, 4), (1.0, 1.0, 1.0)),
                            ((4, 4, 4), (1.0, float("nan"), 1.0))):
        with pytest.raises(_lib.SmcrtError) as e:
            T.render(arr, samples, extent)
        assert e.value.code == abi.ERR_ARG
    with pytest.raises(_lib.SmcrtError) as e:
        T.render_device(arr, (4, 4, 4), (1.0, 1.0, 1.0), 0)
    assert e.value.code == abi.ERR_ARG  # null image pointer
    if not torch.cuda.is_available():
        with pytest.raises(_lib.SmcrtError) as e:
            T.render(arr, (4, 4, 4), (1.0, 1.0, 1.0))
        assert e.value.code == abi.ERR_NO_DEVICE


def test_library_provenance_is_checked_on_load(monkeypatch):
    """The in-tree library carries a manifest of the sources it was built from;
    the loader accepts it only while those sources are unchanged."""
    from signedmcrt_b200 import _lib, build
    if "SMCRT_B200_LIB" in os.environ:
        pytest.skip("another build of the library is selected")
    _lib._check_provenance()  # the library built for this test run
    real = build.source_hashes()
    some = sorted(real)[0]
    monkeypatch.setattr(build, "source_hashes", lambda: dict(real, **{some: "0" * 64}))
    with pytest.raises(RuntimeError, match="built from other sources"):
        _lib._check_provenance()


def test_group_order_is_checked_before_the_device():
    """options.group_order takes 0 (library choice), SMCRT_ORDER_WALK_LAST or
    SMCRT_ORDER_INTERACT_LAST; anything else is SMCRT_ERR_ARG before any device
    is touched."""
    from signedmcrt_b200 import _lib, presets as P, transport as T
    st = P.benchmark_settings("box_slab")
    for bad in (-1, 3):
        with pytest.raises(_lib.SmcrtError) as e:
            T.Transport(P.setup_simulation(st), st, group_order=bad)
        assert e.value.code == abi.ERR_ARG
    assert (abi.ORDER_WALK_LAST, abi.ORDER_INTERACT_LAST) == (1, 2)


def test_trace_step_cap_is_bounded_before_the_device():
    """The per-flight step count shares its slot word with the nearest-region
    cache (21 bits): a larger max_trace_steps is refused with SMCRT_ERR_ARG
    before any device is touched."""
    from signedmcrt_b200 import _lib, presets as P, transport as T
    st = P.benchmark_settings("box_slab")
    with pytest.raises(_lib.SmcrtError) as e:
        T.Transport(P.setup_simulation(st), st, max_trace_steps=(1 << 21))
    assert e.value.code == abi.ERR_ARG
