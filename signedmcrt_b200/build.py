"""Build the sm_100a transport library in-tree: signedmcrt_b200/lib/libsmcrt_b200.so.

Each kernel variant (transport precision x kernel kind) is its own translation
unit, so the variants compile in parallel; the host API and the probes are two
more.  Objects are cached under signedmcrt_b200/_build and rebuilt when any
source or header is newer, or differs from the one the library was built from.
Next to the library, libsmcrt_b200.build.json records the SHA-256 of every source
and header it was compiled from, the nvcc version and the flags; the loader
(`_lib.py`) refuses an in-tree library whose sources have changed since.
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import time
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libsmcrt_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                     "--expt-relaxed-constexpr"]

VARIANTS = [("float", "f32", k) for k in (0, 1, 2)] + [("double", "f64", k) for k in (0, 1, 2)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the sm_100a library needs the CUDA toolkit")


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cu*")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "smcrt.h"]


def manifest_path(lib: Path) -> Path:
    return lib.with_name(lib.stem + ".build.json")


def source_hashes() -> dict[str, str]:
    """SHA-256 of every source and header the library is compiled from, by path
    relative to the repository root."""
    return {str(d.relative_to(ROOT)): hashlib.sha256(d.read_bytes()).hexdigest() for d in _deps()}


def _manifest_matches(lib: Path) -> bool:
    m = manifest_path(lib)
    if not lib.exists() or not m.exists():
        return False
    try:
        return json.loads(m.read_text()).get("sources") == source_hashes()
    except (OSError, ValueError):
        return False


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _units() -> list[tuple[Path, list[str]]]:
    units = []
    for rtype, tag, k in VARIANTS:
        obj = BUILD / f"kernels_{tag}_{k}.o"
        # the FP64 variants are the accuracy mode: no FMA contraction, so their
        # arithmetic follows the CPU restatement operation for operation
        fmad = ["--fmad=false"] if tag == "f64" else []
        units.append((obj, fmad + ["-DSMCRT_R=" + rtype, "-DSMCRT_TAG=" + tag, f"-DSMCRT_K={k}",
                                   "-c", str(CSRC / "smcrt_kernels.cu"), "-o", str(obj)]))
    for name in ("smcrt_probes", "smcrt_api"):
        obj = BUILD / f"{name}.o"
        units.append((obj, ["-c", str(CSRC / f"{name}.cu"), "-o", str(obj)]))
    # the render follows the CPU restatement operation for operation in FP64
    obj = BUILD / "smcrt_render.o"
    units.append((obj, ["--fmad=false", "-c", str(CSRC / "smcrt_render.cu"), "-o", str(obj)]))
    return units


def build(verbose: bool = False, jobs: int | None = None, extra_flags: list[str] | None = None) -> Path:
    """Compile (if stale) and link the library; returns its path."""
    BUILD.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    deps = _deps()
    exe = nvcc()
    flags = NVCC_FLAGS + (extra_flags or [])
    # every unit when the sources differ from the recorded ones (mtimes alone can
    # miss a change, e.g. files copied with their times kept)
    fresh = _manifest_matches(LIB)
    todo = [(obj, args) for obj, args in _units() if not fresh or _stale(obj, deps)]

    def run(item):
        obj, args = item
        cmd = [exe] + flags + ["-I", str(ROOT / "include")] + args
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {obj.name}:\n{r.stdout}\n{r.stderr}")
        return obj

    if todo:
        with ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            list(ex.map(run, todo))
    objs = [obj for obj, _ in _units()]
    if _stale(LIB, objs):
        cmd = [exe] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if todo or not manifest_path(LIB).exists():
        ver = subprocess.run([exe, "--version"], capture_output=True, text=True).stdout.strip().splitlines()
        manifest_path(LIB).write_text(json.dumps({
            "library": LIB.name, "sources": source_hashes(), "nvcc": ver[-1] if ver else "",
            "flags": flags, "units_compiled": [obj.name for obj, _ in todo],
            "built_utc": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}, indent=1) + "\n")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
