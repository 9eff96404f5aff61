"""Loads the in-tree sm_100a library.  There is no CPU fallback: if the library
is missing, or was built from sources other than those beside it (its build
manifest records their SHA-256), every transport entry point raises."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

from . import abi

import os

# SMCRT_B200_LIB selects another build of the same library (e.g. a tuned variant)
LIB_PATH = Path(os.environ.get("SMCRT_B200_LIB", Path(__file__).resolve().parent / "lib" / "libsmcrt_b200.so"))

_lib: C.CDLL | None = None


class SmcrtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"smcrt error {code}: {msg}")
        self.code = code


def _check_provenance() -> None:
    """The in-tree library must have been built from the sources beside it: its
    build manifest records their SHA-256."""
    from . import build
    m = build.manifest_path(LIB_PATH)
    if not m.exists():
        raise RuntimeError(f"{LIB_PATH} has no build manifest ({m.name}): rebuild it with "
                           "`python -m signedmcrt_b200.build`")
    recorded = json.loads(m.read_text()).get("sources", {})
    changed = sorted(k for k, v in build.source_hashes().items() if recorded.get(k) != v)
    if changed:
        raise RuntimeError(f"{LIB_PATH} was built from other sources ({', '.join(changed)} changed): "
                           "rebuild it with `python -m signedmcrt_b200.build`")


def lib() -> C.CDLL:
    """The bound library (loaded once)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m signedmcrt_b200.build` "
                "(the transport runs only on the sm_100a CUDA library; there is no CPU path)")
        if "SMCRT_B200_LIB" not in os.environ:
            _check_provenance()
        _lib = abi.bind(C.CDLL(str(LIB_PATH)))
        v = _lib.smcrt_abi_version()
        if v != abi.ABI_VERSION:
            raise RuntimeError(f"libsmcrt_b200 ABI {v} != expected {abi.ABI_VERSION}")
    return _lib


def check(rc: int) -> None:
    if rc != abi.OK:
        msg = lib().smcrt_last_error()
        raise SmcrtError(rc, msg.decode() if msg else "")
