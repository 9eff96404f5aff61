"""Loads the in-tree sm_100a library.  There is no CPU fallback: if the library
is missing, every transport entry point raises."""
from __future__ import annotations

import ctypes as C
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


def lib() -> C.CDLL:
    """The bound library (loaded once)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m signedmcrt_b200.build` "
                "(the transport runs only on the sm_100a CUDA library; there is no CPU path)")
        _lib = abi.bind(C.CDLL(str(LIB_PATH)))
        v = _lib.smcrt_abi_version()
        if v != abi.ABI_VERSION:
            raise RuntimeError(f"libsmcrt_b200 ABI {v} != expected {abi.ABI_VERSION}")
    return _lib


def check(rc: int) -> None:
    if rc != abi.OK:
        msg = lib().smcrt_last_error()
        raise SmcrtError(rc, msg.decode() if msg else "")
