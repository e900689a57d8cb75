"""Loads libmfixdem.so, the CUDA implementation of the C ABI.

There is no CPU fallback: if the shared object is missing or no CUDA device
is visible, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from . import abi

PKG = Path(__file__).resolve().parent.parent
LIB_PATH = Path(os.environ.get("MFIX_DEM_LIB", PKG / "lib" / "libmfixdem.so"))

_lib = None


class NativeLibraryMissing(RuntimeError):
    pass


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise NativeLibraryMissing(
            f"{LIB_PATH} not found: build it with `python mfix-cfd-dem_b200/build.py` "
            "(this package has no CPU implementation)")
    lib = C.CDLL(str(LIB_PATH))
    abi.bind(lib, "dem_", abi.DEM_ONLY)
    if lib.dem_abi_version() != abi.DEM_ABI_VERSION:
        raise RuntimeError("libmfixdem.so ABI version mismatch")
    _lib = lib
    return lib


def require_cuda():
    """Raises unless a CUDA device is visible to the runtime."""
    try:
        import torch
        ok = torch.cuda.is_available()
    except Exception:
        ok = False
    if not ok:
        raise RuntimeError("no CUDA device: the DEM library runs on the GPU only")
