"""ctypes loader for the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It builds oracle/_build/liboracle*.so on first use when the
shared object is missing and a compiler is available.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT / "mfix-cfd-dem_b200"))

from mfix_dem import abi  # noqa: E402
from mfix_dem.system import DemSystem  # noqa: E402

_LIBS = {}


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def host_cpu_key() -> str:
    """A short key for this host's CPU (model name and feature flags), so a
    -march=native build made on one host is never loaded on another."""
    import hashlib
    text = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    text += line
                if line.strip() == "":
                    break
    except OSError:
        text = os.uname().machine
    return hashlib.sha1(text.encode()).hexdigest()[:12]


def source_key() -> str:
    """A short key for the oracle's sources, so a stale build is not loaded."""
    import hashlib
    h = hashlib.sha1()
    for f in (HERE / "dem_oracle.cpp", HERE / "dem_oracle.h", ROOT / "include" / "dem_b200.h"):
        h.update(f.read_bytes())
    return h.hexdigest()[:10]


def native_path() -> Path:
    """The OpenMP timing build with -march=native for this host's CPU and
    the current sources, compiled here on first use (a few seconds of g++)."""
    d = HERE / "_build" / f"native_{host_cpu_key()}_{source_key()}"
    path = d / "liboracle_omp.so"
    if not path.exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "native", f"NATIVE_DIR={d}"], check=True)
    return path


def load(openmp: bool = False, native: bool = False):
    name = ("liboracle_native.so" if native else "liboracle_omp.so") if openmp else "liboracle.so"
    if name in _LIBS:
        return _LIBS[name]
    if openmp and native:
        path = native_path()
    else:
        path = HERE / "_build" / name
        if not path.exists():
            build()
    lib = C.CDLL(str(path))
    abi.bind(lib, "orc_")
    lib.orc_set_threads.restype = C.c_int
    lib.orc_set_threads.argtypes = [C.c_void_p, C.c_int32]
    lib.orc_download_facet_bins.restype = C.c_int
    lib.orc_download_facet_bins.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                            C.c_int32, C.POINTER(C.c_int32)]
    lib.orc_download_edge_flags.restype = C.c_int
    lib.orc_download_edge_flags.argtypes = [C.c_void_p, C.POINTER(C.c_int8)]
    _LIBS[name] = lib
    return lib


class OracleSystem(DemSystem):
    """The CPU restatement behind the same host interface as the CUDA library."""

    def __init__(self, params, max_pip, openmp=False, threads=1, native=False):
        super().__init__(load(openmp, native), params, max_pip, prefix="orc_")
        if threads != 1:
            self._lib.orc_set_threads(self._h, int(threads))

    def facet_bins(self):
        import numpy as np
        nc = C.c_int32()
        self._lib.orc_download_facet_bins(self._h, None, None, 0, C.byref(nc))
        start = np.empty(nc.value + 1, dtype=np.int32)
        self._lib.orc_download_facet_bins(self._h, start.ctypes.data_as(C.POINTER(C.c_int32)), None, 0, C.byref(nc))
        ids = np.empty(max(int(start[-1]), 1), dtype=np.int32)
        self._lib.orc_download_facet_bins(self._h, start.ctypes.data_as(C.POINTER(C.c_int32)),
                                          ids.ctypes.data_as(C.POINTER(C.c_int32)), ids.shape[0], C.byref(nc))
        return start, ids[: int(start[-1])]

    def edge_flags(self, nf):
        import numpy as np
        fl = np.zeros((nf, 4), dtype=np.int8)
        self._lib.orc_download_edge_flags(self._h, fl.ctypes.data_as(C.POINTER(C.c_int8)))
        return fl
