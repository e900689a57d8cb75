"""CPU-side checks of the C ABI: the CUDA library builds and loads, exports
every entry point include/dem_b200.h declares, and its ctypes mirror matches
the header.  No kernel runs here."""
import ctypes as C
import re
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "dem_b200.h"


def header_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dem_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib_path():
    sys.path.insert(0, str(ROOT / "mfix-cfd-dem_b200"))
    from mfix_dem import _lib
    if not _lib.LIB_PATH.exists():
        subprocess.run([sys.executable, str(ROOT / "mfix-cfd-dem_b200" / "build.py")], check=True)
    return _lib.LIB_PATH


def test_library_exports_every_header_symbol(lib_path):
    lib = C.CDLL(str(lib_path))
    missing = [f for f in header_functions() if not hasattr(lib, f)]
    assert not missing, missing
    assert len(header_functions()) >= 30


def test_abi_version_and_struct_sizes(lib_path):
    from mfix_dem import abi, load_library
    lib = load_library()
    assert lib.dem_abi_version() == abi.DEM_ABI_VERSION
    # sizes of the structs as the C compiler lays them out
    src = f'#include "{HEADER}"\n#include <stdio.h>\nint main(){{printf("%zu %zu %zu %zu %zu\\n", sizeof(dem_params), sizeof(dem_stats), sizeof(dem_fluid_grid), sizeof(dem_batch_limits), sizeof(dem_memory));}}'
    exe = ROOT / "oracle" / "_build" / "abi_sizes"
    exe.parent.mkdir(exist_ok=True)
    subprocess.run(["gcc", "-x", "c", "-o", str(exe), "-"], input=src, text=True, check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert sizes == [C.sizeof(abi.DemParams), C.sizeof(abi.DemStats), C.sizeof(abi.DemFluidGrid),
                     C.sizeof(abi.DemBatchLimits), C.sizeof(abi.DemMemory)]


def test_create_without_device_fails_cleanly(lib_path):
    """With no visible GPU the library returns an error code, never a CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from mfix_dem import abi, load_library
    from cases import settling_case
    lib = load_library()
    _, prm, _, _ = settling_case(n_side=(4, 4, 4))
    h = C.c_void_p()
    rc = lib.dem_create(C.byref(prm), 64, C.byref(h))
    assert rc == abi.DEM_ERR_CUDA


def test_gpu_system_refuses_without_cuda():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from mfix_dem import GpuSystem
    from cases import settling_case
    _, prm, arr, _ = settling_case(n_side=(4, 4, 4))
    with pytest.raises(RuntimeError):
        GpuSystem(prm, arr["pos"].shape[1])
