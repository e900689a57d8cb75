"""B200-native MFiX DEM particle step: host side of the C ABI.

    from mfix_dem import DemSystem, params, load_library
    lib = load_library()
    sys = DemSystem(lib, prm, max_pip)

The compute runs in libmfixdem.so (CUDA, sm_100a); this package only builds
parameters, moves arrays and sequences calls.
"""
from . import abi, params
from ._lib import load as load_library, LIB_PATH
from .system import DemSystem, DemError, BatchSystem

__all__ = ["abi", "params", "load_library", "LIB_PATH", "DemSystem", "DemError", "GpuSystem", "GpuBatch"]


def GpuSystem(prm, max_pip):
    """A DemSystem on the CUDA library (current CUDA device)."""
    from ._lib import require_cuda
    require_cuda()
    return DemSystem(load_library(), prm, max_pip, prefix="dem_")


def GpuBatch(common, limits):
    """A BatchSystem on the CUDA library (current CUDA device)."""
    from ._lib import require_cuda
    require_cuda()
    return BatchSystem(load_library(), common, limits)
