"""The oracle's dem_upload_state: after a first full upload the constant
arrays (radius, mass, inertia, state, phase) may be NULL, as in the
library, so a parity test can hand both the same motion-only uploads."""
import numpy as np
import pytest

from cases import settling_case, make_system
from oracle_ffi import OracleSystem


def test_motion_only_upload_keeps_the_constants():
    from mfix_dem import abi
    from mfix_dem.system import DemError
    case, prm, arr, walls = settling_case(n_side=(4, 6, 4), spacing=0.98, jitter=0.03)
    fresh = OracleSystem(prm, arr["pos"].shape[1])
    with pytest.raises(DemError) as e:
        fresh.upload_state(arr["pos"], arr["vel"], arr["omega"])
    assert e.value.code == abi.DEM_ERR_ARG
    fresh.close()
    a = make_system(OracleSystem, prm, arr, walls)
    b = make_system(OracleSystem, prm, arr, walls)
    for _ in range(20):
        a.step(1)
        b.step(1)
        s = b.download_state()
        b.upload_state(s["pos"], s["vel"], s["omega"])
    sa, sb = a.download_state(), b.download_state()
    for key in ("pos", "vel", "omega", "state"):
        assert np.array_equal(sa[key], sb[key]), key
    assert a.stats()["n_contacts"] == b.stats()["n_contacts"] > 0
