"""A small box filled through a mass-inflow boundary at its top (shared by
the oracle and GPU inflow tests)."""
import numpy as np

from cases import settling_case
from mfix_dem import abi
from mfix_dem import params as P


def inflow_case(spare=160, pi_count=2, pi_factor=12.0, vy=-2.0, d_in=0.9e-3, intg="EULER", coll="LSD",
                outflow=False, seed=11):
    """A 12x60x12 mm box with a few settling spheres and `spare` NONEXISTENT
    slots; its top y = 60 mm (no top facet) is a mass-inflow boundary
    (BC_PLANE 'S': the fluid lies south of the boundary cells) over
    x, z in [0.5, 11.5] mm seeding `pi_count` spheres of diameter `d_in`
    every `pi_factor` steps at velocity (0, vy, 0).  With `outflow` the floor
    (no floor facet) is also a MASS_OUTFLOW boundary."""
    case, prm, arr, walls = settling_case(n_side=(4, 3, 4), spacing=1.05, jitter=0.03, vmax=0.05, seed=seed,
                                          intg=intg, coll=coll, nsn=10)
    n0 = arr["pos"].shape[1]
    n = n0 + spare
    out = {}
    for k, v in arr.items():
        v = np.asarray(v)
        if v.ndim == 2:
            w = np.zeros((v.shape[0], n), dtype=v.dtype)
            w[:, :n0] = v
        else:
            w = np.zeros(n, dtype=v.dtype)
            w[:n0] = v
        out[k] = w
    out["state"][n0:] = abi.DEM_STATE_NONEXISTENT
    out["phase"][n0:] = 1
    out["pmass"][n0:] = 1.0
    if outflow:
        # the initial spheres leave through the floor
        out["vel"][1, :n0] = vy
    else:
        # lift the initial spheres off the floor a little
        out["pos"][1, :n0] += 5e-3
    vertex, norm = walls                      # (F, 3, 3), (F, 3)
    drop = lambda f: norm[f, 1] < -0.5 or (outflow and norm[f, 1] > 0.5)   # the top (and the floor)
    keep = [f for f in range(norm.shape[0]) if not drop(f)]
    walls = (np.ascontiguousarray(vertex[keep]), np.ascontiguousarray(norm[keep]))
    box = case.domain_hi
    rho = case.ro_s0[0]
    bc = P.inflow_bc(prm, "S", (0.5e-3, box[1], 0.5e-3), (box[0] - 0.5e-3, box[1], box[2] - 0.5e-3),
                     d_p0=[d_in], ro_s0=[rho], vel=[(0.0, vy, 0.0)], pi_count=pi_count, pi_factor=pi_factor,
                     min_radius=0.5 * d_in, max_radius=max(0.5 * d_in, float(np.max(arr["radius"]))),
                     face=box[1], layout_seed=seed)
    obc = None
    if outflow:
        obc = P.outflow_bc(prm, "N", (0.0, 0.0, 0.0), (box[0], 0.0, box[2]), face=0.0, mass_outflow=True,
                           vel=[(0.0, -2.0, 0.0)])
    return case, prm, out, walls, bc, obc
