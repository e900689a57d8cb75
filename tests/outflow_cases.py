"""A small box emptied through an outflow boundary at its floor (shared by
the oracle and GPU outflow tests)."""
import numpy as np

from cases import settling_case
from mfix_dem import params as P


def outflow_case(mass_outflow: bool, intg="EULER", coll="LSD", vy=-1.0, seed=7):
    """Spheres on a lattice just above the floor of a 12x60x12 mm box with
    no floor facet, moving down at about `vy`; the floor y = 0 is an outflow
    boundary (BC_PLANE 'N': the fluid lies north of the boundary cells)
    across the whole floor."""
    case, prm, arr, walls = settling_case(n_side=(5, 4, 5), spacing=1.05, jitter=0.03, vmax=0.05, seed=seed,
                                          intg=intg, coll=coll, nsn=10)
    rng = np.random.default_rng(seed)
    arr["vel"][1] = vy * (1.0 + 0.2 * rng.random(arr["vel"].shape[1]))
    vertex, norm = walls                      # (F, 3, 3), (F, 3)
    keep = [f for f in range(norm.shape[0]) if not (norm[f, 1] > 0.5)]   # drop the floor
    walls = (np.ascontiguousarray(vertex[keep]), np.ascontiguousarray(norm[keep]))
    box = case.domain_hi
    bc = P.outflow_bc(prm, "N", (0.0, 0.0, 0.0), (box[0], 0.0, box[2]), face=0.0, mass_outflow=mass_outflow,
                      vel=[(0.0, -2.0, 0.0)])
    return case, prm, arr, walls, bc
