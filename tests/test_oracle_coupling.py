"""CPU checks of the oracle's CFD-DEM coupling (GARG_2012 / Gidaspow / mean
fields) on small cases."""
import math

import numpy as np

from cases import coupled_case, make_coupled
from oracle_ffi import OracleSystem


def test_mean_fields_are_physical_and_deterministic():
    ct = coupled_case()
    s = make_coupled(OracleSystem, ct)
    s.comp_mean_fields()
    ep, rop = s.get_mean_fields()
    case, prm, arr, walls, info, grid, fields = ct
    gi, gj, gk = grid.imax + 2, grid.jmax + 2, grid.kmax + 2
    ep3 = ep.reshape(gk, gj, gi)[1:-1, 1:-1, 1:-1]
    assert np.all(ep3 > 0.0) and np.all(ep3 <= 1.0)
    assert ep3.min() < 0.9            # the bed is there
    s2 = make_coupled(OracleSystem, ct)
    s2.comp_mean_fields()
    ep2, rop2 = s2.get_mean_fields()
    assert np.array_equal(ep, ep2) and np.array_equal(rop, rop2)


def test_drag_opposes_gravity():
    """The upward gas flow gives every particle an upward drag of the order of
    its weight (Gidaspow: Ergun in the bed, Wen-Yu above it)."""
    ct = coupled_case()
    case, prm, arr, walls, info, grid, fields = ct
    s = make_coupled(OracleSystem, ct)
    s.comp_mean_fields()
    s.calc_force()
    fc0, _ = s.download_forces()
    s.drag_gs_des0()
    fc1, _ = s.download_forces()
    drag_y = fc1[1] - fc0[1]
    weight = arr["pmass"] * 9.81
    assert np.all(drag_y > 0.0)
    assert 0.1 < drag_y.mean() / weight.mean() < 10.0
    s.cfnewvalues()
    s.step_coupled(5, 2)


def _faces(lo, d, nc):
    f = [0.0] * (nc + 3)
    f[1] = lo
    f[0] = lo - d
    for i in range(2, nc + 3):
        f[i] = f[i - 1] + d
    return f


def _drag_gas_restated(grid, pos, vel, state, f_gp):
    """DRAG_GS_GAS0's deposition and F_GDS (drag_gs_des0.f:235-497) as plain
    Python loops in the reference's order, from the F_GP the oracle returns:
    cells in IJK order, particles of a cell in ascending index, the eight
    nodes of the cell, then F_GDS per fluid cell."""
    im, jm, km = grid.imax, grid.jmax, grid.kmax
    gi, gj, gk = im + 2, jm + 2, km + 2
    nc = gi * gj * gk
    xe, yn, zt = _faces(0.0, grid.dx, im), _faces(0.0, grid.dy, jm), _faces(0.0, grid.dz, km)

    def cijk(i, j, k):
        return (i - 1) + (j - 1) * gi + (k - 1) * gi * gj

    def fluid(i, j, k):
        return 2 <= i <= im + 1 and 2 <= j <= jm + 1 and 2 <= k <= km + 1

    def search(f, n, x):
        for idx in range(1, n + 3):
            if f[idx - 1] <= x < f[idx]:
                return idx
        return n + 3

    vol = grid.dx * grid.dy * grid.dz
    vol_node = [0.0] * nc
    for k in range(1, km + 2):
        for j in range(1, jm + 2):
            for i in range(1, im + 2):
                fv = lambda a, b, c: vol if fluid(a, b, c) else 0.0  # noqa: E731
                v = 0.125 * (fv(i, j, k) + fv(i + 1, j, k) + fv(i, j + 1, k) + fv(i + 1, j + 1, k))
                v = v + 0.125 * (fv(i, j, k + 1) + fv(i + 1, j + 1, k + 1) + fv(i, j + 1, k + 1)
                                 + fv(i + 1, j, k + 1))
                vol_node[cijk(i, j, k)] = v
    pic = [[] for _ in range(nc)]
    for l in range(pos.shape[1]):
        if state[l] == 0 or state[l] >= 2:     # nonexistent or ghost
            continue
        i = search(xe, im, pos[0, l]); j = search(yn, jm, pos[1, l]); k = search(zt, km, pos[2, l])
        pic[cijk(i, j, k)].append((l, i, j, k))
    am = [0.0] * nc
    bm = [[0.0] * nc for _ in range(3)]
    for k in range(1, gk + 1):
        for j in range(1, gj + 1):
            for i in range(1, gi + 1):
                if not fluid(i, j, k):
                    continue
                for (l, _, _, _) in pic[cijk(i, j, k)]:
                    z0 = (pos[0, l] - xe[i - 1]) / (xe[i] - xe[i - 1])
                    z1 = (pos[1, l] - yn[j - 1]) / (yn[j] - yn[j - 1])
                    z2 = (pos[2, l] - zt[k - 1]) / (zt[k] - zt[k - 1])
                    xx, yy, zz = (1 - z0, z0), (1 - z1, z1), (1 - z2, z2)
                    for kk in range(2):
                        for jj in range(2):
                            for ii in range(2):
                                w = xx[ii] * yy[jj] * zz[kk]
                                node = cijk(i - 1 + ii, j - 1 + jj, k - 1 + kk)
                                ovol = 1.0 / vol_node[node]
                                am[node] = am[node] + f_gp[l] * w * ovol * 1.0
                                for c in range(3):
                                    bm[c][node] = bm[c][node] + f_gp[l] * vel[c, l] * w * ovol * 1.0
    f_gds = [0.0] * nc
    for k in range(1, gk + 1):
        for j in range(1, gj + 1):
            for i in range(1, gi + 1):
                if not fluid(i, j, k):
                    continue
                f = 0.125 * (am[cijk(i, j, k)] + am[cijk(i, j - 1, k)] + am[cijk(i - 1, j - 1, k)]
                             + am[cijk(i - 1, j, k)])
                f = f + 0.125 * (am[cijk(i, j, k - 1)] + am[cijk(i, j - 1, k - 1)]
                                 + am[cijk(i - 1, j - 1, k - 1)] + am[cijk(i - 1, j, k - 1)])
                f_gds[cijk(i, j, k)] = f
    return np.array(f_gds), np.array(am), np.array(bm), np.array(vol_node)


def _moving_case(cells=(4, 10, 4), n=150, ur=1.0):
    ct = coupled_case(cells=cells, n=n)
    ct[5].ur_f_gs = ur
    s = make_coupled(OracleSystem, ct)
    s.comp_mean_fields()
    s.step_coupled(8)          # particles move: DRAG_BM is not trivially zero
    return ct, s


def test_drag_gas_matches_python_restatement():
    """The oracle's DRAG_GS_GAS0 deposition and F_GDS, bit for bit against a
    plain-loop restatement in the reference's order."""
    ct, s = _moving_case()
    f_gds, am, bm, f_gp = s.drag_gs_gas0()
    st = s.download_state()
    rf, ram, rbm, _ = _drag_gas_restated(ct[5], st["pos"], st["vel"], st["state"], f_gp)
    assert np.count_nonzero(am) > 0 and np.count_nonzero(bm[1]) > 0
    assert np.array_equal(am, ram)
    assert np.array_equal(bm, rbm)
    assert np.array_equal(f_gds, rf)


def test_drag_gas_conserves_particle_drag():
    """The node weights of a particle sum to one, so sum DRAG_AM*DES_VOL_NODE
    is the sum of F_GP and sum DRAG_BM(:,c)*DES_VOL_NODE the sum of
    F_GP*V(c); F_GP agrees with DRAG_GS_DES0's (both from DES_DRAG_GP)."""
    ct, s = _moving_case(cells=(6, 16, 6), n=900)
    f_gds, am, bm, f_gp = s.drag_gs_gas0()
    st = s.download_state()
    live = (st["state"] == 1)
    _, _, _, vol_node = _drag_gas_restated(ct[5], st["pos"][:, :1], st["vel"][:, :1],
                                           np.zeros(1, np.int8), f_gp[:1])
    assert np.all(f_gp[live] > 0.0)
    tot = f_gp[live].sum()
    assert abs((am * vol_node).sum() - tot) <= 1e-12 * tot
    for c in range(3):
        ref = (f_gp[live] * st["vel"][c, live]).sum()
        scale = (f_gp[live] * np.abs(st["vel"][c, live])).sum()
        assert abs((bm[c] * vol_node).sum() - ref) <= 1e-12 * scale
    # with UR_F_GS = 1, F_GP does not depend on its previous value: a second
    # call, and a DRAG_GS_DES0 call before it, give the same F_GP
    s.drag_gs_des0()
    f2 = s.drag_gs_gas0()[3]
    assert np.array_equal(f2, f_gp)


def test_drag_gas_under_relaxation():
    """UR_F_GS < 1 relaxes F_GP against the previous call's value."""
    ct, s = _moving_case(ur=0.5)
    f1 = s.drag_gs_gas0()[3]
    f2 = s.drag_gs_gas0()[3]
    f3 = s.drag_gs_gas0()[3]
    live = f1 != 0.0
    assert np.any(live)
    # the same state each time: with the unrelaxed F_GS fixed,
    # F_{k+1} - F_k = 0.5*(F_k - F_{k-1})
    assert not np.array_equal(f1, f2)
    d21, d32 = f2[live] - f1[live], f3[live] - f2[live]
    assert np.all(np.abs(d32 - 0.5 * d21) <= 1e-12 * np.abs(f1[live]))


def _none_case(n=400, cells=(5, 12, 5)):
    ct = coupled_case(cells=cells, n=n, interp="NONE")
    s = make_coupled(OracleSystem, ct)
    s.comp_mean_fields()
    s.step_coupled(6)
    return ct, s


def _cell_of(grid, pos):
    im, jm, km = grid.imax, grid.jmax, grid.kmax
    xe, yn, zt = _faces(0.0, grid.dx, im), _faces(0.0, grid.dy, jm), _faces(0.0, grid.dz, km)

    def search(f, n, x):
        for idx in range(1, n + 3):
            if f[idx - 1] <= x < f[idx]:
                return idx
        return n + 3
    return search(xe, im, pos[0]), search(yn, jm, pos[1]), search(zt, km, pos[2])


def test_none_scheme_matches_python_restatement():
    """COMP_MEAN_FIELDS1, DRAG_GS_GAS1 and DRAG_GS_DES1 without a filter
    (the NONE scheme), bit for bit against plain loops in the reference's
    particle order."""
    ct, s = _none_case()
    case, prm, arr, walls, info, grid, fields = ct
    im, jm, km = grid.imax, grid.jmax, grid.kmax
    gi, gj = im + 2, jm + 2
    nc = gi * gj * (km + 2)
    cijk = lambda i, j, k: (i - 1) + (j - 1) * gi + (k - 1) * gi * gj  # noqa: E731
    fluid = lambda i, j, k: 2 <= i <= im + 1 and 2 <= j <= jm + 1 and 2 <= k <= km + 1  # noqa: E731
    vol = grid.dx * grid.dy * grid.dz
    u, v, w = fields["u_g"], fields["v_g"], fields["w_g"]

    s.comp_mean_fields()
    ep, rop = s.get_mean_fields()
    st = s.download_state()
    pos, vel, state = st["pos"], st["vel"], st["state"]
    rad = arr["radius"]
    rho = grid.ro_s[0]
    sv = [0.0] * nc
    cells = {}
    for l in range(pos.shape[1]):
        if state[l] != 1:
            continue
        cells[l] = _cell_of(grid, pos[:, l])
        r = rad[l]
        sv[cijk(*cells[l])] = sv[cijk(*cells[l])] + ((4.0 / 3.0) * math.pi) * (r * (r * r))
    rop_ref = np.zeros(nc)
    ep_ref = fields["ep_g"].copy()
    for k in range(1, km + 3):
        for j in range(1, gj + 1):
            for i in range(1, gi + 1):
                if fluid(i, j, k):
                    c = cijk(i, j, k)
                    rop_ref[c] = rho * sv[c] / vol
                    ep_ref[c] = 1.0 - min(1.0, 0.0 + rop_ref[c] / rho)
    assert np.array_equal(rop, rop_ref)
    fl = np.array([fluid(i, j, k) for k in range(1, km + 3) for j in range(1, gj + 1) for i in range(1, gi + 1)])
    assert np.array_equal(ep[fl], ep_ref[fl])

    f_gds, bm, f_gp = s.drag_gs_gas1()
    bm_ref = [[0.0] * nc for _ in range(3)]
    fg_ref = [0.0] * nc
    for l, (i, j, k) in cells.items():
        if not fluid(i, j, k):
            continue
        c = cijk(i, j, k)
        weight = 1.0 / vol
        for a in range(3):
            bm_ref[a][c] = bm_ref[a][c] + (f_gp[l] * vel[a, l]) * weight
        fg_ref[c] = fg_ref[c] + f_gp[l] * weight
    assert np.count_nonzero(f_gds) > 0
    assert np.array_equal(bm, np.array(bm_ref))
    assert np.array_equal(f_gds, np.array(fg_ref))

    # DRAG_GS_DES1: the force added is F_GP*(u_cell - v_p), with the gas
    # velocity averaged to the cell centre (FX = FX_BAR = 1/2)
    s.calc_force()
    fc0, _ = s.download_forces()
    s.drag_gs_des1()
    fc1, _ = s.download_forces()
    f_gp2 = s.drag_gs_gas1()[2]        # UR_F_GS = 1: the F_GP DES1 used
    for l, (i, j, k) in list(cells.items())[:60]:
        if not fluid(i, j, k):
            continue
        c = cijk(i, j, k)
        ug = (0.5 * u[cijk(i - 1, j, k)] + 0.5 * u[c], 0.5 * (v[cijk(i, j - 1, k)] + v[c]),
              0.5 * (w[cijk(i, j, k - 1)] + w[c]))
        for a in range(3):
            assert fc1[a, l] == fc0[a, l] + f_gp2[l] * (ug[a] - vel[a, l])


def test_none_scheme_coupled_steps():
    """The coupled step under NONE runs DRAG_GS_DES1 and COMP_MEAN_FIELDS1:
    void fractions stay physical and particles are lifted by the gas."""
    ct, s = _none_case(n=900, cells=(6, 16, 6))
    ep, _ = s.get_mean_fields()
    case, prm, arr, walls, info, grid, fields = ct
    gi, gj, gk = grid.imax + 2, grid.jmax + 2, grid.kmax + 2
    ep3 = ep.reshape(gk, gj, gi)[1:-1, 1:-1, 1:-1]
    assert np.all(ep3 > 0.0) and np.all(ep3 <= 1.0) and ep3.min() < 0.9
    f_gds, bm, f_gp = s.drag_gs_gas1()
    st = s.download_state()
    live = st["state"] == 1
    vol = grid.dx * grid.dy * grid.dz
    assert abs(f_gds.sum() * vol - f_gp[live].sum()) <= 1e-12 * f_gp[live].sum()
