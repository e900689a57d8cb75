// coupling.cu -- CFD-DEM coupling: drag and mean fields (K6, K7, K8).
//
// Replaces, for DES_INTERP_SCHEME = 'GARG_2012' on a uniform Cartesian fluid
// grid without cut cells:
//   PARTICLES_IN_CELL (model/des/particles_in_cell.f:20-234, PIC_SEARCH
//     347-370): fluid cell of every particle and per-cell particle lists;
//   DRAG_GS_DES0 (model/des/drag_gs_des0.f:22-219, DRAG_INTERPOLATION
//     507-566) with DES_DRAG_GP (model/des/drag_gp_des.f:29-260, Model A),
//     DRAG_GIDASPOW (model/drag_gs.f:536-598) and C_DS_SN (model/drag_mod.f:54);
//   COMP_MEAN_FIELDS0 (model/des/comp_mean_fields0.f:6-466, DRAG_WEIGHTFACTOR
//     478-530) and CALC_EPG_DES (model/des/calc_epg_des.f:19-205).
// Fluid cells use MFiX's IJK with one ghost layer (i fastest).  The node
// deposition is a gather: each node adds the contributions of the particles
// of its (up to) 8 cells in IJK order, each cell's particles in ascending
// index, which is the order in which the reference's cell loop adds them, so
// ROP_S and EP_G come out bit-identical.  The drag uses pow(), whose last
// bit may differ from the host's libm.
#include "dem_internal.cuh"

#include <cmath>

using namespace demb;

struct Gas {
  dem_fluid_grid g;
  int gi2, gj2, gk2, ncell, M;
  double vol, pi;
  double* xe = nullptr; double* yn = nullptr; double* zt = nullptr;   // faces 0..nc+2
  double* ep_g = nullptr; double* u_g = nullptr; double* v_g = nullptr; double* w_g = nullptr;
  double* p_force = nullptr;   // (3, ncell) or null
  double* vol_surr = nullptr;  // ncell
  double* rop_s = nullptr;     // (M, ncell)
  double* rops_node = nullptr; // (M, ncell)
  double* vol_node = nullptr;  // ncell: DES_VOL_NODE
  double* drag_am = nullptr;   // ncell: DRAG_AM per node
  double* drag_bm = nullptr;   // (3, ncell): DRAG_BM per node
  double* f_gds = nullptr;     // ncell: F_GDS per cell
  int* pijk = nullptr;         // (n, 4): i, j, k, ijk (1-based), 0 = none
  double* f_gp = nullptr;      // n
  int* pic_cnt = nullptr; int* pic_start = nullptr; int* pic_list = nullptr;
  bool have_mean = false;
};

namespace demb {

struct GasDev {  // by-value kernel view
  int imax, jmax, kmax, gi2, gj2, gk2, ncell, M, no_k, drag_model;
  double vol, pi, ro_g, mu_g, ur_f_gs, usr_d_p0;
  double ro_s[MAXP];
  const double *xe, *yn, *zt;
};

__device__ __forceinline__ int gijk(const GasDev& G, int i, int j, int k) {
  return (i - 1) + (j - 1) * G.gi2 + (k - 1) * G.gi2 * G.gj2;
}
__device__ __forceinline__ bool gfluid(const GasDev& G, int i, int j, int k) {
  return i >= 2 && i <= G.imax + 1 && j >= 2 && j <= G.jmax + 1 &&
         (G.no_k ? k == 1 : (k >= 2 && k <= G.kmax + 1));
}

// PIC_SEARCH: the first idx in [1, nc+2] with f[idx-1] <= x < f[idx]
// (faces increase), nc+3 when none; found by bisection.
__device__ __forceinline__ int face_search(const double* f, int nc, double x) {
  if (!(x >= f[0]) || !(x < f[nc + 2])) return nc + 3;
  int lo = 0, hi = nc + 2;  // f[lo] <= x < f[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (f[mid] <= x) lo = mid; else hi = mid;
  }
  return hi;
}

__global__ void k_pic_locate(DevParams p, GasDev G, double4* __restrict__ pos4, double4* __restrict__ vel4,
                             double4* __restrict__ omg4, int8_t* __restrict__ state, int* __restrict__ pijk,
                             int* __restrict__ cnt, double* __restrict__ fc, double* __restrict__ tow,
                             int* __restrict__ wall_fid, DevErr* __restrict__ err) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= p.n) return;
  int* pj = pijk + 4 * (size_t)l;
  if (state[l] == DEM_STATE_NONEXISTENT) { pj[0] = pj[1] = pj[2] = pj[3] = 0; return; }
  const double4 x = pos4[l];
  const int i = face_search(G.xe, G.imax, x.x);
  const int j = face_search(G.yn, G.jmax, x.y);
  const int k = G.no_k ? 1 : face_search(G.zt, G.kmax, x.z);
  if (!(i >= 1 && i <= G.gi2 && j >= 1 && j <= G.gj2 && k >= 1 && k <= G.gk2)) {
    // outside the fluid grid: DELETE_PARTICLE (particles_in_cell.f:170-180)
    pos4[l] = make_double4(0.0, 0.0, 0.0, 0.0);
    vel4[l] = make_double4(0.0, 0.0, 0.0, 3.4028234663852886e38);
    omg4[l] = make_double4(0.0, 0.0, 0.0, 0.0);
    for (int a = 0; a < 3; ++a) { fc[(size_t)a * p.n + l] = 0.0; tow[(size_t)a * p.n + l] = 0.0; }
    for (int s = 0; s < p.cmax; ++s) wall_fid[(size_t)l * p.cmax + s] = -1;
    state[l] = DEM_STATE_NONEXISTENT;
    atomicAdd(&err->rogue_removed, 1ull);
    pj[0] = pj[1] = pj[2] = pj[3] = 0;
    return;
  }
  const int c = gijk(G, i, j, k);
  pj[0] = i; pj[1] = j; pj[2] = k; pj[3] = c + 1;
  if (state[l] < DEM_STATE_NORMAL_GHOST) atomicAdd(&cnt[c], 1);
}

__global__ void k_pic_scatter(int n, const int8_t* __restrict__ state, const int* __restrict__ pijk,
                              const int* __restrict__ start, int* __restrict__ fill, int* __restrict__ list) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n || state[l] == DEM_STATE_NONEXISTENT || state[l] >= DEM_STATE_NORMAL_GHOST) return;
  const int c = pijk[4 * (size_t)l + 3] - 1;
  list[start[c] + atomicAdd(&fill[c], 1)] = l;
}

__global__ void k_pic_sort(int ncell, const int* __restrict__ start, int* __restrict__ list) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int s = start[c], e = start[c + 1];
  for (int a = s + 1; a < e; ++a) {
    const int v = list[a];
    int b = a - 1;
    while (b >= s && list[b] > v) { list[b + 1] = list[b]; --b; }
    list[b + 1] = v;
  }
}

// Trilinear weights of a point in fluid cell (i,j,k), node (ii,jj,kk) of
// the cell's 2x2x2 stencil (DRAG_WEIGHTFACTOR / DRAG_INTERPOLATION).
__device__ __forceinline__ void cell_weights(const GasDev& G, int i, int j, int k, double x, double y, double z,
                                             double w[2][2][2]) {
  const double dxx = G.xe[i] - G.xe[i - 1], dyy = G.yn[j] - G.yn[j - 1];
  const double z0 = (x - G.xe[i - 1]) / dxx, z1 = (y - G.yn[j - 1]) / dyy;
  const double xx[2] = {1 - z0, z0}, yy[2] = {1 - z1, z1};
  if (G.no_k) {
    for (int jj = 0; jj < 2; ++jj) for (int ii = 0; ii < 2; ++ii) w[0][jj][ii] = xx[ii] * yy[jj];
  } else {
    const double dzz = G.zt[k] - G.zt[k - 1];
    const double z2 = (z - G.zt[k - 1]) / dzz;
    const double zz[2] = {1 - z2, z2};
    for (int kk = 0; kk < 2; ++kk) for (int jj = 0; jj < 2; ++jj) for (int ii = 0; ii < 2; ++ii)
      w[kk][jj][ii] = xx[ii] * yy[jj] * zz[kk];
  }
}

__device__ __forceinline__ double drag_gidaspow(double epg, double mug, double rog, double ropg, double vrel,
                                                double dpm) {
  const double re = mug > 0.0 ? dpm * vrel * ropg / mug : 1.0e32;
  if (re == 0.0) return 0.0;
  if (epg <= 0.8) return 150.0 * (1.0 - epg) * mug / (epg * (dpm * dpm)) + 1.75 * rog * vrel / dpm;
  const double cd = re <= 1000.0 ? 24.0 * (1.0 + 0.15 * pow(re, 0.687)) / (re + SMALL_NUMBER) : 0.44;
  return 0.75 * cd * vrel * ropg * pow(epg, -2.65) / dpm;
}

// The single-sphere user drag of DEM_DRAG_SINGLE_SPHERE (tests/dem/DEM06:
// usr_drag.f, usr_mod.f Re and Cd): 0.75*(RO_g*|u|/d_p)*Cd(Re) with
// Re = RO_g*d_ref*|u|/MU_g and Cd = (24/Re)*(1 + 0.15*Re**0.687), the
// exponent a default-real literal widened to double.
__device__ __forceinline__ double drag_single_sphere(double mug, double rog, double vrel, double dpm, double dref) {
  const double re = (rog * dref * vrel) / mug;
  double cd = 0.0;
  if (re > 0.0) cd = (24.0 / re) * (1.0 + 0.15 * pow(re, (double)0.687f));
  return 0.75 * (rog * vrel / dpm) * cd;
}

// Gas velocity at a particle of fluid cell (i,j,k): staggered face
// velocities averaged to the cell's 2x2x2 node stencil, interpolated with the
// trilinear weights, which are returned too (drag_gs_des0.f:117-170 and
// 313-361, DRAG_INTERPOLATION drag_gs_des0.f:507-566).
__device__ __forceinline__ void gas_velocity(const GasDev& G, int i, int j, int k, const double4& X,
                                             const double* __restrict__ u_g, const double* __restrict__ v_g,
                                             const double* __restrict__ w_g, double velfp[3], double w[2][2][2]) {
  const double avg = G.no_k ? 0.5 : 0.25;
  const int iw = i - 1, js = j - 1, kb = G.no_k ? 1 : k - 1;
  cell_weights(G, i, j, k, X.x, X.y, X.z, w);
  velfp[0] = velfp[1] = velfp[2] = 0.0;
  for (int kk = 0; kk < (G.no_k ? 1 : 2); ++kk)
    for (int jj = 0; jj < 2; ++jj)
      for (int ii = 0; ii < 2; ++ii) {
        const int I = iw + ii, J = js + jj, K = kb + kk;
        const int c = gijk(G, I, J, K), ipjk = gijk(G, I + 1, J, K), ijpk = gijk(G, I, J + 1, K),
                  ipjpk = gijk(G, I + 1, J + 1, K);
        double v0 = avg * (u_g[c] + u_g[ijpk]);
        double v1 = avg * (v_g[c] + v_g[ipjk]);
        double v2;
        if (!G.no_k) {
          const int ijpkp = gijk(G, I, J + 1, K + 1), ipjkp = gijk(G, I + 1, J, K + 1), ijkp = gijk(G, I, J, K + 1);
          v0 = v0 + avg * (u_g[ijkp] + u_g[ijpkp]);
          v1 = v1 + avg * (v_g[ijkp] + v_g[ipjkp]);
          v2 = avg * (w_g[c] + w_g[ijpk] + w_g[ipjk] + w_g[ipjpk]);
        } else {
          v2 = 0.0;
        }
        const double wt = w[kk][jj][ii];
        velfp[0] = velfp[0] + v0 * wt;
        velfp[1] = velfp[1] + v1 * wt;
        if (!G.no_k) velfp[2] = velfp[2] + v2 * wt;
      }
}

// DES_DRAG_GP (drag_gp_des.f:97-257, Model A, Gidaspow): the relaxed F_GP
// of a particle of radius r with velocity V in gas of void fraction epg;
// PVOL through *pvol.
__device__ __forceinline__ double relaxed_fgp(const GasDev& G, double epg, double r, const double velfp[3],
                                              const double4& V, double f_old, double* pvol) {
  const double vs[3] = {velfp[0] - V.x, velfp[1] - V.y, velfp[2] - V.z};
  const double vrel = sqrt(dot3(vs, vs));
  const double dpm = 2.0 * r;
  const double dga = G.drag_model == DEM_DRAG_SINGLE_SPHERE
                         ? drag_single_sphere(G.mu_g, G.ro_g, vrel, dpm, G.usr_d_p0)
                         : drag_gidaspow(epg, G.mu_g, G.ro_g, G.ro_g * epg, vrel, dpm);
  *pvol = ((4.0 / 3.0) * G.pi) * (r * (r * r));
  const double fgs = dga * *pvol;
  return (1.0 - G.ur_f_gs) * f_old + G.ur_f_gs * fgs;
}

// DES_DRAG_GP per particle of a fluid cell.  ADD_FC (DRAG_GS_DES0):
// FC += F_GP*(u_g@p - v_p) + P_FORCE*PVOL as well; without it only F_GP is
// updated (the first half of DRAG_GS_GAS0, whose per-particle F_GP does not
// depend on the deposition order).
template <bool ADD_FC>
__global__ void k_drag(DevParams p, GasDev G, const double4* __restrict__ pos4, const double4* __restrict__ vel4,
                       const int8_t* __restrict__ state, const int* __restrict__ pijk,
                       const double* __restrict__ ep_g, const double* __restrict__ u_g,
                       const double* __restrict__ v_g, const double* __restrict__ w_g,
                       const double* __restrict__ p_force, double* __restrict__ f_gp, double* __restrict__ fc) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= p.n) return;
  const int8_t st = state[l];
  if (st == DEM_STATE_NONEXISTENT || st >= DEM_STATE_NORMAL_GHOST) return;
  const int i = pijk[4 * (size_t)l], j = pijk[4 * (size_t)l + 1], k = pijk[4 * (size_t)l + 2];
  if (!gfluid(G, i, j, k)) return;
  const double4 X = pos4[l], V = vel4[l];
  double w[2][2][2], velfp[3];
  gas_velocity(G, i, j, k, X, u_g, v_g, w_g, velfp, w);
  const int ijk = gijk(G, i, j, k);
  double pvol;
  const double fg = relaxed_fgp(G, ep_g[ijk], X.w, velfp, V, f_gp[l], &pvol);
  f_gp[l] = fg;
  if (!ADD_FC) return;
  const double vp[3] = {V.x, V.y, V.z};
  const size_t n = (size_t)p.n;
  for (int c = 0; c < 3; ++c) fc[c * n + l] = fc[c * n + l] + fg * (velfp[c] - vp[c]);
  if (p_force)
    for (int c = 0; c < 3; ++c) fc[c * n + l] = fc[c * n + l] + p_force[3 * (size_t)ijk + c] * pvol;
}

// DRAG_GS_GAS0 deposition as a gather per node: the node's cells in
// ascending IJK, their particles in PIC order, as the reference's scatter
// adds them; DRAG_AM += F_GP*W/DES_VOL_NODE, DRAG_BM(:,c) += F_GP*V(c)*W/
// DES_VOL_NODE (statistical weight 1).
__global__ void k_drag_node(GasDev G, const double4* __restrict__ pos4, const double4* __restrict__ vel4,
                            const int* __restrict__ pic_start, const int* __restrict__ pic_list,
                            const double* __restrict__ f_gp, const double* __restrict__ vol_node,
                            double* __restrict__ drag_am, double* __restrict__ drag_bm) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ni = G.imax + 1, nj = G.jmax + 1, nk = G.no_k ? 1 : G.kmax + 1;
  if (t >= ni * nj * nk) return;
  const int I = t % ni + 1, J = (t / ni) % nj + 1, K = t / (ni * nj) + 1;
  const int node = gijk(G, I, J, K);
  const double ovol = 1.0 / vol_node[node];
  double am = 0.0, bm[3] = {0.0, 0.0, 0.0};
  for (int k = K; k <= (G.no_k ? K : K + 1); ++k)
    for (int j = J; j <= J + 1; ++j)
      for (int i = I; i <= I + 1; ++i) {
        if (!gfluid(G, i, j, k)) continue;
        const int c = gijk(G, i, j, k);
        const int ii = I - (i - 1), jj = J - (j - 1), kk = G.no_k ? 0 : K - (k - 1);
        for (int q = pic_start[c]; q < pic_start[c + 1]; ++q) {
          const int np = pic_list[q];
          const double4 X = pos4[np], V = vel4[np];
          double w[2][2][2];
          cell_weights(G, i, j, k, X.x, X.y, X.z, w);
          const double wt = w[kk][jj][ii], fg = f_gp[np];
          am = am + fg * wt * ovol;
          bm[0] = bm[0] + fg * V.x * wt * ovol;
          bm[1] = bm[1] + fg * V.y * wt * ovol;
          bm[2] = bm[2] + fg * V.z * wt * ovol;
        }
      }
  drag_am[node] = am;
  for (int c = 0; c < 3; ++c) drag_bm[(size_t)c * G.ncell + node] = bm[c];
}

// F_GDS per cell: the mean of the DRAG_AM of the cell's nodes, in the
// reference's order (drag_gs_des0.f:451-494); zero outside the fluid.
__global__ void k_fgds(GasDev G, const double* __restrict__ drag_am, double* __restrict__ f_gds) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.ncell) return;
  const int i = c % G.gi2 + 1, j = (c / G.gi2) % G.gj2 + 1, k = c / (G.gi2 * G.gj2) + 1;
  if (!gfluid(G, i, j, k)) { f_gds[c] = 0.0; return; }
  const double avf = G.no_k ? 0.25 : 0.125;
  double f = avf * (drag_am[c] + drag_am[gijk(G, i, j - 1, k)] + drag_am[gijk(G, i - 1, j - 1, k)] +
                    drag_am[gijk(G, i - 1, j, k)]);
  if (!G.no_k)
    f = f + avf * (drag_am[gijk(G, i, j, k - 1)] + drag_am[gijk(G, i, j - 1, k - 1)] +
                   drag_am[gijk(G, i - 1, j - 1, k - 1)] + drag_am[gijk(G, i - 1, j, k - 1)]);
  f_gds[c] = f;
}

// ---- DES_INTERP_SCHEME = NONE: the ...1 routines without a filter ------

// CALC_CELL_CENTER_GAS_VEL (drag_gs_des1.f:313-370) on a uniform grid
// (FX = FX_BAR = 1/2, set_geometry.f:344-345); (i,j,k) is a fluid cell.
__device__ __forceinline__ void cell_center_vel(const GasDev& G, int i, int j, int k,
                                                const double* __restrict__ u_g, const double* __restrict__ v_g,
                                                const double* __restrict__ w_g, double v[3]) {
  const int ijk = gijk(G, i, j, k);
  v[0] = 0.5 * u_g[gijk(G, i - 1, j, k)] + 0.5 * u_g[ijk];       // AVG_X_E
  v[1] = 0.5 * (v_g[gijk(G, i, j - 1, k)] + v_g[ijk]);           // AVG_Y_N
  v[2] = G.no_k ? 0.0 : 0.5 * (w_g[gijk(G, i, j, k - 1)] + w_g[ijk]);   // AVG_Z_T
}

__device__ __forceinline__ double sphere_vol(const GasDev& G, double r) {
  return ((4.0 / 3.0) * G.pi) * (r * (r * r));
}

// DRAG_GS_DES1 without a filter (drag_gs_des1.f:34-160, Model A, not
// explicitly coupled), per NORMAL particle: cell-centre gas velocity, F_GP
// by DES_DRAG_GP, FC += F_GP*(u_g - v_p) + P_FORCE*PVOL; F_GP = 0 outside the
// fluid.  Without ADD_FC (the F_GP half of DRAG_GS_GAS1) only F_GP of
// particles in fluid cells changes.
template <bool ADD_FC>
__global__ void k_drag1(DevParams p, GasDev G, const double4* __restrict__ pos4, const double4* __restrict__ vel4,
                        const int8_t* __restrict__ state, const int* __restrict__ pijk,
                        const double* __restrict__ ep_g, const double* __restrict__ u_g,
                        const double* __restrict__ v_g, const double* __restrict__ w_g,
                        const double* __restrict__ p_force, double* __restrict__ f_gp, double* __restrict__ fc) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= p.n || state[l] != DEM_STATE_NORMAL) return;
  const int i = pijk[4 * (size_t)l], j = pijk[4 * (size_t)l + 1], k = pijk[4 * (size_t)l + 2];
  if (!gfluid(G, i, j, k)) {
    if (ADD_FC) f_gp[l] = 0.0;
    return;
  }
  const double4 X = pos4[l], V = vel4[l];
  double velfp[3];
  cell_center_vel(G, i, j, k, u_g, v_g, w_g, velfp);
  const int ijk = gijk(G, i, j, k);
  double pvol;
  const double fg = relaxed_fgp(G, ep_g[ijk], X.w, velfp, V, f_gp[l], &pvol);
  f_gp[l] = fg;
  if (!ADD_FC) return;
  const double vp[3] = {V.x, V.y, V.z};
  const size_t n = (size_t)p.n;
  for (int c = 0; c < 3; ++c) fc[c * n + l] = fc[c * n + l] + fg * (velfp[c] - vp[c]);
  if (p_force)
    for (int c = 0; c < 3; ++c) fc[c * n + l] = fc[c * n + l] + p_force[3 * (size_t)ijk + c] * pvol;
}

// DRAG_GS_GAS1 deposition without a filter, per cell: its NORMAL particles in
// ascending index (the reference's particle loop restricted to the cell),
// DRAG_BM(IJK,:) += F_GP*V/VOL, F_GDS(IJK) += F_GP/VOL; zero outside the fluid.
__global__ void k_gas1_cell(GasDev G, const double4* __restrict__ vel4, const int8_t* __restrict__ state,
                            const int* __restrict__ pic_start, const int* __restrict__ pic_list,
                            const double* __restrict__ f_gp, double* __restrict__ f_gds,
                            double* __restrict__ drag_bm) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.ncell) return;
  const int i = c % G.gi2 + 1, j = (c / G.gi2) % G.gj2 + 1, k = c / (G.gi2 * G.gj2) + 1;
  double f = 0.0, bm[3] = {0.0, 0.0, 0.0};
  if (gfluid(G, i, j, k)) {
    const double weight = 1.0 / G.vol;
    for (int q = pic_start[c]; q < pic_start[c + 1]; ++q) {
      const int np = pic_list[q];
      if (state[np] != DEM_STATE_NORMAL) continue;
      const double lforce = f_gp[np];
      const double4 V = vel4[np];
      bm[0] = bm[0] + (lforce * V.x) * weight;
      bm[1] = bm[1] + (lforce * V.y) * weight;
      bm[2] = bm[2] + (lforce * V.z) * weight;
      f = f + lforce * weight;
    }
  }
  f_gds[c] = f;
  for (int a = 0; a < 3; ++a) drag_bm[(size_t)a * G.ncell + c] = bm[a];
}

// COMP_MEAN_FIELDS1 with FILTER_SIZE = 0 (comp_mean_fields1.f:46-104) and
// CALC_EPG_DES, per cell: SOLVOLINC = sum of PVOL of its NORMAL particles in
// ascending index, ROP_S = RO_S*SOLVOLINC/VOL and EP_G on fluid cells.
__global__ void k_mean_fields1(GasDev G, const double4* __restrict__ pos4, const uint8_t* __restrict__ phase,
                               const int8_t* __restrict__ state, const int* __restrict__ pic_start,
                               const int* __restrict__ pic_list, double* __restrict__ rop_s,
                               double* __restrict__ ep_g) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.ncell) return;
  const int i = c % G.gi2 + 1, j = (c / G.gi2) % G.gj2 + 1, k = c / (G.gi2 * G.gj2) + 1;
  const bool fl = gfluid(G, i, j, k);
  double sv[MAXP];
  for (int m = 0; m < G.M; ++m) sv[m] = 0.0;
  if (fl)
    for (int q = pic_start[c]; q < pic_start[c + 1]; ++q) {
      const int np = pic_list[q];
      if (state[np] != DEM_STATE_NORMAL) continue;
      const int m = phase[np];
      sv[m] = sv[m] + sphere_vol(G, pos4[np].w);
    }
  double sum_eps = 0.0;
  for (int m = 0; m < G.M; ++m) {
    const double r = fl ? G.ro_s[m] * sv[m] / G.vol : 0.0;
    rop_s[(size_t)m * G.ncell + c] = r;
    sum_eps = sum_eps + r / G.ro_s[m];
  }
  if (fl) ep_g[c] = 1.0 - fmin(1.0, sum_eps);
}

// COMP_MEAN_FIELDS0 node deposition as a gather over the node's cells.
__global__ void k_node_deposit(GasDev G, const double4* __restrict__ pos4, const double4* __restrict__ vel4,
                               const uint8_t* __restrict__ phase, const int* __restrict__ pic_start,
                               const int* __restrict__ pic_list, double* __restrict__ rops_node) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ni = G.imax + 1, nj = G.jmax + 1, nk = G.no_k ? 1 : G.kmax + 1;
  if (t >= ni * nj * nk) return;
  const int I = t % ni + 1, J = (t / ni) % nj + 1, K = t / (ni * nj) + 1;
  const int node = gijk(G, I, J, K);
  double acc[MAXP];
  for (int m = 0; m < G.M; ++m) acc[m] = 0.0;
  for (int k = K; k <= (G.no_k ? K : K + 1); ++k)
    for (int j = J; j <= J + 1; ++j)
      for (int i = I; i <= I + 1; ++i) {
        if (!gfluid(G, i, j, k)) continue;
        const int c = gijk(G, i, j, k);
        const int ii = I - (i - 1), jj = J - (j - 1), kk = G.no_k ? 0 : K - (k - 1);
        for (int q = pic_start[c]; q < pic_start[c + 1]; ++q) {
          const int np = pic_list[q];
          const double4 X = pos4[np];
          double w[2][2][2];
          cell_weights(G, i, j, k, X.x, X.y, X.z, w);
          const double temp1 = w[kk][jj][ii] * vel4[np].w;
          const int m = phase[np];
          acc[m] = acc[m] + temp1;
        }
      }
  for (int m = 0; m < G.M; ++m) rops_node[(size_t)m * G.ncell + node] = acc[m];
}

// Node -> cell averaging, normalisation and CALC_EPG_DES, per cell.
__global__ void k_cell_fields(GasDev G, const double* __restrict__ vol_surr, const double* __restrict__ rops_node,
                              double* __restrict__ rop_s, double* __restrict__ ep_g) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.ncell) return;
  const int II = c % G.gi2 + 1, JJ = (c / G.gi2) % G.gj2 + 1, KK = c / (G.gi2 * G.gj2) + 1;
  const int ni = G.imax + 1, nj = G.jmax + 1, nk = G.no_k ? 1 : G.kmax + 1;
  double acc[MAXP];
  for (int m = 0; m < G.M; ++m) acc[m] = 0.0;
  for (int K = (G.no_k ? KK : KK - 1); K <= KK; ++K)
    for (int J = JJ - 1; J <= JJ; ++J)
      for (int I = II - 1; I <= II; ++I) {
        if (I < 1 || I > ni || J < 1 || J > nj || K < 1 || K > nk) continue;
        const int node = gijk(G, I, J, K);
        const double vs = vol_surr[node];
        if (vs == 0.0) continue;
        for (int m = 0; m < G.M; ++m) {
          const double dens = rops_node[(size_t)m * G.ncell + node] / vs;
          acc[m] = acc[m] + dens * G.vol;
        }
      }
  if (gfluid(G, II, JJ, KK)) {
    double sum_eps = 0.0;
    for (int m = 0; m < G.M; ++m) {
      if (acc[m] > 0.0) acc[m] = acc[m] / G.vol;
      sum_eps = sum_eps + acc[m] / G.ro_s[m];
    }
    ep_g[c] = 1.0 - fmin(1.0, sum_eps);
  }
  for (int m = 0; m < G.M; ++m) rop_s[(size_t)m * G.ncell + c] = acc[m];
}

// CALC_DES_BEDHEIGHT (des_granular_temperature.f:201-267) partial sums:
// thread per fluid cell in IJK order, its (EP_S*h*VOL, EP_S*VOL) per phase
// when ROP_S > 0, added over the block in a fixed tree order; the host adds
// the blocks in order.  part[(block * M + m) * 2 + {0, 1}].
constexpr int BED_T = 256;
__global__ void k_bed_partials(GasDev G, const double* __restrict__ rop_s, double* __restrict__ part) {
  __shared__ double sn[BED_T], sd[BED_T];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = c < G.ncell ? (c / G.gi2) % G.gj2 + 1 : 1;
  const double hcell = 0.5 * (G.yn[j] + G.yn[j - 1]);
  for (int m = 0; m < G.M; ++m) {
    double a = 0.0, b = 0.0;
    if (c < G.ncell) {
      const double r = rop_s[(size_t)m * G.ncell + c];
      if (r > 0.0) {
        const double ep = r / G.ro_s[m];
        a = ep * hcell * G.vol;
        b = ep * G.vol;
      }
    }
    sn[threadIdx.x] = a;
    sd[threadIdx.x] = b;
    __syncthreads();
    for (int s = BED_T / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) { sn[threadIdx.x] += sn[threadIdx.x + s]; sd[threadIdx.x] += sd[threadIdx.x + s]; }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      part[((size_t)blockIdx.x * G.M + m) * 2] = sn[0];
      part[((size_t)blockIdx.x * G.M + m) * 2 + 1] = sd[0];
    }
    __syncthreads();
  }
}

static GasDev gas_view(dem_handle* h) {
  Gas* s = h->gas;
  GasDev G;
  G.imax = s->g.imax; G.jmax = s->g.jmax; G.kmax = s->g.kmax;
  G.gi2 = s->gi2; G.gj2 = s->gj2; G.gk2 = s->gk2; G.ncell = s->ncell; G.M = s->M; G.no_k = h->dp.no_k;
  G.vol = s->vol; G.pi = s->pi; G.ro_g = s->g.ro_g; G.mu_g = s->g.mu_g; G.ur_f_gs = s->g.ur_f_gs;
  G.drag_model = s->g.drag_model; G.usr_d_p0 = s->g.usr_d_p0;
  for (int m = 0; m < MAXP; ++m) G.ro_s[m] = s->g.ro_s[m];
  G.xe = s->xe; G.yn = s->yn; G.zt = s->zt;
  return G;
}

static int run_pic(dem_handle* h) {
  Gas* s = h->gas;
  const GasDev G = gas_view(h);
  const int T = 256, B = (h->n + T - 1) / T;
  cudaMemsetAsync(s->pic_cnt, 0, sizeof(int) * (s->ncell + 1), h->stream);
  const int c = h->cur;
  k_pic_locate<<<B, T, 0, h->stream>>>(h->dp, G, h->pos4[c], h->vel4[c], h->omg4[c], h->state, s->pijk,
                                       s->pic_cnt, h->fc, h->tow, h->wall_fid, h->derr);
  DEM_LAUNCH(h);
  if (int rc = exclusive_scan(h, s->pic_cnt, s->pic_start, s->ncell, s->pic_start + s->ncell)) return rc;
  cudaMemsetAsync(s->pic_cnt, 0, sizeof(int) * (s->ncell + 1), h->stream);
  k_pic_scatter<<<B, T, 0, h->stream>>>(h->n, h->state, s->pijk, s->pic_start, s->pic_cnt, s->pic_list);
  k_pic_sort<<<(s->ncell + T - 1) / T, T, 0, h->stream>>>(s->ncell, s->pic_start, s->pic_list);
  h->launches += 2;
  return check_cuda(h, cudaGetLastError(), "particles_in_cell");
}

static int run_mean_fields(dem_handle* h) {
  ProfScope ps(h, DEM_PROF_COUPLING);
  if (int rc = run_pic(h)) return rc;
  Gas* s = h->gas;
  const GasDev G = gas_view(h);
  const int T = 256;
  if (s->g.interp_scheme == DEM_INTERP_NONE) {   // COMP_MEAN_FIELDS1
    k_mean_fields1<<<(G.ncell + T - 1) / T, T, 0, h->stream>>>(G, h->pos4[h->cur], h->phase, h->state,
                                                               s->pic_start, s->pic_list, s->rop_s, s->ep_g);
    DEM_LAUNCH(h);
    s->have_mean = true;
    return check_cuda(h, cudaGetLastError(), "mean fields");
  }
  const int nnodes = (G.imax + 1) * (G.jmax + 1) * (G.no_k ? 1 : G.kmax + 1);
  const int c = h->cur;
  k_node_deposit<<<(nnodes + T - 1) / T, T, 0, h->stream>>>(G, h->pos4[c], h->vel4[c], h->phase, s->pic_start,
                                                            s->pic_list, s->rops_node);
  k_cell_fields<<<(G.ncell + T - 1) / T, T, 0, h->stream>>>(G, s->vol_surr, s->rops_node, s->rop_s, s->ep_g);
  h->launches += 2;
  s->have_mean = true;
  return check_cuda(h, cudaGetLastError(), "mean fields");
}

static int run_drag(dem_handle* h) {
  ProfScope ps(h, DEM_PROF_COUPLING);
  Gas* s = h->gas;
  const GasDev G = gas_view(h);
  const int T = 256, B = (h->n + T - 1) / T;
  const int c = h->cur;
  k_drag<true><<<B, T, 0, h->stream>>>(h->dp, G, h->pos4[c], h->vel4[c], h->state, s->pijk, s->ep_g, s->u_g,
                                       s->v_g, s->w_g, s->p_force, s->f_gp, h->fc);
  DEM_LAUNCH(h);
  return check_cuda(h, cudaGetLastError(), "drag");
}

static int run_drag1(dem_handle* h) {
  ProfScope ps(h, DEM_PROF_COUPLING);
  Gas* s = h->gas;
  const GasDev G = gas_view(h);
  const int T = 256, B = (h->n + T - 1) / T;
  const int c = h->cur;
  k_drag1<true><<<B, T, 0, h->stream>>>(h->dp, G, h->pos4[c], h->vel4[c], h->state, s->pijk, s->ep_g, s->u_g,
                                        s->v_g, s->w_g, s->p_force, s->f_gp, h->fc);
  DEM_LAUNCH(h);
  return check_cuda(h, cudaGetLastError(), "drag");
}

// CALC_DRAG_DES: the particle side of the drag by DES_INTERP_SCHEME.
static int run_calc_drag(dem_handle* h) {
  return h->gas->g.interp_scheme == DEM_INTERP_NONE ? run_drag1(h) : run_drag(h);
}

// DRAG_GS_GAS1: F_GP per particle, then the per-cell gather.
static int run_drag_gas1(dem_handle* h) {
  ProfScope ps(h, DEM_PROF_COUPLING);
  Gas* s = h->gas;
  const GasDev G = gas_view(h);
  const int T = 256, B = (h->n + T - 1) / T;
  const int c = h->cur;
  k_drag1<false><<<B, T, 0, h->stream>>>(h->dp, G, h->pos4[c], h->vel4[c], h->state, s->pijk, s->ep_g, s->u_g,
                                         s->v_g, s->w_g, nullptr, s->f_gp, nullptr);
  k_gas1_cell<<<(G.ncell + T - 1) / T, T, 0, h->stream>>>(G, h->vel4[c], h->state, s->pic_start, s->pic_list,
                                                          s->f_gp, s->f_gds, s->drag_bm);
  h->launches += 2;
  return check_cuda(h, cudaGetLastError(), "drag gas");
}

// DRAG_GS_GAS0: F_GP per particle, the node gather, F_GDS per cell.
static int run_drag_gas(dem_handle* h) {
  ProfScope ps(h, DEM_PROF_COUPLING);
  Gas* s = h->gas;
  const GasDev G = gas_view(h);
  const int T = 256, B = (h->n + T - 1) / T;
  const int c = h->cur;
  k_drag<false><<<B, T, 0, h->stream>>>(h->dp, G, h->pos4[c], h->vel4[c], h->state, s->pijk, s->ep_g, s->u_g,
                                        s->v_g, s->w_g, nullptr, s->f_gp, nullptr);
  cudaMemsetAsync(s->drag_am, 0, sizeof(double) * s->ncell, h->stream);
  cudaMemsetAsync(s->drag_bm, 0, sizeof(double) * 3 * s->ncell, h->stream);
  const int nnodes = (G.imax + 1) * (G.jmax + 1) * (G.no_k ? 1 : G.kmax + 1);
  k_drag_node<<<(nnodes + T - 1) / T, T, 0, h->stream>>>(G, h->pos4[c], h->vel4[c], s->pic_start, s->pic_list,
                                                         s->f_gp, s->vol_node, s->drag_am, s->drag_bm);
  k_fgds<<<(G.ncell + T - 1) / T, T, 0, h->stream>>>(G, s->drag_am, s->f_gds);
  h->launches += 3;
  return check_cuda(h, cudaGetLastError(), "drag gas");
}

void free_gas(dem_handle* h) {
  Gas* s = h->gas;
  if (!s) return;
  void* ptrs[] = {s->xe, s->yn, s->zt, s->ep_g, s->u_g, s->v_g, s->w_g, s->p_force, s->vol_surr, s->rop_s,
                  s->rops_node, s->vol_node, s->drag_am, s->drag_bm, s->f_gds, s->pijk, s->f_gp,
                  s->pic_cnt, s->pic_start, s->pic_list};
  for (void* q : ptrs) if (q) cudaFree(q);
  delete s;
  h->gas = nullptr;
}

}  // namespace demb

#define API_GUARD(h) do { if (!(h)) return DEM_ERR_ARG; cudaSetDevice((h)->dev); } while (0)

extern "C" {

int dem_set_gas_fields(dem_handle* h, const dem_fluid_grid* g, const double* ep_g, const double* u_g,
                       const double* v_g, const double* w_g, const double* p_force) {
  API_GUARD(h);
  if (h->batch()) return set_err(h, DEM_ERR_ARG, "coupling is not available on a batch handle");
  if (!g || !ep_g || !u_g || !v_g || !w_g) return set_err(h, DEM_ERR_ARG, "null gas field");
  if (!h->have_state) return set_err(h, DEM_ERR_STATE, "upload particles first");
  if (g->imax < 1 || g->jmax < 1 || (!h->dp.no_k && g->kmax < 1) || !(g->dx > 0) || !(g->dy > 0) ||
      (!h->dp.no_k && !(g->dz > 0)))
    return set_err(h, DEM_ERR_ARG, "bad fluid grid");
  for (int m = 0; m < h->dp.nph; ++m)
    if (!(g->ro_s[m] > 0.0)) return set_err(h, DEM_ERR_ARG, "ro_s must be positive");
  if (g->interp_scheme != DEM_INTERP_GARG && g->interp_scheme != DEM_INTERP_NONE)
    return set_err(h, DEM_ERR_ARG, "unknown interp_scheme");
  if (g->drag_model != DEM_DRAG_GIDASPOW && g->drag_model != DEM_DRAG_SINGLE_SPHERE)
    return set_err(h, DEM_ERR_ARG, "unknown drag_model");
  if (g->drag_model == DEM_DRAG_SINGLE_SPHERE && !(g->usr_d_p0 > 0.0))
    return set_err(h, DEM_ERR_ARG, "usr_d_p0 must be positive for the single-sphere drag");
  free_gas(h);
  Gas* s = new Gas();
  h->gas = s;
  s->g = *g;
  s->gi2 = g->imax + 2; s->gj2 = g->jmax + 2; s->gk2 = h->dp.no_k ? 1 : g->kmax + 2;
  s->ncell = s->gi2 * s->gj2 * s->gk2;
  s->M = h->dp.nph;
  s->pi = 4.0 * std::atan(1.0);
  s->vol = g->dx * g->dy * (h->dp.no_k ? (h->prm.domain_hi[2] - h->prm.domain_lo[2]) : g->dz);
  const size_t nc = s->ncell;
  // face positions, accumulated as the fluid grid set-up does
  auto faces = [](double lo, double d, int n) {
    std::vector<double> f(n + 3);
    f[1] = lo; f[0] = lo - d;
    for (int i = 2; i <= n + 2; ++i) f[i] = f[i - 1] + d;
    return f;
  };
  std::vector<double> fx = faces(h->prm.domain_lo[0], g->dx, g->imax);
  std::vector<double> fy = faces(h->prm.domain_lo[1], g->dy, g->jmax);
  std::vector<double> fz = faces(h->prm.domain_lo[2], g->dz, h->dp.no_k ? 0 : g->kmax);
  // VOL_SURR (make_arrays_des.f:78-105)
  auto fluid = [&](int i, int j, int k) {
    return i >= 2 && i <= g->imax + 1 && j >= 2 && j <= g->jmax + 1 &&
           (h->dp.no_k ? k == 1 : (k >= 2 && k <= g->kmax + 1));
  };
  auto cidx = [&](int i, int j, int k) { return (i - 1) + (j - 1) * s->gi2 + (k - 1) * s->gi2 * s->gj2; };
  std::vector<double> vs(nc, 0.0);
  const int nk1 = h->dp.no_k ? 1 : g->kmax + 1;
  for (int k = 1; k <= nk1; ++k)
    for (int j = 1; j <= g->jmax + 1; ++j)
      for (int i = 1; i <= g->imax + 1; ++i) {
        double v = 0.0;
        for (int kk = k; kk <= (h->dp.no_k ? k : k + 1); ++kk)
          for (int jj = j; jj <= j + 1; ++jj)
            for (int ii = i; ii <= i + 1; ++ii)
              if (fluid(ii, jj, kk)) v = v + s->vol;
        vs[cidx(i, j, k)] = v;
      }
  // DES_VOL_NODE (cfassign.f:104-228): a quarter (2D) or an eighth (3D) of
  // each fluid cell sharing the node, summed in the reference's order
  std::vector<double> vn(nc, 0.0);
  const double avn = h->dp.no_k ? 0.25 : 0.125;
  auto fv = [&](int i, int j, int k) { return fluid(i, j, k) ? s->vol : 0.0; };
  for (int k = 1; k <= nk1; ++k)
    for (int j = 1; j <= g->jmax + 1; ++j)
      for (int i = 1; i <= g->imax + 1; ++i) {
        double v = avn * (fv(i, j, k) + fv(i + 1, j, k) + fv(i, j + 1, k) + fv(i + 1, j + 1, k));
        if (!h->dp.no_k)
          v = v + avn * (fv(i, j, k + 1) + fv(i + 1, j + 1, k + 1) + fv(i, j + 1, k + 1) + fv(i + 1, j, k + 1));
        vn[cidx(i, j, k)] = v;
      }
  bool ok = true;
  auto A = [&](void** p, size_t b) { if (ok && cudaMalloc(p, b ? b : 8) != cudaSuccess) ok = false; };
  A((void**)&s->xe, sizeof(double) * fx.size());
  A((void**)&s->yn, sizeof(double) * fy.size());
  A((void**)&s->zt, sizeof(double) * fz.size());
  A((void**)&s->ep_g, sizeof(double) * nc);
  A((void**)&s->u_g, sizeof(double) * nc);
  A((void**)&s->v_g, sizeof(double) * nc);
  A((void**)&s->w_g, sizeof(double) * nc);
  if (p_force) A((void**)&s->p_force, sizeof(double) * 3 * nc);
  A((void**)&s->vol_surr, sizeof(double) * nc);
  A((void**)&s->rop_s, sizeof(double) * nc * s->M);
  A((void**)&s->rops_node, sizeof(double) * nc * s->M);
  A((void**)&s->vol_node, sizeof(double) * nc);
  A((void**)&s->drag_am, sizeof(double) * nc);
  A((void**)&s->drag_bm, sizeof(double) * 3 * nc);
  A((void**)&s->f_gds, sizeof(double) * nc);
  A((void**)&s->pijk, sizeof(int) * 4 * (size_t)h->n);
  A((void**)&s->f_gp, sizeof(double) * (size_t)h->n);
  A((void**)&s->pic_cnt, sizeof(int) * (nc + 1));
  A((void**)&s->pic_start, sizeof(int) * (nc + 1));
  A((void**)&s->pic_list, sizeof(int) * (size_t)h->n);
  if (!ok) { free_gas(h); return set_err(h, DEM_ERR_CUDA, "cudaMalloc gas fields"); }
  cudaMemcpyAsync(s->xe, fx.data(), sizeof(double) * fx.size(), cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(s->yn, fy.data(), sizeof(double) * fy.size(), cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(s->zt, fz.data(), sizeof(double) * fz.size(), cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(s->ep_g, ep_g, sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(s->u_g, u_g, sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(s->v_g, v_g, sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(s->w_g, w_g, sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream);
  if (p_force) cudaMemcpyAsync(s->p_force, p_force, sizeof(double) * 3 * nc, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(s->vol_surr, vs.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(s->vol_node, vn.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream);
  cudaMemsetAsync(s->drag_am, 0, sizeof(double) * nc, h->stream);
  cudaMemsetAsync(s->drag_bm, 0, sizeof(double) * 3 * nc, h->stream);
  cudaMemsetAsync(s->f_gds, 0, sizeof(double) * nc, h->stream);
  cudaMemsetAsync(s->rop_s, 0, sizeof(double) * nc * s->M, h->stream);
  cudaMemsetAsync(s->f_gp, 0, sizeof(double) * (size_t)h->n, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "set gas fields")) { free_gas(h); return rc; }
  if (int rc = run_pic(h)) return rc;
  return fetch_errors(h);
}

int dem_get_mean_fields(dem_handle* h, double* ep_g, double* rop_s) {
  API_GUARD(h);
  if (!h->gas) return set_err(h, DEM_ERR_STATE, "no gas fields");
  Gas* s = h->gas;
  if (ep_g) cudaMemcpyAsync(ep_g, s->ep_g, sizeof(double) * s->ncell, cudaMemcpyDeviceToHost, h->stream);
  if (rop_s) cudaMemcpyAsync(rop_s, s->rop_s, sizeof(double) * s->ncell, cudaMemcpyDeviceToHost, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "get mean fields");
}

int dem_comp_mean_fields(dem_handle* h) {
  API_GUARD(h);
  if (!h->gas) return set_err(h, DEM_ERR_STATE, "no gas fields");
  if (int rc = run_mean_fields(h)) return rc;
  return fetch_errors(h);
}

int dem_calc_des_bedheight(dem_handle* h, double* bed_height) {
  API_GUARD(h);
  if (!h->gas) return set_err(h, DEM_ERR_STATE, "no gas fields");
  if (!bed_height) return set_err(h, DEM_ERR_ARG, "null output");
  Gas* s = h->gas;
  const GasDev G = gas_view(h);
  const int M = s->M, nb = (s->ncell + BED_T - 1) / BED_T;
  double* part = (double*)stage_buffer(h, sizeof(double) * 2 * M * (size_t)nb + 64);
  if (!part) return set_err(h, DEM_ERR_CUDA, "cudaMalloc stage");
  k_bed_partials<<<nb, BED_T, 0, h->stream>>>(G, s->rop_s, part);
  DEM_LAUNCH(h);
  std::vector<double> hp((size_t)2 * M * nb);
  cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(h->herr, h->derr, sizeof(DevErr), cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "bed height")) return rc;
  // the block partials in block order
  std::vector<double> num(M, 0.0), den(M, 0.0);
  for (int b = 0; b < nb; ++b)
    for (int m = 0; m < M; ++m) {
      num[m] += hp[((size_t)b * M + m) * 2];
      den[m] += hp[((size_t)b * M + m) * 2 + 1];
    }
  // PIP > 0: some particle exists
  int pip = 0;
  {
    std::vector<int8_t> st(h->n);
    cudaMemcpyAsync(st.data(), h->state, h->n, cudaMemcpyDeviceToHost, h->stream);
    if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "bed height")) return rc;
    for (int8_t v : st) pip += v != DEM_STATE_NONEXISTENT;
  }
  for (int m = 0; m < M; ++m) bed_height[m] = pip > 0 ? num[m] / den[m] : 0.0;
  return 0;
}

int dem_drag_gs_des0(dem_handle* h) {
  API_GUARD(h);
  if (!h->gas) return set_err(h, DEM_ERR_STATE, "no gas fields");
  if (int rc = run_drag(h)) return rc;
  return check_cuda(h, cudaStreamSynchronize(h->stream), "drag");
}

int dem_drag_gs_gas0(dem_handle* h, double* f_gds, double* drag_am, double* drag_bm, double* f_gp) {
  API_GUARD(h);
  if (!h->gas) return set_err(h, DEM_ERR_STATE, "no gas fields");
  if (int rc = run_drag_gas(h)) return rc;
  Gas* s = h->gas;
  const size_t nc = (size_t)s->ncell;
  if (f_gds) cudaMemcpyAsync(f_gds, s->f_gds, sizeof(double) * nc, cudaMemcpyDeviceToHost, h->stream);
  if (drag_am) cudaMemcpyAsync(drag_am, s->drag_am, sizeof(double) * nc, cudaMemcpyDeviceToHost, h->stream);
  if (drag_bm) cudaMemcpyAsync(drag_bm, s->drag_bm, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, h->stream);
  if (f_gp) cudaMemcpyAsync(f_gp, s->f_gp, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToHost, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "drag gas");
}

int dem_drag_gs_des1(dem_handle* h) {
  API_GUARD(h);
  if (!h->gas) return set_err(h, DEM_ERR_STATE, "no gas fields");
  if (int rc = run_drag1(h)) return rc;
  return check_cuda(h, cudaStreamSynchronize(h->stream), "drag");
}

int dem_drag_gs_gas1(dem_handle* h, double* f_gds, double* drag_bm, double* f_gp) {
  API_GUARD(h);
  if (!h->gas) return set_err(h, DEM_ERR_STATE, "no gas fields");
  if (int rc = run_drag_gas1(h)) return rc;
  Gas* s = h->gas;
  const size_t nc = (size_t)s->ncell;
  if (f_gds) cudaMemcpyAsync(f_gds, s->f_gds, sizeof(double) * nc, cudaMemcpyDeviceToHost, h->stream);
  if (drag_bm) cudaMemcpyAsync(drag_bm, s->drag_bm, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, h->stream);
  if (f_gp) cudaMemcpyAsync(f_gp, s->f_gp, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToHost, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "drag gas");
}

int dem_step_coupled(dem_handle* h, int32_t nn_first, int32_t nsteps) {
  API_GUARD(h);
  if (!h->gas) return set_err(h, DEM_ERR_STATE, "no gas fields");
  if (!h->have_state || !h->have_pairs) return set_err(h, DEM_ERR_STATE, "state or pair list missing");
  if (nsteps < 0 || nn_first < 1) return set_err(h, DEM_ERR_ARG, "bad step range");
  const DevParams& p = h->dp;
  const bool anyper = p.per[0] || p.per[1] || (p.per[2] && !p.no_k);
  for (int k = 0; k < nsteps; ++k) {
    const int nn = nn_first + k;
    cudaMemsetAsync(&h->derr->n_contacts, 0, 2 * sizeof(unsigned long long), h->stream);
    if (int rc = run_force(h, false)) return rc;              // CALC_FORCE_DEM
    if (int rc = run_calc_drag(h)) return rc;                 // CALC_DRAG_DES
    bool force = false;
    if (h->obc.empty()) {
      if (int rc = run_cfnewvalues(h)) return rc;             // CFUPDATEOLD + CFNEWVALUES
      if (int rc = run_mass_inflow(h)) return rc;             // MASS_INFLOW_DEM
    } else if (int rc = run_cfnewvalues_outflow(h, &force)) { // + exit velocities, MASS_OUTFLOW_DEM
      return rc;
    }
    const bool do_nsearch = (nn == 1) || (nn % h->prm.neighbor_search_n == 0) || force;
    if (do_nsearch || anyper) {
      if (int rc = run_desgrid_pic(h, do_nsearch)) return rc;
    }
    if (do_nsearch) {
      if (int rc = run_neighbour(h, true)) return rc;
    }
    if (int rc = run_mean_fields(h)) return rc;               // PARTICLES_IN_CELL + COMP_MEAN_FIELDS
    h->s_time = h->s_time + h->prm.dtsolid;
    h->steps_done++;
  }
  return fetch_errors(h);
}

}  // extern "C"
