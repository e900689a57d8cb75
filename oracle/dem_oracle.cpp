// dem_oracle.cpp -- CPU restatement of the MFiX DEM particle step.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never part of
// the product path.  Each routine restates the cited Fortran of the reference
// (paths relative to the MFiX source root) in the same floating-point
// operation order as the serial (non-OpenMP) build, so that a compiler
// without FMA contraction reproduces the reference's double-precision
// results.  Build with -ffp-contract=off.
//
// Data layout: per-particle vectors are Fortran (MAX_PIP,3) column-major
// (x block, y block, z block); indices are 0-based inside, 1-based at the
// orc_* boundary.  Periodic axes use the minimum-image convention in place of
// the reference's ghost copies (see periodic_shift()).

#include "dem_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <deque>
#include <vector>
#include <cfloat>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double SMALL_NUMBER = 1.0e-15;     // param1_mod.f:26
constexpr double UNDEFINED    = 9.87654321e31; // param1_mod.f:20
constexpr double TOL_STL      = 1.0e-6;      // cartesian_grid_init_namelist.f:748
constexpr double TOL_EDGE     = 1.0e-9;      // stl_preproc_des_mod.f:383
constexpr float  STL_NB_ANGLE = 5.0f;        // cartesian_grid_init_namelist.f:765 (REAL literal)

inline double dot3(const double a[3], const double b[3]) {
  // gfortran DOT_PRODUCT: accumulate left to right from zero.
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
inline void cross3(const double x[3], const double y[3], double out[3]) {
  // CROSS, discretelement_mod.f:918-920
  out[0] = x[1] * y[2] - x[2] * y[1];
  out[1] = x[2] * y[0] - x[0] * y[2];
  out[2] = x[0] * y[1] - x[1] * y[0];
}

struct FacetEntry {
  int id;       // 0-based facet
  int dir;      // 0-based axis of smallest extent
  double mn, mx;
};

struct Oracle {
  dem_params p{};
  int n = 0;
  int nthreads = 1;
  std::string err;

  // particle state (Fortran column blocks)
  std::vector<double> pos, vel, omg, rad, pmass, omoi;
  std::vector<int8_t> state;
  std::vector<int> phase;  // 0-based
  std::vector<double> fc, tow, acc_old, rot_acc_old;
  bool first_pass = true;
  bool have_state = false;

  // DES grid (desgrid_mod.f:506-865, single rank)
  int istart1, iend1, istart2, iend2, jstart1, jend1, jstart2, jend2;
  int kstart1, kend1, kstart2, kend2;
  int c1, c2, c3, ncell2;
  std::vector<int> dg_pijk;              // 1-based cell, 0 = none
  std::vector<int> cell_start, cell_list;  // dg_pic as CSR over 0-based cell

  // pairs: row_end[i] = pairs in rows 0..i; nbrs 0-based; pft (3,P)
  std::vector<int> row_end, nbrs;
  std::vector<double> pft;

  // walls
  int nf = 0;
  std::vector<double> vertex, norm_face;   // (3,3,F), (3,F)
  std::vector<int8_t> ignore_edge;         // (F,4) edges 0..3
  std::vector<int> fbin_start;             // CSR over 0-based cells
  std::vector<FacetEntry> fbin;
  int cmax = 8;
  std::vector<int> wall_fid;               // (cmax, n) 0-based facet, -1 free
  std::vector<double> wall_pft;            // (3, cmax, n)

  // bookkeeping
  double s_time = 0.0;
  int64_t steps_done = 0, rogue_removed = 0, n_contacts = 0, n_wall_contacts = 0;
  double max_overlap_ratio = 0.0;

  // coupling (uniform Cartesian fluid grid; MFiX IJK with one ghost layer,
  // i fastest)
  bool have_gas = false;
  dem_fluid_grid g{};
  int gi2 = 0, gj2 = 0, gk2 = 0;          // imax+2, jmax+2, kmax+2
  std::vector<double> xe, yn, zt;         // face positions, index 0..imax+2
  std::vector<double> ep_g, u_g, v_g, w_g, p_force, rop_s, vol_surr;
  std::vector<double> vol_node;            // DES_VOL_NODE per node
  std::vector<dem_outflow_bc> obc;         // DEM outflow boundaries (DEM_BCMO_MAP order)
  std::vector<double> vel_old;             // DES_VEL_OLD when outflow boundaries are set
  bool exit_first_pass = true;             // UPDATE_EXIT_DES_VEL's own FIRST_PASS
  int64_t n_outflow_deleted = 0;
  struct Inflow { dem_inflow_bc bc; std::vector<double> p, q; std::vector<int32_t> layout; };
  std::vector<Inflow> ibc;                 // DEM mass-inflow boundaries (DEM_BCMI_MAP order)
  std::deque<double> irand;                // queued RANDOM_NUMBER values
  uint64_t irng = 0;                       // splitmix64 state when the queue is empty
  int64_t n_inflow_added = 0;
  std::vector<double> drag_am, drag_bm, f_gds;  // DRAG_AM, DRAG_BM(:,3), F_GDS
  std::vector<int> pijk;                  // (n,4): i, j, k, ijk (1-based), 0 = none
  std::vector<double> f_gp;               // F_GP(n)
  std::vector<int> pic_start, pic_list;   // particles per fluid cell, ascending
  double pi_c = 4.0 * std::atan(1.0);
  double ro_s[DEM_MAX_PHASES] = {0};

  int fail(int code, const std::string& m) { err = m; return code; }

  // ---------------------------------------------------------------------
  // DES grid index functions (desgrid_mod.f:184-188, 338-368, 391-419)
  int funijk(int i, int j, int k) const { return j + i * c1 + k * c2 + c3; }
  int jof(int ijk) const { return ((ijk - 1) % c2) % c1 + jstart2; }
  int iof(int ijk) const { return ((ijk - jof(ijk) + jstart2 - 1) % c2) / c1 + istart2; }
  int kof(int ijk) const { return (ijk - c3 - iof(ijk) * c1 - jof(ijk)) / c2; }
  int iofpos(double x) const { return (int)std::floor((x - p.dg_xstart) * p.dg_dxinv) + istart1; }
  int jofpos(double y) const { return (int)std::floor((y - p.dg_ystart) * p.dg_dyinv) + jstart1; }
  int kofpos(double z) const { return (int)std::floor((z - p.dg_zstart) * p.dg_dzinv) + kstart1; }

  void grid_init() {
    // desgrid_init (desgrid_mod.f:571-604, 780-850) for one rank.
    istart1 = 2; iend1 = p.dg_imax + 1; istart2 = 1; iend2 = p.dg_imax + 2;
    jstart1 = 2; jend1 = p.dg_jmax + 1; jstart2 = 1; jend2 = p.dg_jmax + 2;
    if (p.no_k) { kstart1 = kend1 = kstart2 = kend2 = 1; }
    else { kstart1 = 2; kend1 = p.dg_kmax + 1; kstart2 = 1; kend2 = p.dg_kmax + 2; }
    c1 = jend2 - jstart2 + 1;
    c2 = c1 * (iend2 - istart2 + 1);
    c3 = -c1 * istart2 - c2 * kstart2 - jstart2 + 1;
    ncell2 = (iend2 - istart2 + 1) * (jend2 - jstart2 + 1) * (kend2 - kstart2 + 1);
  }

  double* X(std::vector<double>& v, int c) { return v.data() + (size_t)c * n; }
  double  P(const std::vector<double>& v, int i, int c) const { return v[(size_t)c * n + i]; }

  // Minimum-image shift for periodic axes: the displacement pos(j)-pos(i) is
  // the one to the nearest periodic copy of j, which is the copy the
  // reference's ghost exchange would have placed in i's stencil.
  double periodic_shift(int c, double d) const {
    if (!p.periodic[c]) return 0.0;
    double L = p.domain_hi[c] - p.domain_lo[c];
    if (d > 0.5 * L) return -L;
    if (d < -0.5 * L) return L;
    return 0.0;
  }
  void pair_dist(int i, int j, double d[3]) const {
    // DIST = DES_POS_NEW(I,:) - DES_POS_NEW(LL,:) (calc_force_dem.f:214)
    for (int c = 0; c < 3; ++c) {
      double pj = P(pos, j, c);
      double pi = P(pos, i, c);
      double s = periodic_shift(c, pj - pi);
      if (s != 0.0) pj = pj + s;
      d[c] = pj - pi;
    }
  }

  // ---------------------------------------------------------------------
  // Periodic self-exchange of crossing particles (the serial path of
  // DES_PAR_EXCHANGE, mpi_funs_des_mod.f:38-160): a particle whose cell
  // index lies past the last interior cell is moved by one period.
  void periodic_wrap() {
    int lo[3] = {istart1, jstart1, kstart1}, hi[3] = {iend1, jend1, kend1};
    for (int i = 0; i < n; ++i) {
      if (state[i] == DEM_STATE_NONEXISTENT) continue;
      for (int c = 0; c < 3; ++c) {
        if (!p.periodic[c]) continue;
        if (c == 2 && p.no_k) continue;
        double x = P(pos, i, c);
        int ci = c == 0 ? iofpos(x) : (c == 1 ? jofpos(x) : kofpos(x));
        double L = p.domain_hi[c] - p.domain_lo[c];
        if (ci > hi[c]) X(pos, c)[i] = x - L;
        else if (ci < lo[c]) X(pos, c)[i] = x + L;
      }
    }
  }

  // DESGRID_PIC(.TRUE.) (desgrid_mod.f:877-995), serial order.
  void desgrid_pic() {
    bool anyper = p.periodic[0] || p.periodic[1] || (p.periodic[2] && !p.no_k);
    if (anyper) periodic_wrap();
    std::vector<int> cnt(ncell2, 0);
    for (int i = 0; i < n; ++i) {
      if (state[i] == DEM_STATE_NONEXISTENT) { dg_pijk[i] = 0; continue; }
      int li = std::min(iend2, std::max(istart2, iofpos(P(pos, i, 0))));
      int lj = std::min(jend2, std::max(jstart2, jofpos(P(pos, i, 1))));
      int lk = p.no_k ? 1 : std::min(kend2, std::max(kstart2, kofpos(P(pos, i, 2))));
      dg_pijk[i] = funijk(li, lj, lk);
      cnt[dg_pijk[i] - 1]++;
    }
    cell_start.assign(ncell2 + 1, 0);
    for (int c = 0; c < ncell2; ++c) cell_start[c + 1] = cell_start[c] + cnt[c];
    cell_list.assign(cell_start[ncell2], 0);
    std::vector<int> fillp(cell_start.begin(), cell_start.end() - 1);
    for (int i = 0; i < n; ++i) {
      if (state[i] == DEM_STATE_NONEXISTENT) continue;
      cell_list[fillp[dg_pijk[i] - 1]++] = i;
    }
  }

  // DELETE_PARTICLE (mass_outflow_dem.f:201-303)
  void delete_particle(int i) {
    for (int c = 0; c < 3; ++c) {
      X(pos, c)[i] = 0.0; X(vel, c)[i] = 0.0; X(omg, c)[i] = 0.0;
      X(fc, c)[i] = 0.0; X(tow, c)[i] = 0.0;
    }
    rad[i] = 0.0;
    pmass[i] = (double)FLT_MAX;  // HUGE(0.0)
    omoi[i] = 0.0;
    for (int s = 0; s < cmax; ++s) wall_fid[(size_t)i * cmax + s] = -1;
    state[i] = DEM_STATE_NONEXISTENT;
  }

  // DESGRID_NEIGH_BUILD (desgrid_mod.f:1002-1299), serial build with add_pair
  // (des_allocate_mod.f:555-567).  Rows follow the (lk, lj, li) stencil order
  // and ascending particle index inside each cell.  The serial loop deletes a
  // rogue particle when it reaches it and, because its do_exit flag stays
  // set, gives every later particle an empty row; particles before the first
  // rogue one still see it as NORMAL.  Rows are therefore computed with the
  // pre-deletion states for cur < first_rogue, and the rogue particles are
  // deleted afterwards, which is the same result.
  int row_scan(int cur, int* out) const {
    const double fr = p.factor_rlm, mr = p.max_radius;
    bool coarse_x = 1.0 > 2.0 * mr * fr * p.dg_dxinv;
    bool coarse_y = 1.0 > 2.0 * mr * fr * p.dg_dyinv;
    bool coarse_z = 1.0 > 2.0 * mr * fr * p.dg_dzinv;
    int cnt = 0;
    int lijk = dg_pijk[cur];
    int lic = iof(lijk), ljc = jof(lijk), lkc = kof(lijk);
    int il = 1, iu = 1, jl = 1, ju = 1, kl = 1, ku = 1;
    double cp[3] = {P(pos, cur, 0), P(pos, cur, 1), P(pos, cur, 2)};
    if (coarse_x) {
      double t = (cp[0] - p.dg_xstart) * p.dg_dxinv;
      double off = t - (double)(long long)std::floor(t);
      if (off >= 0.5) il = 0; else iu = 0;
    }
    if (coarse_y) {
      double t = (cp[1] - p.dg_ystart) * p.dg_dyinv;
      double off = t - (double)(long long)std::floor(t);
      if (off >= 0.5) jl = 0; else ju = 0;
    }
    if (p.no_k) { kl = 0; ku = 0; }
    else if (coarse_z) {
      double t = (cp[2] - p.dg_zstart) * p.dg_dzinv;
      double off = t - (double)(long long)std::floor(t);
      if (off >= 0.5) kl = 0; else ku = 0;
    }
    for (int lk = lkc - kl; lk <= lkc + ku; ++lk)
    for (int lj = ljc - jl; lj <= ljc + ju; ++lj)
    for (int li = lic - il; li <= lic + iu; ++li) {
      // periodic axes: the ghost layer holds copies of the opposite
      // interior layer shifted by one period.
      int ri = li, rj = lj, rk = lk;
      double sh[3] = {0.0, 0.0, 0.0};
      if (p.periodic[0]) {
        if (li < istart1) { ri = iend1; sh[0] = -(p.domain_hi[0] - p.domain_lo[0]); }
        else if (li > iend1) { ri = istart1; sh[0] = (p.domain_hi[0] - p.domain_lo[0]); }
      }
      if (p.periodic[1]) {
        if (lj < jstart1) { rj = jend1; sh[1] = -(p.domain_hi[1] - p.domain_lo[1]); }
        else if (lj > jend1) { rj = jstart1; sh[1] = (p.domain_hi[1] - p.domain_lo[1]); }
      }
      if (p.periodic[2] && !p.no_k) {
        if (lk < kstart1) { rk = kend1; sh[2] = -(p.domain_hi[2] - p.domain_lo[2]); }
        else if (lk > kend1) { rk = kstart1; sh[2] = (p.domain_hi[2] - p.domain_lo[2]); }
      }
      bool ghost = (sh[0] != 0.0 || sh[1] != 0.0 || sh[2] != 0.0);
      int cell = funijk(ri, rj, rk) - 1;
      for (int s = cell_start[cell]; s < cell_start[cell + 1]; ++s) {
        int nb = cell_list[s];
        if (nb == cur) continue;
        if (nb < cur && state[nb] == DEM_STATE_NORMAL) continue;
        if (state[nb] == DEM_STATE_NONEXISTENT) continue;
        double srad = fr * (rad[cur] + rad[nb]);
        double d[3];
        for (int c = 0; c < 3; ++c) {
          double pn = P(pos, nb, c);
          if (ghost && sh[c] != 0.0) pn = pn + sh[c];
          d[c] = cp[c] - pn;
        }
        double d2 = dot3(d, d);
        if (d2 > srad * srad) continue;
        if (out) out[cnt] = nb;
        ++cnt;
      }
    }
    return cnt;
  }

  bool is_rogue(int cur) const {
    if (state[cur] != DEM_STATE_NORMAL) return false;
    int lijk = dg_pijk[cur];
    int lic = iof(lijk), ljc = jof(lijk), lkc = kof(lijk);
    return (lic < istart1 || lic > iend1 || ljc < jstart1 || ljc > jend1 ||
            lkc < kstart1 || lkc > kend1);
  }

  void neigh_build() {
    int first_rogue = n;
    for (int cur = 0; cur < n; ++cur) if (is_rogue(cur)) { first_rogue = cur; break; }
    std::vector<int> cnt(n, 0);
#pragma omp parallel for schedule(dynamic, 512) num_threads(nthreads) if (nthreads > 1)
    for (int cur = 0; cur < n; ++cur) {
      if (state[cur] != DEM_STATE_NORMAL || cur >= first_rogue) continue;
      cnt[cur] = row_scan(cur, nullptr);
    }
    row_end.assign(n, 0);
    long long tot = 0;
    for (int cur = 0; cur < n; ++cur) { tot += cnt[cur]; row_end[cur] = (int)tot; }
    nbrs.assign((size_t)tot, 0);
#pragma omp parallel for schedule(dynamic, 512) num_threads(nthreads) if (nthreads > 1)
    for (int cur = 0; cur < n; ++cur) {
      if (!cnt[cur]) continue;
      row_scan(cur, nbrs.data() + (cur ? row_end[cur - 1] : 0));
    }
    for (int cur = first_rogue; cur < n; ++cur) {
      if (!is_rogue(cur)) continue;
      if (p.remove_rogue) { delete_particle(cur); rogue_removed++; }
      else err = "NORMAL particle found in GHOST cell";
    }
  }

  // NEIGHBOUR (neighbour.f:21-126): rebuild and carry PFT over by matching
  // the neighbour id inside the old row of the same particle.
  void neighbour() {
    std::vector<int> old_end = row_end, old_nbrs = nbrs;
    std::vector<double> old_pft = pft;
    neigh_build();
    pft.assign((size_t)3 * nbrs.size(), 0.0);
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads) if (nthreads > 1)
    for (int ll = 0; ll < n; ++ll) {
      int s = ll ? row_end[ll - 1] : 0, e = row_end[ll];
      int so = 0, eo = 0;
      if (!old_end.empty()) { so = ll ? old_end[ll - 1] : 0; eo = old_end[ll]; }
      for (int cc = s; cc < e; ++cc) {
        bool found = false;
        for (int co = so; co < eo; ++co) {
          if (nbrs[cc] == old_nbrs[co]) {
            for (int c = 0; c < 3; ++c) pft[3 * (size_t)cc + c] = old_pft[3 * (size_t)co + c];
            found = true;
            break;
          }
        }
        if (!found) for (int c = 0; c < 3; ++c) pft[3 * (size_t)cc + c] = 0.0;
      }
    }
  }

  // ---------------------------------------------------------------------
  // Walls
  double V(int f, int v, int c) const { return vertex[(size_t)v + 3 * c + 9 * (size_t)f]; }

  // TRI_BOX_OVERLAP (stl_functions_des_mod.f:280-536), Akenine-Moller test.
  static bool tri_box_overlap(const double ctr[3], const double hs[3], const double vt[3][3]) {
    double v0[3], v1[3], v2[3], e0[3], e1[3], e2[3];
    for (int c = 0; c < 3; ++c) {
      v0[c] = vt[0][c] - ctr[c]; v1[c] = vt[1][c] - ctr[c]; v2[c] = vt[2][c] - ctr[c];
    }
    for (int c = 0; c < 3; ++c) { e0[c] = v1[c] - v0[c]; e1[c] = v2[c] - v1[c]; e2[c] = v0[c] - v2[c]; }
    auto axtest = [&](double pa, double pb, double rad) {
      double lmin = pa < pb ? pa : pb, lmax = pa < pb ? pb : pa;
      return (lmin > rad || lmax < -rad);
    };
    auto z12 = [&](double pa1, double pa2, double rad) {  // ATEST_Z12 orders (p2<p1)
      double lmin, lmax;
      if (pa2 < pa1) { lmin = pa2; lmax = pa1; } else { lmin = pa1; lmax = pa2; }
      return (lmin > rad || lmax < -rad);
    };
    double fex, fey, fez;
    // edge e0
    fex = std::fabs(e0[0]); fey = std::fabs(e0[1]); fez = std::fabs(e0[2]);
    { double a = e0[2], b = e0[1];  // X01
      if (axtest(a * v0[1] - b * v0[2], a * v2[1] - b * v2[2], fez * hs[1] + fey * hs[2])) return false; }
    { double a = e0[2], b = e0[0];  // Y02
      if (axtest(-a * v0[0] + b * v0[2], -a * v2[0] + b * v2[2], fez * hs[0] + fex * hs[2])) return false; }
    { double a = e0[1], b = e0[0];  // Z12
      if (z12(a * v1[0] - b * v1[1], a * v2[0] - b * v2[1], fey * hs[0] + fex * hs[1])) return false; }
    // edge e1
    fex = std::fabs(e1[0]); fey = std::fabs(e1[1]); fez = std::fabs(e1[2]);
    { double a = e1[2], b = e1[1];  // X01
      if (axtest(a * v0[1] - b * v0[2], a * v2[1] - b * v2[2], fez * hs[1] + fey * hs[2])) return false; }
    { double a = e1[2], b = e1[0];  // Y02
      if (axtest(-a * v0[0] + b * v0[2], -a * v2[0] + b * v2[2], fez * hs[0] + fex * hs[2])) return false; }
    { double a = e1[1], b = e1[0];  // Z0
      if (axtest(a * v0[0] - b * v0[1], a * v1[0] - b * v1[1], fey * hs[0] + fex * hs[1])) return false; }
    // edge e2
    fex = std::fabs(e2[0]); fey = std::fabs(e2[1]); fez = std::fabs(e2[2]);
    { double a = e2[2], b = e2[1];  // X2
      if (axtest(a * v0[1] - b * v0[2], a * v1[1] - b * v1[2], fez * hs[1] + fey * hs[2])) return false; }
    { double a = e2[2], b = e2[0];  // Y1
      if (axtest(-a * v0[0] + b * v0[2], -a * v1[0] + b * v1[2], fez * hs[0] + fex * hs[2])) return false; }
    { double a = e2[1], b = e2[0];  // Z12
      if (z12(a * v1[0] - b * v1[1], a * v2[0] - b * v2[1], fey * hs[0] + fex * hs[1])) return false; }
    auto fmin3 = [](double a, double b, double c) { double m = a; if (b < m) m = b; if (c < m) m = c; return m; };
    auto fmax3 = [](double a, double b, double c) { double m = a; if (b > m) m = b; if (c > m) m = c; return m; };
    for (int c = 0; c < 3; ++c)
      if (fmin3(v0[c], v1[c], v2[c]) > hs[c] || fmax3(v0[c], v1[c], v2[c]) < -hs[c]) return false;
    double nrm[3];
    nrm[0] = e0[1] * e1[2] - e0[2] * e1[1];
    nrm[1] = e0[2] * e1[0] - e0[0] * e1[2];
    nrm[2] = e0[0] * e1[1] - e0[1] * e1[0];
    double vmin[3], vmax[3];
    for (int c = 0; c < 3; ++c) {
      double v = v0[c];
      if (nrm[c] > 0.0) { vmin[c] = -hs[c] - v; vmax[c] = hs[c] - v; }
      else { vmin[c] = hs[c] - v; vmax[c] = -hs[c] - v; }
    }
    if (dot3(nrm, vmin) > 0.0) return false;
    if (dot3(nrm, vmax) >= 0.0) return true;
    return false;
  }

  // BIN_FACETS_TO_DG + ADD_FACET_FOR_DES + ADD_FACET
  // (stl_preproc_des_mod.f:135-349) and
  // FLAG_FACETS_WHERE_EDGE_COLLISION_IS_IGNORED (361-490).
  void bin_facets() {
    std::vector<std::vector<FacetEntry>> bins(ncell2);
    const double buffer = 1.1 * p.max_radius;
    const double ldx = 1.0 / p.dg_dxinv, ldy = 1.0 / p.dg_dyinv, ldz = 1.0 / p.dg_dzinv;
    for (int f = 0; f < nf; ++f) {
      double x1 = std::min({V(f,0,0), V(f,1,0), V(f,2,0)}), x2 = std::max({V(f,0,0), V(f,1,0), V(f,2,0)});
      double y1 = std::min({V(f,0,1), V(f,1,1), V(f,2,1)}), y2 = std::max({V(f,0,1), V(f,1,1), V(f,2,1)});
      double z1 = std::min({V(f,0,2), V(f,1,2), V(f,2,2)}), z2 = std::max({V(f,0,2), V(f,1,2), V(f,2,2)});
      int i1 = iend2, i2 = istart2, j1 = jend2, j2 = jstart2, k1 = kend2, k2 = kstart2;
      if (x2 >= p.domain_lo[0] - TOL_STL && x1 <= p.domain_hi[0] + TOL_STL) {
        i1 = std::max(iofpos(x1) - 1, istart2); i2 = std::min(iofpos(x2) + 1, iend2);
      }
      if (y2 >= p.domain_lo[1] - TOL_STL && y1 <= p.domain_hi[1] + TOL_STL) {
        j1 = std::max(jofpos(y1) - 1, jstart2); j2 = std::min(jofpos(y2) + 1, jend2);
      }
      if (!p.no_k) {
        if (z2 >= p.domain_lo[2] - TOL_STL && z1 <= p.domain_hi[2] + TOL_STL) {
          k1 = std::max(kofpos(z1) - 1, kstart2); k2 = std::min(kofpos(z2) + 1, kend2);
        }
      }
      double vt[3][3];
      for (int v = 0; v < 3; ++v) for (int c = 0; c < 3; ++c) vt[v][c] = V(f, v, c);
      for (int kk = k1; kk <= k2; ++kk)
      for (int jj = j1; jj <= j2; ++jj)
      for (int ii = i1; ii <= i2; ++ii) {
        double ctr[3], hs[3];
        ctr[0] = p.dg_xstart + ((double)(ii - istart1) + 0.5) * ldx; hs[0] = 0.5 * ldx + buffer;
        ctr[1] = p.dg_ystart + ((double)(jj - jstart1) + 0.5) * ldy; hs[1] = 0.5 * ldy + buffer;
        if (!p.no_k) { ctr[2] = p.dg_zstart + ((double)(kk - kstart1) + 0.5) * ldz; hs[2] = 0.5 * ldz + buffer; }
        else { ctr[2] = 0.5 * ldz; hs[2] = 0.5 * ldz; }
        if (!tri_box_overlap(ctr, hs, vt)) continue;
        auto& b = bins[funijk(ii, jj, kk) - 1];
        bool dup = false;
        for (auto& e : b) if (e.id == f) { dup = true; break; }
        if (dup) continue;
        FacetEntry e{f, 0, 0.0, 0.0};
        double smallest = (double)FLT_MAX;  // HUGE(0.0)
        for (int c = 0; c < 3; ++c) {
          double mn = std::min({V(f,0,c), V(f,1,c), V(f,2,c)});
          double mx = std::max({V(f,0,c), V(f,1,c), V(f,2,c)});
          if (std::fabs(mx - mn) < smallest) { e.dir = c; e.mn = mn; e.mx = mx; smallest = std::fabs(mx - mn); }
        }
        b.push_back(e);
      }
    }
    fbin_start.assign(ncell2 + 1, 0);
    fbin.clear();
    for (int c = 0; c < ncell2; ++c) {
      fbin_start[c] = (int)fbin.size();
      for (auto& e : bins[c]) fbin.push_back(e);
    }
    fbin_start[ncell2] = (int)fbin.size();

    // edge flags
    ignore_edge.assign((size_t)nf * 4, 0);
    const double pi = 4.0 * std::atan(1.0);
    const double cos_nb = std::cos((double)STL_NB_ANGLE / 180.0 * pi) + 1.0e-6;
    auto edge_centers = [&](int f, double ec[3][3]) {
      for (int c = 0; c < 3; ++c) {
        ec[0][c] = 0.5 * (V(f,0,c) + V(f,1,c));
        ec[1][c] = 0.5 * (V(f,0,c) + V(f,2,c));
        ec[2][c] = 0.5 * (V(f,1,c) + V(f,2,c));
      }
    };
    for (int cell = 0; cell < ncell2; ++cell) {
      int s = fbin_start[cell], e = fbin_start[cell + 1];
      for (int a = s; a < e; ++a) {
        int fa = fbin[a].id; double ec[3][3]; edge_centers(fa, ec);
        for (int ed = 0; ed < 3; ++ed)
          for (int b = s; b < e; ++b) {
            if (a == b) continue;
            int fb = fbin[b].id; double nec[3][3]; edge_centers(fb, nec);
            for (int ned = 0; ned < 3; ++ned) {
              double d[3] = {nec[ned][0] - ec[ed][0], nec[ned][1] - ec[ed][1], nec[ned][2] - ec[ed][2]};
              if (dot3(d, d) < TOL_EDGE) {
                const double* na = &norm_face[3 * (size_t)fa];
                const double* nb = &norm_face[3 * (size_t)fb];
                double dp = na[0] * nb[0] + na[1] * nb[1] + na[2] * nb[2];
                if (dp > cos_nb) {
                  ignore_edge[(size_t)fa * 4 + ed + 1] = 1;
                  ignore_edge[(size_t)fb * 4 + ned + 1] = 1;
                }
              }
            }
          }
      }
    }
  }

  // ClosestPtPointTriangle (stl_functions_des_mod.f:25-160)
  void closest_pt(int f, const double pp[3], double cpt[3], bool& poe, int& edge) const {
    poe = false; edge = 0;
    double a[3], b[3], c[3], ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int k = 0; k < 3; ++k) { a[k] = V(f,0,k); b[k] = V(f,1,k); c[k] = V(f,2,k); }
    for (int k = 0; k < 3; ++k) { ab[k] = b[k] - a[k]; ac[k] = c[k] - a[k]; ap[k] = pp[k] - a[k]; }
    double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    auto ign = [&](int e) { return ignore_edge[(size_t)f * 4 + e] != 0; };
    if (d1 < 0.0 && d2 < 0.0) {
      for (int k = 0; k < 3; ++k) cpt[k] = a[k];
      poe = true; if (ign(1)) cpt[0] = UNDEFINED; edge = 1; return;
    }
    for (int k = 0; k < 3; ++k) bp[k] = pp[k] - b[k];
    double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 > 0.0 && d4 < d3) {
      for (int k = 0; k < 3; ++k) cpt[k] = b[k];
      poe = true; if (ign(1)) cpt[0] = UNDEFINED; edge = 1; return;
    }
    double vc = d1 * d4 - d3 * d2;
    if (vc < 0.0 && d1 > 0.0 && d3 < 0.0) {
      double v = d1 / (d1 - d3);
      for (int k = 0; k < 3; ++k) cpt[k] = a[k] + v * ab[k];
      poe = true; if (ign(1)) cpt[0] = UNDEFINED; edge = 1; return;
    }
    for (int k = 0; k < 3; ++k) cp[k] = pp[k] - c[k];
    double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 > 0.0 && d5 < d6) {
      for (int k = 0; k < 3; ++k) cpt[k] = c[k];
      poe = true; if (ign(2)) cpt[0] = UNDEFINED; edge = 2; return;
    }
    double vb = d5 * d2 - d1 * d6;
    if (vb < 0.0 && d2 > 0.0 && d6 < 0.0) {
      double w = d2 / (d2 - d6);
      for (int k = 0; k < 3; ++k) cpt[k] = a[k] + w * ac[k];
      poe = true; if (ign(2)) cpt[0] = UNDEFINED; edge = 2; return;
    }
    double va = d3 * d6 - d5 * d4;
    if (va < 0.0 && (d4 - d3) > 0.0 && (d5 - d6) > 0.0) {
      double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
      for (int k = 0; k < 3; ++k) cpt[k] = b[k] + w * (c[k] - b[k]);
      poe = true; if (ign(3)) cpt[0] = UNDEFINED; edge = 3; return;
    }
    double denom = 1.0 / (va + vb + vc);
    double v = vb * denom, w = vc * denom;
    for (int k = 0; k < 3; ++k) cpt[k] = a[k] + ab[k] * v + ac[k] * w;
    if (p.no_k) cpt[2] = pp[2];
    poe = false; edge = 0;
  }

  // GET_COLLISION / UPDATE_COLLISION / REMOVE_COLLISION
  // (calc_collision_wall_mod.f:651-792)
  int get_collision(int ll, int f, double out[3]) {
    int* fid = &wall_fid[(size_t)ll * cmax];
    double* wp = &wall_pft[(size_t)ll * cmax * 3];
    int free_index = -1;
    for (int s = 0; s < cmax; ++s) {
      if (f == fid[s]) { for (int c = 0; c < 3; ++c) out[c] = wp[3 * s + c]; return 0; }
      else if (fid[s] == -1) free_index = s;
    }
    if (free_index == -1) {
      int cell = dg_pijk[ll] - 1;
      for (int s = 0; s < cmax && free_index == -1; ++s) {
        bool in_cell = false;
        for (int q = fbin_start[cell]; q < fbin_start[cell + 1]; ++q)
          if (fid[s] == fbin[q].id) { in_cell = true; break; }
        if (!in_cell) free_index = s;
      }
    }
    if (free_index == -1) return DEM_ERR_WALL_SLOTS;
    fid[free_index] = f;
    for (int c = 0; c < 3; ++c) { wp[3 * free_index + c] = 0.0; out[c] = 0.0; }
    return 0;
  }
  void update_collision(int ll, int f, const double v[3]) {
    int* fid = &wall_fid[(size_t)ll * cmax];
    double* wp = &wall_pft[(size_t)ll * cmax * 3];
    for (int s = 0; s < cmax; ++s)
      if (fid[s] == f) { for (int c = 0; c < 3; ++c) wp[3 * s + c] = v[c]; return; }
  }
  void remove_collision(int ll, int f) {
    int* fid = &wall_fid[(size_t)ll * cmax];
    for (int s = 0; s < cmax; ++s) if (fid[s] == f) { fid[s] = -1; return; }
  }

  // CALC_DEM_FORCE_WITH_WALL_STL (calc_collision_wall_mod.f:180-629) for one
  // particle, spheres only, static walls (CFRELVEL_WALL 806-847 with zero
  // wall velocity).
  int wall_force_one(int ll, int64_t& nwc) {
    if (state[ll] != DEM_STATE_NORMAL) return 0;
    int cell = dg_pijk[ll] - 1;
    int fs = fbin_start[cell], fe = fbin_start[cell + 1];
    if (fe - fs < 1) {
      for (int s = 0; s < cmax; ++s) wall_fid[(size_t)ll * cmax + s] = -1;
      for (int s = 0; s < 3 * cmax; ++s) wall_pft[(size_t)ll * cmax * 3 + s] = 0.0;
      return 0;
    }
    const double r = rad[ll];
    const double radsq = r * r;
    double xp[3] = {P(pos, ll, 0), P(pos, ll, 1), P(pos, ll, 2)};
    double v[3] = {P(vel, ll, 0), P(vel, ll, 1), P(vel, ll, 2)};
    double w[3] = {P(omg, ll, 0), P(omg, ll, 1), P(omg, ll, 2)};
    double pmax[3], pmin[3];
    for (int c = 0; c < 3; ++c) { pmax[c] = xp[c] + r; pmin[c] = xp[c] - r; }
    const int ph = phase[ll];
    for (int q = fs; q < fe; ++q) {
      const FacetEntry& fe_ = fbin[q];
      int nf_ = fe_.id;
      if (fe_.mn > pmax[fe_.dir]) { remove_collision(ll, nf_); continue; }
      if (fe_.mx < pmin[fe_.dir]) { remove_collision(ll, nf_); continue; }
      double d1[3] = {V(nf_,0,0) - xp[0], V(nf_,0,1) - xp[1], V(nf_,0,2) - xp[2]};
      double line_t = dot3(d1, &norm_face[3 * (size_t)nf_]);
      if (line_t <= -1.0001 * r) { remove_collision(ll, nf_); continue; }
      double cpt[3]; bool poe; int edge;
      closest_pt(nf_, xp, cpt, poe, edge);
      double dist[3] = {cpt[0] - xp[0], cpt[1] - xp[1], cpt[2] - xp[2]};
      double distsq = dot3(dist, dist);
      if (distsq >= radsq - SMALL_NUMBER) { remove_collision(ll, nf_); continue; }
      if (poe && ignore_edge[(size_t)nf_ * 4 + edge]) continue;
      double distmod = std::sqrt(distsq);
      double nrm[3] = {dist[0], dist[1], dist[2]};
      if (distsq > 0) { double s = std::sqrt(distsq); for (int c = 0; c < 3; ++c) nrm[c] = dist[c] / s; }
      double overlap_n = r - distmod;
      double wxn[3]; cross3(w, nrm, wxn);
      double vrot[3] = {distmod * wxn[0], distmod * wxn[1], distmod * wxn[2]};
      double vrel[3];
      for (int c = 0; c < 3; ++c) { vrel[c] = v[c] + vrot[c]; vrel[c] = vrel[c] - (0.0 + 0.0); }
      double vrn = dot3(vrel, nrm);
      double vt[3] = {vrel[0] - vrn * nrm[0], vrel[1] - vrn * nrm[1], vrel[2] - vrn * nrm[2]};
      double kn_w, kt_w, etan_w, etat_w;
      if (p.coll_model == DEM_COLL_HERTZ) {
        double so = 0.0;
        if (overlap_n > 0) so = std::sqrt(overlap_n);
        kn_w = p.hert_kwn[ph] * so * std::sqrt(r);
        kt_w = p.hert_kwt[ph] * so * std::sqrt(r);
        etan_w = p.des_etan_wall[ph] * std::sqrt(so) * std::sqrt(p.hert_kwn[ph] * std::sqrt(r) * pmass[ll]);
        etat_w = p.des_etat_wall[ph] * std::sqrt(so) * std::sqrt(p.hert_kwt[ph] * std::sqrt(r) * pmass[ll]);
      } else {
        kn_w = p.kn_w; kt_w = p.kt_w;
        etan_w = p.des_etan_wall[ph] * std::sqrt(pmass[ll]);
        etat_w = p.des_etat_wall[ph] * std::sqrt(pmass[ll]);
      }
      double fn[3];
      for (int c = 0; c < 3; ++c) fn[c] = -(kn_w * overlap_n * nrm[c] + etan_w * vrn * nrm[c]);
      double hist[3];
      int rc = get_collision(ll, nf_, hist);
      if (rc) return rc;
      double ot[3];
      for (int c = 0; c < 3; ++c) ot[c] = p.dtsolid * vt[c] + hist[c];
      double mag = std::sqrt(dot3(ot, ot));
      double ft[3];
      if (mag > 0.0) {
        for (int c = 0; c < 3; ++c) ft[c] = -kt_w * ot[c] - etat_w * vt[c];
        double ftmd = std::sqrt(dot3(ft, ft));
        double fnmd = p.mew_w * std::sqrt(dot3(fn, fn));
        if (ftmd > fnmd) {
          double tg[3];
          for (int c = 0; c < 3; ++c) tg[c] = ot[c] / mag;
          for (int c = 0; c < 3; ++c) ft[c] = -fnmd * tg[c];
          for (int c = 0; c < 3; ++c) ot[c] = (fnmd / kt_w) * tg[c];
        }
      } else {
        ft[0] = ft[1] = ft[2] = 0.0;
      }
      update_collision(ll, nf_, ot);
      nwc++;
      for (int c = 0; c < 3; ++c) X(fc, c)[ll] = X(fc, c)[ll] + fn[c] + ft[c];
      double nxf[3]; cross3(nrm, ft, nxf);
      for (int c = 0; c < 3; ++c) X(tow, c)[ll] = X(tow, c)[ll] + distmod * nxf[c];
      if (p.mew_rw > 0.0) {
        double om = std::sqrt(dot3(w, w));
        if (om > 0.0) {
          for (int c = 0; c < 3; ++c) {
            double rf = -(p.mew_rw * (2.0 * r) * kn_w * overlap_n * w[c] / om);
            X(tow, c)[ll] = X(tow, c)[ll] + rf;
          }
        }
      }
    }
    return 0;
  }

  // One pair of CALC_FORCE_DEM (calc_force_dem.f:204-506) with CFRELVEL
  // (cfrelvel.f:54-77).  Returns 0 and fills outputs; *contact = false when
  // the pair is apart (history reset).
  struct PairOut {
    double fc[3], tl[3], ti[3], rl[3], ri[3];
    bool contact, roll_l, roll_i;
  };
  int pair_force(int ll, int i, const double* pft_in, double* pft_out, PairOut& o) const {
    o.contact = false; o.roll_l = o.roll_i = false;
    double rl = rad[ll], ri = rad[i];
    double r_lm = rl + ri;
    double dist[3];
    pair_dist(ll, i, dist);
    double dmag = dot3(dist, dist);
    double fct[3] = {0.0, 0.0, 0.0};
    if (dmag > (r_lm - SMALL_NUMBER) * (r_lm - SMALL_NUMBER)) {
      pft_out[0] = pft_out[1] = pft_out[2] = 0.0;
      return 0;
    }
    if (dmag == 0) return DEM_ERR_ZERO_DISTANCE;
    dmag = std::sqrt(dmag);
    double nrm[3] = {dist[0] / dmag, dist[1] / dmag, dist[2] / dmag};
    double overlap_n = r_lm - dmag;
    // CFRELVEL
    double vrel[3];
    for (int c = 0; c < 3; ++c) vrel[c] = P(vel, ll, c) - P(vel, i, c);
    double dcl = (dmag * dmag + rl * rl - ri * ri) / (2.0 * dmag);
    double dci = dmag - dcl;
    double osum[3];
    for (int c = 0; c < 3; ++c) osum[c] = P(omg, ll, c) * dcl + P(omg, i, c) * dci;
    double vrot[3]; cross3(osum, nrm, vrot);
    for (int c = 0; c < 3; ++c) vrel[c] = vrel[c] + vrot[c];
    double vrn = dot3(vrel, nrm);
    double vt[3] = {vrel[0] - vrn * nrm[0], vrel[1] - vrn * nrm[1], vrel[2] - vrn * nrm[2]};
    int pl = phase[ll], pi_ = phase[i];
    int ix = pl * DEM_MAX_PHASES + pi_;
    double rad_eff = (rl * ri) / (rl + ri);
    double m_eff = (pmass[ll] * pmass[i]) / (pmass[ll] + pmass[i]);
    double kn, kt, etan, etat;
    if (p.coll_model == DEM_COLL_HERTZ) {
      double so = std::sqrt(overlap_n);
      kn = p.hert_kn[ix] * so * std::sqrt(rad_eff);
      kt = p.hert_kt[ix] * so * std::sqrt(rad_eff);
      so = std::sqrt(so);
      etan = p.des_etan[ix] * so * std::sqrt(p.hert_kn[ix] * std::sqrt(rad_eff) * m_eff);
      etat = p.des_etat[ix] * so * std::sqrt(p.hert_kt[ix] * std::sqrt(rad_eff) * m_eff);
    } else {
      kn = p.kn; kt = p.kt;
      etan = p.des_etan[ix] * std::sqrt(m_eff);
      etat = p.des_etat[ix] * std::sqrt(m_eff);
    }
    double fn[3];
    for (int c = 0; c < 3; ++c) fn[c] = -(kn * overlap_n * nrm[c] + etan * vrn * nrm[c]);
    double ot[3];
    for (int c = 0; c < 3; ++c) ot[c] = p.dtsolid * vt[c] + pft_in[c];
    double mag = std::sqrt(dot3(ot, ot));
    double ft[3];
    if (mag > 0.0) {
      for (int c = 0; c < 3; ++c) ft[c] = -kt * ot[c] - etat * vt[c];
      double ftmd = std::sqrt(dot3(ft, ft));
      double fnmd = p.mew * std::sqrt(dot3(fn, fn));
      if (ftmd > fnmd) {
        double tg[3];
        for (int c = 0; c < 3; ++c) tg[c] = ot[c] / mag;
        for (int c = 0; c < 3; ++c) ft[c] = -fnmd * tg[c];
        for (int c = 0; c < 3; ++c) ot[c] = (fnmd / kt) * tg[c];
      }
    } else {
      ft[0] = ft[1] = ft[2] = 0.0;
    }
    for (int c = 0; c < 3; ++c) pft_out[c] = ot[c];
    double dcl2 = dmag / 2.0 + (rl * rl - ri * ri) / (2.0 * dmag);
    double dci2 = dmag - dcl2;
    double tf[3]; cross3(nrm, ft, tf);
    for (int c = 0; c < 3; ++c) { o.tl[c] = dcl2 * tf[c]; o.ti[c] = dci2 * tf[c]; }
    for (int c = 0; c < 3; ++c) fct[c] = fct[c] + fn[c] + ft[c];
    for (int c = 0; c < 3; ++c) o.fc[c] = fct[c];
    if (p.mew_r > 0.0) {
      double wl[3] = {P(omg, ll, 0), P(omg, ll, 1), P(omg, ll, 2)};
      double om = std::sqrt(dot3(wl, wl));
      if (om > 0.0) {
        o.roll_l = true;
        for (int c = 0; c < 3; ++c) o.rl[c] = -(p.mew_r * (2.0 * rl) * kn * overlap_n * wl[c] / om);
      }
      double wi[3] = {P(omg, i, 0), P(omg, i, 1), P(omg, i, 2)};
      om = std::sqrt(dot3(wi, wi));
      if (om > 0.0) {
        o.roll_i = true;
        for (int c = 0; c < 3; ++c) o.ri[c] = -(p.mew_r * (2.0 * ri) * kn * overlap_n * wi[c] / om);
      }
    }
    o.contact = true;
    return 0;
  }

  // CALC_FORCE_DEM (calc_force_dem.f:18-544), serial order: walls first, then
  // LL ascending, CC ascending, scattering into FC/TOW.
  // CALC_FORCE_DEM adds to FC/TOW, which CFNEWVALUES leaves at zero
  // (cfnewvalues.f:709-723); the entry point starts from zero so that a
  // force evaluation outside the DES_TIME_STEP sequence (forces taken and not
  // integrated) does not carry into the next one -- the CUDA library's
  // dem_calc_force stores the sums the same way.
  int calc_force() {
    std::fill(fc.begin(), fc.end(), 0.0);
    std::fill(tow.begin(), tow.end(), 0.0);
    n_contacts = 0; n_wall_contacts = 0; max_overlap_ratio = 0.0;
    int wrc = 0;
    int64_t nwc = 0;
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads) if (nthreads > 1) reduction(+ : nwc)
    for (int ll = 0; ll < n; ++ll) {
      int64_t c0 = 0;
      int rc = wall_force_one(ll, c0);
      nwc += c0;
      if (rc) wrc = rc;
    }
    n_wall_contacts = nwc;
    if (wrc) return fail(wrc, "COLLISION_ARRAY_MAX too small");
#ifdef _OPENMP
    if (nthreads > 1) return calc_force_omp();
#endif
    for (int ll = 0; ll < n; ++ll) {
      if (state[ll] == DEM_STATE_NONEXISTENT) continue;
      int s = ll ? row_end[ll - 1] : 0, e = row_end[ll];
      for (int cc = s; cc < e; ++cc) {
        int i = nbrs[cc];
        if (state[i] == DEM_STATE_NONEXISTENT) continue;
        PairOut o;
        double* pf = &pft[3 * (size_t)cc];
        double in[3] = {pf[0], pf[1], pf[2]};
        int rc = pair_force(ll, i, in, pf, o);
        if (rc) { char b[96]; snprintf(b, sizeof b, "distance between particles is zero: %d %d", ll + 1, i + 1); return fail(rc, b); }
        if (!o.contact) continue;
        n_contacts++;
        for (int c = 0; c < 3; ++c) { X(fc, c)[ll] = X(fc, c)[ll] + o.fc[c]; }
        for (int c = 0; c < 3; ++c) { X(fc, c)[i] = X(fc, c)[i] - o.fc[c]; }
        for (int c = 0; c < 3; ++c) { X(tow, c)[ll] = X(tow, c)[ll] + o.tl[c]; }
        for (int c = 0; c < 3; ++c) { X(tow, c)[i] = X(tow, c)[i] + o.ti[c]; }
        if (o.roll_l) for (int c = 0; c < 3; ++c) X(tow, c)[ll] = X(tow, c)[ll] + o.rl[c];
        if (o.roll_i) for (int c = 0; c < 3; ++c) X(tow, c)[i] = X(tow, c)[i] + o.ri[c];
      }
    }
    return 0;
  }

#ifdef _OPENMP
  // OpenMP mode of the same loop (the reference's SMP build: !$omp do over
  // LL with !$omp atomic scatter, calc_force_dem.f:139-412).  Used only to
  // time the CPU baseline; its summation order is not deterministic.
  int calc_force_omp() {
    int rc_all = 0;
    int64_t ncont = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads) reduction(+ : ncont)
    for (int ll = 0; ll < n; ++ll) {
      if (state[ll] == DEM_STATE_NONEXISTENT) continue;
      int s = ll ? row_end[ll - 1] : 0, e = row_end[ll];
      for (int cc = s; cc < e; ++cc) {
        int i = nbrs[cc];
        if (state[i] == DEM_STATE_NONEXISTENT) continue;
        PairOut o;
        double* pf = &pft[3 * (size_t)cc];
        double in[3] = {pf[0], pf[1], pf[2]};
        int rc = pair_force(ll, i, in, pf, o);
        if (rc) { rc_all = rc; continue; }
        if (!o.contact) continue;
        ncont++;
        for (int c = 0; c < 3; ++c) {
#pragma omp atomic
          fc[(size_t)c * n + ll] += o.fc[c];
#pragma omp atomic
          fc[(size_t)c * n + i] -= o.fc[c];
#pragma omp atomic
          tow[(size_t)c * n + ll] += o.tl[c];
#pragma omp atomic
          tow[(size_t)c * n + i] += o.ti[c];
          if (o.roll_l) {
#pragma omp atomic
            tow[(size_t)c * n + ll] += o.rl[c];
          }
          if (o.roll_i) {
#pragma omp atomic
            tow[(size_t)c * n + i] += o.ri[c];
          }
        }
      }
    }
    n_contacts = ncont;
    if (rc_all) return fail(rc_all, "distance between particles is zero");
    return 0;
  }
#endif

  // CFUPDATEOLD + CFNEWVALUES (cfupdateold.f:33-41, cfnewvalues.f:669-812).
  void cfnewvalues() {
    const double dt = p.dtsolid;
    if (first_pass && p.intg_method == DEM_INTG_AB2) {
      for (int l = 0; l < n; ++l) {
        // cfnewvalues.f:672-676: skip NONEXISTENT, ENTERING(_GHOST), GHOST and
        // RIGID_MOTION_GHOST (functions.inc:858-880).
        int s = state[l];
        if (s == DEM_STATE_NONEXISTENT || s == DEM_STATE_ENTERING || s == 102) continue;
        if (s == DEM_STATE_NORMAL_GHOST || s == 110) continue;
        for (int c = 0; c < 3; ++c) {
          X(acc_old, c)[l] = P(fc, l, c) / pmass[l] + p.grav[c];
          X(rot_acc_old, c)[l] = P(tow, l, c);
        }
      }
    }
    if (p.intg_method == DEM_INTG_EULER) {
      for (int c = 0; c < 3; ++c) {
        double* v = X(vel, c); double* x = X(pos, c); double* f = X(fc, c);
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
        for (int l = 0; l < n; ++l) {
          if (state[l] == DEM_STATE_NORMAL) v[l] = v[l] + dt * (f[l] / pmass[l] + p.grav[c]);
          if (state[l] < DEM_STATE_NORMAL_GHOST) x[l] = x[l] + v[l] * dt;
          f[l] = 0.0;
        }
      }
      for (int c = 0; c < 3; ++c) {
        double* w = X(omg, c); double* t = X(tow, c);
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
        for (int l = 0; l < n; ++l) {
          if (state[l] == DEM_STATE_NORMAL) w[l] = w[l] + t[l] * omoi[l] * dt;
          t[l] = 0.0;
        }
      }
    } else {
      for (int c = 0; c < 3; ++c) {
        double* v = X(vel, c); double* x = X(pos, c); double* f = X(fc, c); double* a = X(acc_old, c);
        for (int l = 0; l < n; ++l) {
          // CFUPDATEOLD copies NEW into OLD for existing non-ghost particles.
          double vold = vel_old.empty() ? v[l] : X(vel_old, c)[l], xold = x[l];
          if (state[l] == DEM_STATE_NORMAL) f[l] = f[l] / pmass[l] + p.grav[c];
          if (state[l] == DEM_STATE_NORMAL) v[l] = vold + 0.5 * (3.0 * f[l] - a[l]) * dt;
          a[l] = f[l];
          if (state[l] < DEM_STATE_NORMAL_GHOST) x[l] = xold + 0.5 * (vold + v[l]) * dt;
          f[l] = 0.0;
        }
      }
      for (int c = 0; c < 3; ++c) {
        double* w = X(omg, c); double* t = X(tow, c); double* ra = X(rot_acc_old, c);
        for (int l = 0; l < n; ++l) {
          double wold = w[l];
          if (state[l] == DEM_STATE_NORMAL) w[l] = wold + 0.5 * (3.0 * t[l] * omoi[l] - ra[l]) * dt;
          if (state[l] == DEM_STATE_NORMAL) ra[l] = t[l] * omoi[l];
          t[l] = 0.0;
        }
      }
    }
    first_pass = false;
  }

  // ---------------------------------------------------------------------
  // CFD-DEM coupling, GARG_2012 interpolation (drag_gs_des0.f,
  // comp_mean_fields0.f, calc_epg_des.f, particles_in_cell.f).
  int cijk(int i, int j, int k) const { return (i - 1) + (j - 1) * gi2 + (k - 1) * gi2 * gj2; }  // 0-based
  bool fluid_at(int i, int j, int k) const {
    return i >= 2 && i <= g.imax + 1 && j >= 2 && j <= g.jmax + 1 &&
           (p.no_k ? k == 1 : (k >= 2 && k <= g.kmax + 1));
  }
  double vol() const { return g.dx * g.dy * (p.no_k ? (p.domain_hi[2] - p.domain_lo[2]) : g.dz); }

  void gas_setup() {
    gi2 = g.imax + 2; gj2 = g.jmax + 2; gk2 = p.no_k ? 1 : g.kmax + 2;
    auto faces = [](double lo, double d, int nc) {
      std::vector<double> f(nc + 3);
      f[1] = lo;
      f[0] = lo - d;
      for (int i = 2; i <= nc + 2; ++i) f[i] = f[i - 1] + d;
      return f;
    };
    xe = faces(p.domain_lo[0], g.dx, g.imax);
    yn = faces(p.domain_lo[1], g.dy, g.jmax);
    zt = faces(p.domain_lo[2], g.dz, p.no_k ? 0 : g.kmax);
    // VOL_SURR (make_arrays_des.f:78-105): fluid volume of the cells that
    // share node (I,J,K), nodes I = ISTART2..IEND1
    vol_surr.assign((size_t)gi2 * gj2 * gk2, 0.0);
    const int kk0 = p.no_k ? 1 : 1, kk1 = p.no_k ? 1 : g.kmax + 1;
    for (int k = kk0; k <= kk1; ++k)
      for (int j = 1; j <= g.jmax + 1; ++j)
        for (int i = 1; i <= g.imax + 1; ++i) {
          double v = 0.0;
          for (int kk = k; kk <= (p.no_k ? k : k + 1); ++kk)
            for (int jj = j; jj <= j + 1; ++jj)
              for (int ii = i; ii <= i + 1; ++ii)
                if (fluid_at(ii, jj, kk)) v = v + vol();
          vol_surr[cijk(i, j, k)] = v;
        }
    // DES_VOL_NODE (cfassign.f:104-228): a quarter (2D) or an eighth (3D)
    // of the volume of each fluid cell sharing node (I,J,K), summed in the
    // reference's order (the k+1 plane as ijkp, ipjpkp, ijpkp, ipjkp)
    vol_node.assign(vol_surr.size(), 0.0);
    const double avn = p.no_k ? 0.25 : 0.125;
    auto fv = [&](int i, int j, int k) { return fluid_at(i, j, k) ? vol() : 0.0; };
    for (int k = kk0; k <= kk1; ++k)
      for (int j = 1; j <= g.jmax + 1; ++j)
        for (int i = 1; i <= g.imax + 1; ++i) {
          double v = avn * (fv(i, j, k) + fv(i + 1, j, k) + fv(i, j + 1, k) + fv(i + 1, j + 1, k));
          if (!p.no_k)
            v = v + avn * (fv(i, j, k + 1) + fv(i + 1, j + 1, k + 1) + fv(i, j + 1, k + 1) + fv(i + 1, j, k + 1));
          vol_node[cijk(i, j, k)] = v;
        }
    pijk.assign((size_t)4 * n, 0);
    f_gp.assign(n, 0.0);
  }

  // PIC_SEARCH (particles_in_cell.f:347-370): first IDX in [1, nc+2] with
  // faces[IDX-1] <= x < faces[IDX]; nc+3 when there is none.
  static int pic_search(const std::vector<double>& f, int nc, double x) {
    for (int idx = 1; idx <= nc + 2; ++idx)
      if (x >= f[idx - 1] && x < f[idx]) return idx;
    return nc + 3;
  }

  // PARTICLES_IN_CELL (particles_in_cell.f:20-234): fluid cell of every
  // particle, per-cell lists in ascending particle order; particles outside
  // the grid are deleted.
  void particles_in_cell() {
    std::vector<int> cnt(vol_surr.size(), 0);
    for (int l = 0; l < n; ++l) {
      if (state[l] == DEM_STATE_NONEXISTENT) continue;
      int i = pic_search(xe, g.imax, P(pos, l, 0));
      int j = pic_search(yn, g.jmax, P(pos, l, 1));
      int k = p.no_k ? 1 : pic_search(zt, g.kmax, P(pos, l, 2));
      bool on = i >= 1 && i <= gi2 && j >= 1 && j <= gj2 && k >= 1 && k <= gk2;
      if (!on) { delete_particle(l); for (int c = 0; c < 4; ++c) pijk[4 * (size_t)l + c] = 0; continue; }
      pijk[4 * (size_t)l] = i; pijk[4 * (size_t)l + 1] = j; pijk[4 * (size_t)l + 2] = k;
      pijk[4 * (size_t)l + 3] = cijk(i, j, k) + 1;
      if (state[l] < DEM_STATE_NORMAL_GHOST) cnt[cijk(i, j, k)]++;
    }
    pic_start.assign(cnt.size() + 1, 0);
    for (size_t c = 0; c < cnt.size(); ++c) pic_start[c + 1] = pic_start[c] + cnt[c];
    pic_list.assign(pic_start.back(), 0);
    std::vector<int> fill(pic_start.begin(), pic_start.end() - 1);
    for (int l = 0; l < n; ++l) {
      if (state[l] == DEM_STATE_NONEXISTENT || state[l] >= DEM_STATE_NORMAL_GHOST) continue;
      pic_list[fill[pijk[4 * (size_t)l + 3] - 1]++] = l;
    }
  }

  // Trilinear weights in the cell whose west/south/bottom node is
  // (xe[i-1], yn[j-1], zt[k-1]) -- DRAG_WEIGHTFACTOR (comp_mean_fields0.f:
  // 478-530) and the weights of DRAG_INTERPOLATION (drag_gs_des0.f:507-566).
  void weights(int i, int j, int k, const double x[3], double w[2][2][2]) const {
    const double dxx = xe[i] - xe[i - 1], dyy = yn[j] - yn[j - 1];
    double z0 = (x[0] - xe[i - 1]) / dxx, z1 = (x[1] - yn[j - 1]) / dyy;
    double xx[2] = {1 - z0, z0}, yy[2] = {1 - z1, z1};
    if (p.no_k) {
      for (int jj = 0; jj < 2; ++jj) for (int ii = 0; ii < 2; ++ii) w[0][jj][ii] = xx[ii] * yy[jj];
    } else {
      const double dzz = zt[k] - zt[k - 1];
      double z2 = (x[2] - zt[k - 1]) / dzz;
      double zz[2] = {1 - z2, z2};
      for (int kk = 0; kk < 2; ++kk) for (int jj = 0; jj < 2; ++jj) for (int ii = 0; ii < 2; ++ii)
        w[kk][jj][ii] = xx[ii] * yy[jj] * zz[kk];
    }
  }

  // DRAG_GIDASPOW (drag_gs.f:536-598) with C_DS_SN (drag_mod.f:54).
  static double drag_gidaspow(double epg, double mug, double rog, double ropg, double vrel, double dpm) {
    const double LARGE_NUMBER = 1.0e32;
    double re = mug > 0.0 ? dpm * vrel * ropg / mug : LARGE_NUMBER;
    if (re == 0.0) return 0.0;
    if (epg <= 0.8) return 150.0 * (1.0 - epg) * mug / (epg * (dpm * dpm)) + 1.75 * rog * vrel / dpm;
    double cd = re <= 1000.0 ? 24.0 * (1.0 + 0.15 * std::pow(re, 0.687)) / (re + SMALL_NUMBER) : 0.44;
    return 0.75 * cd * vrel * ropg * std::pow(epg, -2.65) / dpm;
  }

  // The DEM06 regression's user drag (usr_drag.f with usr_mod.f Re, Cd):
  // 0.75*(RO_g*VREL/DPM)*Cd(Re), Re = (RO_g0*D_p0*Vs)/MU_g0,
  // Cd = (24/Re)*(1 + 0.15*Re**0.687) with a default-real exponent.
  static double drag_single_sphere(double mug, double rog, double vrel, double dpm, double dref) {
    const double re = (rog * dref * vrel) / mug;
    double cd = 0.0;
    if (re > 0.0) cd = (24.0 / re) * (1.0 + 0.15 * std::pow(re, (double)0.687f));
    return 0.75 * (rog * vrel / dpm) * cd;
  }

  // Gas velocity at a particle of fluid cell (i,j,k): the staggered face
  // velocities averaged to the 2x2x2 node stencil and interpolated with the
  // trilinear weights (drag_gs_des0.f:117-170 and 313-361,
  // DRAG_INTERPOLATION drag_gs_des0.f:507-566).  Returns the weights too.
  void gas_velocity(int l, int i, int j, int k, double velfp[3], double w[2][2][2]) const {
    const double avg = p.no_k ? 0.5 : 0.25;
    const int iw = i - 1, js = j - 1, kb = p.no_k ? 1 : k - 1;
    double vst[2][2][2][3];
    for (int kk = 0; kk < (p.no_k ? 1 : 2); ++kk)
      for (int jj = 0; jj < 2; ++jj)
        for (int ii = 0; ii < 2; ++ii) {
          int I = iw + ii, J = js + jj, K = kb + kk;
          int c = cijk(I, J, K), ipjk = cijk(I + 1, J, K), ijpk = cijk(I, J + 1, K), ipjpk = cijk(I + 1, J + 1, K);
          double* v = vst[kk][jj][ii];
          v[0] = avg * (u_g[c] + u_g[ijpk]);
          v[1] = avg * (v_g[c] + v_g[ipjk]);
          if (!p.no_k) {
            int ijpkp = cijk(I, J + 1, K + 1), ipjkp = cijk(I + 1, J, K + 1), ijkp = cijk(I, J, K + 1);
            v[0] = v[0] + avg * (u_g[ijkp] + u_g[ijpkp]);
            v[1] = v[1] + avg * (v_g[ijkp] + v_g[ipjkp]);
            v[2] = avg * (w_g[c] + w_g[ijpk] + w_g[ipjk] + w_g[ipjpk]);
          } else {
            v[2] = 0.0;
          }
        }
    double x[3] = {P(pos, l, 0), P(pos, l, 1), P(pos, l, 2)};
    weights(i, j, k, x, w);
    velfp[0] = velfp[1] = velfp[2] = 0.0;
    for (int kk = 0; kk < (p.no_k ? 1 : 2); ++kk)
      for (int jj = 0; jj < 2; ++jj)
        for (int ii = 0; ii < 2; ++ii)
          for (int c = 0; c < (p.no_k ? 2 : 3); ++c) velfp[c] = velfp[c] + vst[kk][jj][ii][c] * w[kk][jj][ii];
  }

  // DES_DRAG_GP (drag_gp_des.f:97-257, Model A, Gidaspow): F_GP of particle
  // l in fluid cell ijk with the under-relaxation UR_F_GS; returns PVOL.
  double update_f_gp(int l, int ijk, const double velfp[3]) {
    double vp[3] = {P(vel, l, 0), P(vel, l, 1), P(vel, l, 2)};
    const double epg = ep_g[ijk];
    double vs[3] = {velfp[0] - vp[0], velfp[1] - vp[1], velfp[2] - vp[2]};
    double vrel = std::sqrt(dot3(vs, vs));
    double dpm = 2.0 * rad[l];
    double dga = g.drag_model == DEM_DRAG_SINGLE_SPHERE ? drag_single_sphere(g.mu_g, g.ro_g, vrel, dpm, g.usr_d_p0)
                                                        : drag_gidaspow(epg, g.mu_g, g.ro_g, g.ro_g * epg, vrel, dpm);
    double pvol = ((4.0 / 3.0) * pi_c) * (rad[l] * (rad[l] * rad[l]));
    double fgs = dga * pvol;
    f_gp[l] = (1.0 - g.ur_f_gs) * f_gp[l] + g.ur_f_gs * fgs;
    return pvol;
  }

  // DRAG_GS_DES0 (drag_gs_des0.f:22-219): gas velocity at the particle,
  // DES_DRAG_GP and FC += F_GP*(u_g - v_p) + P_FORCE*PVOL.
  void drag() {
    for (int l = 0; l < n; ++l) {
      int8_t st = state[l];
      if (st == DEM_STATE_NONEXISTENT || st >= DEM_STATE_NORMAL_GHOST) continue;
      int i = pijk[4 * (size_t)l], j = pijk[4 * (size_t)l + 1], k = pijk[4 * (size_t)l + 2];
      if (!fluid_at(i, j, k)) continue;
      double velfp[3], w[2][2][2];
      gas_velocity(l, i, j, k, velfp, w);
      const int ijk = cijk(i, j, k);
      const double pvol = update_f_gp(l, ijk, velfp);
      double vp[3] = {P(vel, l, 0), P(vel, l, 1), P(vel, l, 2)};
      for (int c = 0; c < 3; ++c) X(fc, c)[l] = X(fc, c)[l] + f_gp[l] * (velfp[c] - vp[c]);
      if (!p_force.empty())
        for (int c = 0; c < 3; ++c) X(fc, c)[l] = X(fc, c)[l] + p_force[3 * (size_t)ijk + c] * pvol;
    }
  }

  // DRAG_GS_GAS0 (drag_gs_des0.f:235-497): per fluid cell in IJK order and
  // per particle in PIC order, F_GP again (DES_DRAG_GP) and its deposition
  // to the cell's 2x2x2 nodes, DRAG_AM += F_GP*W/DES_VOL_NODE and
  // DRAG_BM(:,c) += F_GP*V_p(c)*W/DES_VOL_NODE (statistical weight 1 for
  // DEM); then F_GDS per fluid cell as the mean of its nodes' DRAG_AM
  // (drag_gs_des0.f:451-494), zero elsewhere.  Serial, non-periodic: the
  // node exchange DES_ADDNODEVALUES adds nothing.
  void drag_gas() {
    const size_t nc = vol_surr.size();
    drag_am.assign(nc, 0.0);
    drag_bm.assign(3 * nc, 0.0);
    f_gds.assign(nc, 0.0);
    const double wtp = 1.0;
    for (int k = 1; k <= gk2; ++k)
      for (int j = 1; j <= gj2; ++j)
        for (int i = 1; i <= gi2; ++i) {
          if (!fluid_at(i, j, k)) continue;
          const int ijk = cijk(i, j, k);
          const int iw = i - 1, js = j - 1, kb = p.no_k ? 1 : k - 1;
          for (int q = pic_start[ijk]; q < pic_start[ijk + 1]; ++q) {
            const int np = pic_list[q];
            if (state[np] == DEM_STATE_NONEXISTENT || state[np] >= DEM_STATE_NORMAL_GHOST) continue;
            double velfp[3], w[2][2][2];
            gas_velocity(np, i, j, k, velfp, w);
            update_f_gp(np, ijk, velfp);
            const double vn[3] = {P(vel, np, 0), P(vel, np, 1), P(vel, np, 2)};
            for (int kk = 0; kk < (p.no_k ? 1 : 2); ++kk)
              for (int jj = 0; jj < 2; ++jj)
                for (int ii = 0; ii < 2; ++ii) {
                  const int node = cijk(iw + ii, js + jj, kb + kk);
                  const double ovol = 1.0 / vol_node[node];
                  drag_am[node] = drag_am[node] + f_gp[np] * w[kk][jj][ii] * ovol * wtp;
                  for (int c = 0; c < 3; ++c)
                    drag_bm[c * nc + node] = drag_bm[c * nc + node] + f_gp[np] * vn[c] * w[kk][jj][ii] * ovol * wtp;
                }
          }
        }
    const double avf = p.no_k ? 0.25 : 0.125;
    for (int k = 1; k <= gk2; ++k)
      for (int j = 1; j <= gj2; ++j)
        for (int i = 1; i <= gi2; ++i) {
          const int ijk = cijk(i, j, k);
          if (!fluid_at(i, j, k)) { f_gds[ijk] = 0.0; continue; }
          double f = avf * (drag_am[ijk] + drag_am[cijk(i, j - 1, k)] + drag_am[cijk(i - 1, j - 1, k)] +
                            drag_am[cijk(i - 1, j, k)]);
          if (!p.no_k)
            f = f + avf * (drag_am[cijk(i, j, k - 1)] + drag_am[cijk(i, j - 1, k - 1)] +
                           drag_am[cijk(i - 1, j - 1, k - 1)] + drag_am[cijk(i - 1, j, k - 1)]);
          f_gds[ijk] = f;
        }
  }

  // ---- DES_INTERP_SCHEME = NONE: the ...1 routines without a filter ----

  // PVOL (generate_particles_mod.f:1399): 4/3 pi r^3.
  double pvol_of(int l) const { return ((4.0 / 3.0) * pi_c) * (rad[l] * (rad[l] * rad[l])); }

  // CALC_CELL_CENTER_GAS_VEL (drag_gs_des1.f:313-370) on a uniform grid
  // (FX = FX_BAR = 1/2, set_geometry.f:344-345): the gas velocity at the
  // centre of fluid cell (i,j,k); zero outside the fluid.
  void cell_center_vel(int i, int j, int k, double v[3]) const {
    if (!fluid_at(i, j, k)) { v[0] = v[1] = v[2] = 0.0; return; }
    const int ijk = cijk(i, j, k);
    v[0] = 0.5 * u_g[cijk(i - 1, j, k)] + 0.5 * u_g[ijk];     // AVG_X_E
    v[1] = 0.5 * (v_g[cijk(i, j - 1, k)] + v_g[ijk]);         // AVG_Y_N
    v[2] = p.no_k ? 0.0 : 0.5 * (w_g[cijk(i, j, k - 1)] + w_g[ijk]);   // AVG_Z_T
  }

  // COMP_MEAN_FIELDS1 with FILTER_SIZE = 0 (comp_mean_fields1.f:46-104):
  // SOLVOLINC(PIJK(NP,4), M) += PVOL(NP) over NORMAL particles in index
  // order, ROP_S = RO_S*SOLVOLINC/VOL on fluid cells; then CALC_EPG_DES.
  void comp_mean_fields1() {
    const size_t nc = vol_surr.size();
    const int M = p.n_phases;
    std::vector<double> solvolinc(nc * M, 0.0);
    rop_s.assign(nc * M, 0.0);
    for (int l = 0; l < n; ++l) {
      if (state[l] != DEM_STATE_NORMAL) continue;
      const int ijk = pijk[4 * (size_t)l + 3] - 1;
      double& sv = solvolinc[(size_t)phase[l] * nc + ijk];
      sv = sv + pvol_of(l);
    }
    for (int k = 1; k <= gk2; ++k)
      for (int j = 1; j <= gj2; ++j)
        for (int i = 1; i <= gi2; ++i) {
          if (!fluid_at(i, j, k)) continue;
          const int ijk = cijk(i, j, k);
          for (int m = 0; m < M; ++m)
            rop_s[(size_t)m * nc + ijk] = ro_s[m] * solvolinc[(size_t)m * nc + ijk] / vol();
          double sum_eps = 0.0;
          for (int m = 0; m < M; ++m) sum_eps = sum_eps + rop_s[(size_t)m * nc + ijk] / ro_s[m];
          ep_g[ijk] = 1.0 - std::min(1.0, sum_eps);
        }
  }

  // DRAG_GS_DES1 without a filter (drag_gs_des1.f:34-160, Model A, not
  // explicitly coupled): per NORMAL particle the cell-centre gas velocity of
  // its cell, DES_DRAG_GP with EP_G of the cell, FC += F_GP*(u_g - v_p) +
  // P_FORCE*PVOL; F_GP = 0 for a particle outside the fluid cells.
  void drag_des1() {
    for (int l = 0; l < n; ++l) {
      if (state[l] != DEM_STATE_NORMAL) continue;
      const int i = pijk[4 * (size_t)l], j = pijk[4 * (size_t)l + 1], k = pijk[4 * (size_t)l + 2];
      if (!fluid_at(i, j, k)) { f_gp[l] = 0.0; continue; }
      const int ijk = cijk(i, j, k);
      double velfp[3];
      cell_center_vel(i, j, k, velfp);
      const double pvol = update_f_gp(l, ijk, velfp);
      double vp[3] = {P(vel, l, 0), P(vel, l, 1), P(vel, l, 2)};
      for (int c = 0; c < 3; ++c) X(fc, c)[l] = X(fc, c)[l] + f_gp[l] * (velfp[c] - vp[c]);
      if (!p_force.empty())
        for (int c = 0; c < 3; ++c) X(fc, c)[l] = X(fc, c)[l] + p_force[3 * (size_t)ijk + c] * pvol;
    }
  }

  // DRAG_GS_GAS1 without a filter (drag_gs_des1.f:179-301): per NORMAL
  // particle of a fluid cell, in index order, F_GP again and DRAG_BM(IJK,:)
  // += F_GP*V/VOL, F_GDS(IJK) += F_GP/VOL in its own cell; zero elsewhere.
  void drag_gas1() {
    const size_t nc = vol_surr.size();
    drag_bm.assign(3 * nc, 0.0);
    f_gds.assign(nc, 0.0);
    for (int l = 0; l < n; ++l) {
      if (state[l] != DEM_STATE_NORMAL) continue;
      const int i = pijk[4 * (size_t)l], j = pijk[4 * (size_t)l + 1], k = pijk[4 * (size_t)l + 2];
      if (!fluid_at(i, j, k)) continue;
      const int ijk = cijk(i, j, k);
      double velfp[3];
      cell_center_vel(i, j, k, velfp);
      update_f_gp(l, ijk, velfp);
      const double lforce = f_gp[l];
      const double ldbm[3] = {lforce * P(vel, l, 0), lforce * P(vel, l, 1), lforce * P(vel, l, 2)};
      const double weight = 1.0 / vol();
      for (int c = 0; c < 3; ++c) drag_bm[c * nc + ijk] = drag_bm[c * nc + ijk] + ldbm[c] * weight;
      f_gds[ijk] = f_gds[ijk] + lforce * weight;
    }
  }

  // COMP_MEAN_FIELDS0 (comp_mean_fields0.f:139-435) + CALC_EPG_DES
  // (calc_epg_des.f:123-150), one solids phase per particle phase.
  void comp_mean_fields() {
    particles_in_cell();
    if (g.interp_scheme == DEM_INTERP_NONE) { comp_mean_fields1(); return; }
    const size_t nc = vol_surr.size();
    const int M = p.n_phases;
    std::vector<double> rops_node(nc * M, 0.0);
    rop_s.assign(nc * M, 0.0);
    for (int k = 1; k <= gk2; ++k)
      for (int j = 1; j <= gj2; ++j)
        for (int i = 1; i <= gi2; ++i) {
          if (!fluid_at(i, j, k)) continue;
          const int ijk = cijk(i, j, k);
          const int iw = i - 1, js = j - 1, kb = p.no_k ? 1 : k - 1;
          for (int q = pic_start[ijk]; q < pic_start[ijk + 1]; ++q) {
            int np = pic_list[q];
            double x[3] = {P(pos, np, 0), P(pos, np, 1), P(pos, np, 2)};
            double w[2][2][2];
            weights(i, j, k, x, w);
            const int m = phase[np];
            const double temp2 = pmass[np];
            for (int kk = 0; kk < (p.no_k ? 1 : 2); ++kk)
              for (int jj = 0; jj < 2; ++jj)
                for (int ii = 0; ii < 2; ++ii) {
                  int node = cijk(iw + ii, js + jj, kb + kk);
                  double temp1 = w[kk][jj][ii] * temp2;
                  rops_node[(size_t)m * nc + node] = rops_node[(size_t)m * nc + node] + temp1;
                }
          }
        }
    const int kn1 = p.no_k ? 1 : g.kmax + 1;
    for (int k = 1; k <= kn1; ++k)
      for (int j = 1; j <= g.jmax + 1; ++j)
        for (int i = 1; i <= g.imax + 1; ++i) {
          const int ijk = cijk(i, j, k);
          if (vol_surr[ijk] == 0.0) continue;
          for (int m = 0; m < M; ++m) {
            double dens = rops_node[(size_t)m * nc + ijk] / vol_surr[ijk];
            for (int kk = k; kk <= (p.no_k ? k : k + 1); ++kk)
              for (int jj = j; jj <= j + 1; ++jj)
                for (int ii = i; ii <= i + 1; ++ii) {
                  int c2 = cijk(ii, jj, kk);
                  rop_s[(size_t)m * nc + c2] = rop_s[(size_t)m * nc + c2] + dens * vol();
                }
          }
        }
    for (int k = 1; k <= gk2; ++k)
      for (int j = 1; j <= gj2; ++j)
        for (int i = 1; i <= gi2; ++i) {
          if (!fluid_at(i, j, k)) continue;
          const int ijk = cijk(i, j, k);
          double sum_eps = 0.0;
          for (int m = 0; m < M; ++m) {
            double& r = rop_s[(size_t)m * nc + ijk];
            if (r > 0.0) r = r / vol();
            sum_eps = sum_eps + r / ro_s[m];
          }
          ep_g[ijk] = 1.0 - std::min(1.0, sum_eps);
        }
  }

  int step_coupled(int nn) {
    int rc = calc_force();
    if (rc) return rc;
    if (g.interp_scheme == DEM_INTERP_NONE) drag_des1(); else drag();   // CALC_DRAG_DES
    bool ok = true;
    const bool force = integrate_with_outflow(&ok);
    if (!ok) return fail(DEM_ERR_CAPACITY, "no NONEXISTENT slot left for an inflow particle (MAX_PIP)");
    bool do_nsearch = (nn == 1) || (nn % p.neighbor_search_n == 0) || force;
    bool anyper = p.periodic[0] || p.periodic[1] || (p.periodic[2] && !p.no_k);
    if (do_nsearch || anyper) desgrid_pic();
    if (do_nsearch) neighbour();
    comp_mean_fields();
    s_time = s_time + p.dtsolid;
    steps_done++;
    return 0;
  }

  // DES_TIME_STEP(NN) for pure DEM (des_time_march.f:342-432).
  // Outflow boundaries -----------------------------------------------
  bool in_bc_box(const dem_outflow_bc& b, int l) const {
    const int c = dg_pijk[l];
    if (c < 1) return false;
    const int ijk[3] = {iof(c), jof(c), kof(c)};
    for (int a = 0; a < 3; ++a)
      if (ijk[a] < b.dg_lo[a] || ijk[a] > b.dg_hi[a]) return false;
    return true;
  }
  static void bc_plane(int plane, double freeze[3], int& idx, double& sgn) {
    freeze[0] = freeze[1] = freeze[2] = 0.0;
    switch (plane) {
      case 'N': idx = 1; sgn = -1.0; break;
      case 'S': idx = 1; sgn = 1.0; break;
      case 'E': idx = 0; sgn = -1.0; break;
      case 'W': idx = 0; sgn = 1.0; break;
      case 'T': idx = 2; sgn = -1.0; break;
      default: idx = 2; sgn = 1.0; break;  // 'B'
    }
    freeze[idx] = 1.0;
  }

  // UPDATE_EXIT_DES_VEL (mass_outflow_dem.f:444-514): EXITING particles in the
  // cells of a non-MASS_OUTFLOW boundary keep integrating their force, with
  // the velocity frozen to the boundary-normal component.  The particle loop
  // of each boundary is a particle loop here (a particle is in one cell).
  void update_exit_vel() {
    const double dt = p.dtsolid;
    for (const dem_outflow_bc& b : obc) {
      if (b.mass_outflow) continue;
      double fz[3]; int idx; double sgn;
      bc_plane(b.plane, fz, idx, sgn);
      for (int l = 0; l < n; ++l) {
        if (state[l] != DEM_STATE_EXITING || !in_bc_box(b, l)) continue;
        for (int c = 0; c < 3; ++c) {
          double* v = X(vel, c); double* f = X(fc, c); double* a = X(acc_old, c);
          if (exit_first_pass && p.intg_method == DEM_INTG_AB2) a[l] = f[l] / pmass[l] + p.grav[c];
          if (p.intg_method == DEM_INTG_EULER) {
            v[l] = v[l] + dt * (f[l] / pmass[l] + p.grav[c]);
          } else {
            f[l] = f[l] / pmass[l] + p.grav[c];
            v[l] = X(vel_old, c)[l] + 0.5 * (3.0 * f[l] - a[l]) * dt;
            a[l] = f[l];
          }
          v[l] = v[l] * fz[c];
        }
      }
    }
    exit_first_pass = false;
  }

  // MASS_OUTFLOW_DEM (mass_outflow_dem.f:13-188); returns whether a particle
  // was deleted (FORCE_NSEARCH).
  bool mass_outflow() {
    bool force = false;
    for (const dem_outflow_bc& b : obc) {
      double fz[3]; int idx; double sgn;
      bc_plane(b.plane, fz, idx, sgn);
      for (int l = 0; l < n; ++l) {
        if (!in_bc_box(b, l)) continue;
        const int8_t st = state[l];
        if (st == DEM_STATE_NONEXISTENT || st >= DEM_STATE_NORMAL_GHOST || st == DEM_STATE_ENTERING) continue;
        const double x = P(pos, l, idx);
        const double dist = (b.plane == 'N' || b.plane == 'E' || b.plane == 'T') ? x - b.face : b.face - x;
        if (dist > rad[l]) {
          state[l] = DEM_STATE_NORMAL;
        } else if (dist > 0.0) {
          if (!b.mass_outflow) {
            if (P(vel, l, idx) * sgn > 0.0) {
              for (int c = 0; c < 3; ++c) X(vel, c)[l] = X(vel, c)[l] * fz[c];
              state[l] = DEM_STATE_EXITING;
            }
          } else {
            const int m = phase[l];
            for (int c = 0; c < 3; ++c) X(vel, c)[l] = b.vel[m][c];
            state[l] = DEM_STATE_EXITING;
          }
        } else {
          delete_particle(l);
          n_outflow_deleted++;
          force = true;
        }
      }
    }
    return force;
  }

  // Inflow boundaries ------------------------------------------------
  double next_rand() {
    if (!irand.empty()) { const double r = irand.front(); irand.pop_front(); return r; }
    // splitmix64, 53 bits in [0,1)
    uint64_t z = (irng += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * 0x1.0p-53;
  }

  // MASS_INFLOW_DEM (mass_inflow_dem.f:44-293) for plain spheres: per
  // boundary, the entering test over the DG_PIC lists of its cells
  // (82-140), RAND(3), the time window, then PI_COUNT particles from
  // SEED_NEW_PARTICLE (306-408) and SET_NEW_PARTICLE_PROPS (419-642) into
  // the first NONEXISTENT slots from LS = 1 on, and DEM_MI_TIME advanced.
  // Returns false when no NONEXISTENT slot is left.
  bool mass_inflow() {
    int ls = 0;
    for (Inflow& I : ibc) {
      dem_inflow_bc& b = I.bc;
      const int idx = (b.plane == 'N' || b.plane == 'S') ? 1 : ((b.plane == 'E' || b.plane == 'W') ? 0 : 2);
      for (int lk = b.dg_lo[2]; lk <= b.dg_hi[2]; ++lk)
        for (int li = b.dg_lo[0]; li <= b.dg_hi[0]; ++li)
          for (int lj = b.dg_lo[1]; lj <= b.dg_hi[1]; ++lj) {
            const int c = funijk(li, lj, lk) - 1;
            if (c < 0 || c >= ncell2 || cell_start.empty()) continue;
            for (int e = cell_start[c]; e < cell_start[c + 1]; ++e) {
              const int np = cell_list[e];
              if (state[np] == DEM_STATE_EXITING) continue;
              const double x = P(pos, np, idx);
              const double dist = (b.plane == 'N' || b.plane == 'E' || b.plane == 'T') ? x - b.face : b.face - x;
              if (dist > rad[np] && state[np] == DEM_STATE_ENTERING) state[np] = DEM_STATE_NORMAL;
            }
          }
      double rnd[3];
      for (double& r : rnd) r = next_rand();
      if (b.mi_time > s_time) continue;
      if (s_time < b.start_time || s_time > b.end_time) continue;
      for (int ip = 0; ip < b.pi_count; ++ip) {
        const int vac = b.vacancy;
        b.vacancy = vac % b.occupants + 1;
        int m1;
        if (b.polydisperse) {
          int ri = (int)std::ceil((double)b.n_layout * rnd[0]);
          ri = std::min(std::max(ri, 1), b.n_layout);
          m1 = I.layout[ri - 1];
        } else {
          m1 = I.layout[0];
        }
        const int m = m1 - 1;
        const double d = b.d_p0[m];
        const double rand1 = 0.5 * d + (b.window - d) * rnd[0];
        const double rand2 = 0.5 * d + (b.window - d) * rnd[1];
        double x[3];
        const double pv = I.p[vac - 1] + rand1, qv = I.q[vac - 1] + rand2;
        switch (b.plane) {
          case 'N': case 'S': x[0] = pv; x[2] = qv; x[1] = b.offset; break;
          case 'E': case 'W': x[1] = pv; x[2] = qv; x[0] = b.offset; break;
          default: x[0] = pv; x[1] = qv; x[2] = b.offset; break;
        }
        if (p.no_k) x[2] = 0.0;
        const int li = iofpos(x[0]), lj = jofpos(x[1]), lk = kofpos(x[2]);
        // one rank: DG_ISTART..DG_IEND span the ghost layers (desgrid_mod.f:756-761)
        bool owns = istart2 <= li && li <= iend2 && jstart2 <= lj && lj <= jend2;
        if (!p.no_k) owns = owns && kstart2 <= lk && lk <= kend2;
        if (!owns) continue;
        while (ls < n && state[ls] != DEM_STATE_NONEXISTENT) ++ls;
        if (ls >= n) return false;
        const int np = ls;
        state[np] = DEM_STATE_ENTERING;
        for (int c = 0; c < 3; ++c) {
          X(pos, c)[np] = x[c];
          X(vel, c)[np] = b.vel[m][c];
          X(omg, c)[np] = 0.0;
        }
        rad[np] = d * 0.5;
        const double pvol = (4.0 / 3.0) * M_PI * (rad[np] * rad[np] * rad[np]);
        pmass[np] = pvol * b.ro_s0[m];
        omoi[np] = 2.5 / (pmass[np] * (rad[np] * rad[np]));
        phase[np] = m;
        const int ci = std::min(iend2, std::max(istart2, li));
        const int cj = std::min(jend2, std::max(jstart2, lj));
        const int ck = p.no_k ? 1 : std::min(kend2, std::max(kstart2, lk));
        dg_pijk[np] = funijk(ci, cj, ck);
        n_inflow_added++;
      }
      b.mi_time = b.mi_time + b.pi_factor * p.dtsolid;
    }
    return true;
  }

  // The part of DES_TIME_STEP between the forces and the neighbour search
  // with flow boundaries: CFUPDATEOLD's DES_VEL_OLD, UPDATE_EXIT_DES_VEL,
  // CFNEWVALUES, MASS_INFLOW_DEM, MASS_OUTFLOW_DEM.  Returns FORCE_NSEARCH;
  // *ok turns false when an inflow particle found no slot.
  bool integrate_with_outflow(bool* ok = nullptr) {
    if (obc.empty()) {
      cfnewvalues();
      const bool seeded = ibc.empty() || mass_inflow();
      if (ok) *ok = seeded;
      return false;
    }
    vel_old = vel;
    update_exit_vel();
    cfnewvalues();
    vel_old.clear();
    const bool seeded = ibc.empty() || mass_inflow();
    if (ok) *ok = seeded;
    return mass_outflow();
  }

  int step(int nn) {
    int rc = calc_force();
    if (rc) return rc;
    bool ok = true;
    const bool force = integrate_with_outflow(&ok);
    if (!ok) return fail(DEM_ERR_CAPACITY, "no NONEXISTENT slot left for an inflow particle (MAX_PIP)");
    bool do_nsearch = (nn == 1) || (nn % p.neighbor_search_n == 0) || force;
    bool anyper = p.periodic[0] || p.periodic[1] || (p.periodic[2] && !p.no_k);
    if (do_nsearch || anyper) desgrid_pic();
    if (do_nsearch) neighbour();
    s_time = s_time + p.dtsolid;
    steps_done++;
    return 0;
  }
};

}  // namespace

struct orc_handle { Oracle o; };

extern "C" {

int orc_create(const dem_params* p, int32_t max_pip, orc_handle** out) {
  if (!p || !out || max_pip <= 0) return DEM_ERR_ARG;
  if (p->dg_imax < 1 || p->dg_jmax < 1 || (!p->no_k && p->dg_kmax < 1)) return DEM_ERR_ARG;
  if (p->n_phases < 1 || p->n_phases > DEM_MAX_PHASES) return DEM_ERR_ARG;
  auto* h = new orc_handle();
  Oracle& o = h->o;
  o.p = *p;
  o.n = max_pip;
  o.cmax = p->collision_array_max > 0 ? p->collision_array_max : 8;
  o.grid_init();
  size_t n3 = (size_t)3 * max_pip;
  o.pos.assign(n3, 0.0); o.vel.assign(n3, 0.0); o.omg.assign(n3, 0.0);
  o.fc.assign(n3, 0.0); o.tow.assign(n3, 0.0); o.acc_old.assign(n3, 0.0); o.rot_acc_old.assign(n3, 0.0);
  o.rad.assign(max_pip, 0.0); o.pmass.assign(max_pip, 0.0); o.omoi.assign(max_pip, 0.0);
  o.state.assign(max_pip, 0); o.phase.assign(max_pip, 0);
  o.dg_pijk.assign(max_pip, 0);
  o.row_end.assign(max_pip, 0);
  o.wall_fid.assign((size_t)o.cmax * max_pip, -1);
  o.wall_pft.assign((size_t)3 * o.cmax * max_pip, 0.0);
  o.fbin_start.assign(o.ncell2 + 1, 0);
  *out = h;
  return 0;
}

int orc_destroy(orc_handle* h) { delete h; return 0; }
const char* orc_last_error(const orc_handle* h) { return h ? h->o.err.c_str() : "null handle"; }
int orc_set_threads(orc_handle* h, int32_t nt) { h->o.nthreads = nt < 1 ? 1 : nt; return 0; }

// DTSOLID of the following steps (des_time_march.f:308-314, 470-476).
int orc_set_dtsolid(orc_handle* h, double dtsolid) {
  if (!(dtsolid > 0.0) || !std::isfinite(dtsolid)) return h->o.fail(DEM_ERR_ARG, "DTSOLID must be positive");
  h->o.p.dtsolid = dtsolid;
  return 0;
}

int orc_set_walls(orc_handle* h, const double* vertex, const double* norm_face, int32_t nf) {
  Oracle& o = h->o;
  if (nf < 0) return DEM_ERR_ARG;
  o.nf = nf;
  o.vertex.assign(vertex, vertex + (size_t)9 * nf);
  o.norm_face.assign(norm_face, norm_face + (size_t)3 * nf);
  o.bin_facets();
  return 0;
}

int orc_upload_state(orc_handle* h, const double* pos, const double* vel, const double* omega,
                     const double* radius, const double* pmass, const double* omoi,
                     const int8_t* state, const int32_t* phase, int32_t max_pip) {
  Oracle& o = h->o;
  if (max_pip != o.n) return o.fail(DEM_ERR_ARG, "max_pip mismatch");
  if (!pos || !vel || !omega) return o.fail(DEM_ERR_ARG, "null array");
  // after a first full upload, radius, pmass, omoi, state and phase may be
  // NULL: the handle keeps its own (as dem_upload_state)
  if ((!radius || !pmass || !omoi || !state || !phase) && !o.have_state)
    return o.fail(DEM_ERR_ARG, "the first upload needs every array");
  size_t n3 = (size_t)3 * o.n;
  std::copy(pos, pos + n3, o.pos.begin());
  std::copy(vel, vel + n3, o.vel.begin());
  std::copy(omega, omega + n3, o.omg.begin());
  if (radius) std::copy(radius, radius + o.n, o.rad.begin());
  if (pmass) std::copy(pmass, pmass + o.n, o.pmass.begin());
  if (omoi) std::copy(omoi, omoi + o.n, o.omoi.begin());
  if (state) std::copy(state, state + o.n, o.state.begin());
  if (phase) {
    for (int i = 0; i < o.n; ++i) {
      int ph = phase[i] - 1;
      if (o.state[i] != DEM_STATE_NONEXISTENT && (ph < 0 || ph >= o.p.n_phases))
        return o.fail(DEM_ERR_ARG, "phase out of range");
      o.phase[i] = ph < 0 ? 0 : ph;
    }
  }
  o.have_state = true;
  return 0;
}

int orc_download_state(orc_handle* h, double* pos, double* vel, double* omega, int8_t* state, int32_t max_pip) {
  Oracle& o = h->o;
  if (max_pip != o.n) return DEM_ERR_ARG;
  size_t n3 = (size_t)3 * o.n;
  if (pos) std::copy(o.pos.begin(), o.pos.begin() + n3, pos);
  if (vel) std::copy(o.vel.begin(), o.vel.begin() + n3, vel);
  if (omega) std::copy(o.omg.begin(), o.omg.begin() + n3, omega);
  if (state) std::copy(o.state.begin(), o.state.end(), state);
  return 0;
}

int orc_download_forces(orc_handle* h, double* fc, double* tow, int32_t max_pip) {
  Oracle& o = h->o;
  if (max_pip != o.n) return DEM_ERR_ARG;
  if (fc) std::copy(o.fc.begin(), o.fc.end(), fc);
  if (tow) std::copy(o.tow.begin(), o.tow.end(), tow);
  return 0;
}

int orc_set_ab2_history(orc_handle* h, const double* acc_old, const double* rot_acc_old,
                        int32_t first_pass, int32_t max_pip) {
  Oracle& o = h->o;
  if (max_pip != o.n) return DEM_ERR_ARG;
  if (acc_old) std::copy(acc_old, acc_old + (size_t)3 * o.n, o.acc_old.begin());
  if (rot_acc_old) std::copy(rot_acc_old, rot_acc_old + (size_t)3 * o.n, o.rot_acc_old.begin());
  o.first_pass = first_pass != 0;
  return 0;
}

int orc_get_ab2_history(orc_handle* h, double* acc_old, double* rot_acc_old, int32_t max_pip) {
  Oracle& o = h->o;
  if (max_pip != o.n) return DEM_ERR_ARG;
  if (acc_old) std::copy(o.acc_old.begin(), o.acc_old.end(), acc_old);
  if (rot_acc_old) std::copy(o.rot_acc_old.begin(), o.rot_acc_old.end(), rot_acc_old);
  return 0;
}

int orc_pair_count(orc_handle* h, int64_t* np) { *np = (int64_t)h->o.nbrs.size(); return 0; }

int orc_download_pairs(orc_handle* h, int32_t* ni, int32_t* nb, double* pf, int64_t cap, int32_t max_pip) {
  Oracle& o = h->o;
  if (max_pip != o.n) return DEM_ERR_ARG;
  if ((nb || pf) && cap < (int64_t)o.nbrs.size()) return o.fail(DEM_ERR_CAPACITY, "pair capacity too small");
  if (ni) for (int i = 0; i < o.n; ++i) ni[i] = o.row_end[i] + 1;
  if (nb) for (size_t c = 0; c < o.nbrs.size(); ++c) nb[c] = o.nbrs[c] + 1;
  if (pf) std::copy(o.pft.begin(), o.pft.end(), pf);
  return 0;
}

int orc_upload_pairs(orc_handle* h, const int32_t* ni, const int32_t* nb, const double* pf,
                     int64_t np, int32_t max_pip) {
  Oracle& o = h->o;
  if (max_pip != o.n) return DEM_ERR_ARG;
  o.row_end.resize(o.n);
  for (int i = 0; i < o.n; ++i) o.row_end[i] = ni[i] - 1;
  o.nbrs.resize(np);
  for (int64_t c = 0; c < np; ++c) o.nbrs[c] = nb[c] - 1;
  o.pft.assign(pf, pf + 3 * np);
  return 0;
}

int orc_download_wall_history(orc_handle* h, int32_t* fid, double* pf, int32_t max_pip) {
  Oracle& o = h->o;
  if (max_pip != o.n) return DEM_ERR_ARG;
  if (fid) for (size_t s = 0; s < o.wall_fid.size(); ++s) fid[s] = o.wall_fid[s] < 0 ? -1 : o.wall_fid[s] + 1;
  if (pf) std::copy(o.wall_pft.begin(), o.wall_pft.end(), pf);
  return 0;
}

int orc_upload_wall_history(orc_handle* h, const int32_t* fid, const double* pf, int32_t max_pip) {
  Oracle& o = h->o;
  if (max_pip != o.n || !fid || !pf) return o.fail(DEM_ERR_ARG, "bad wall history arrays");
  for (size_t s = 0; s < o.wall_fid.size(); ++s)
    if (fid[s] != -1 && (fid[s] < 1 || fid[s] > o.nf)) return o.fail(DEM_ERR_ARG, "facet id out of range");
  for (size_t s = 0; s < o.wall_fid.size(); ++s) o.wall_fid[s] = fid[s] < 0 ? -1 : fid[s] - 1;
  std::copy(pf, pf + o.wall_pft.size(), o.wall_pft.begin());
  return 0;
}

int orc_set_outflow_bcs(orc_handle* h, const dem_outflow_bc* bcs, int32_t n) {
  Oracle& o = h->o;
  if (n < 0 || (n > 0 && !bcs)) return o.fail(DEM_ERR_ARG, "bad outflow boundaries");
  for (int32_t b = 0; b < n; ++b) {
    const int pl = bcs[b].plane;
    if (pl != 'N' && pl != 'S' && pl != 'E' && pl != 'W' && pl != 'T' && pl != 'B')
      return o.fail(DEM_ERR_ARG, "unknown BC_PLANE");
    for (int a = 0; a < 3; ++a)
      if (bcs[b].dg_lo[a] > bcs[b].dg_hi[a]) return o.fail(DEM_ERR_ARG, "empty DES-cell box");
    for (int c = 0; c < b; ++c) {
      bool overlap = true;
      for (int a = 0; a < 3; ++a)
        overlap = overlap && bcs[b].dg_lo[a] <= bcs[c].dg_hi[a] && bcs[c].dg_lo[a] <= bcs[b].dg_hi[a];
      if (overlap) return o.fail(DEM_ERR_ARG, "outflow boundary boxes overlap");
    }
  }
  o.obc.assign(bcs, bcs + n);
  o.exit_first_pass = true;
  return 0;
}

int orc_set_inflow_bcs(orc_handle* h, const dem_inflow_bc* bcs, int32_t n, uint64_t seed) {
  Oracle& o = h->o;
  if (n < 0 || (n > 0 && !bcs)) return o.fail(DEM_ERR_ARG, "bad inflow boundaries");
  for (int32_t i = 0; i < n; ++i) {
    const dem_inflow_bc& b = bcs[i];
    const int pl = b.plane;
    if (pl != 'N' && pl != 'S' && pl != 'E' && pl != 'W' && pl != 'T' && pl != 'B')
      return o.fail(DEM_ERR_ARG, "unknown BC_PLANE");
    if (b.pi_count < 0 || (b.pi_count > 0 && (b.occupants < 1 || !b.p || !b.q)))
      return o.fail(DEM_ERR_ARG, "inflow layout missing");
    if (b.vacancy < 1 || (b.occupants > 0 && b.vacancy > b.occupants))
      return o.fail(DEM_ERR_ARG, "inflow vacancy out of range");
    if (b.n_layout < 1 || !b.poly_layout) return o.fail(DEM_ERR_ARG, "inflow phase layout missing");
    for (int32_t j = 0; j < b.n_layout; ++j)
      if (b.poly_layout[j] < 1 || b.poly_layout[j] > o.p.n_phases) return o.fail(DEM_ERR_ARG, "inflow phase out of range");
    for (int a = 0; a < 3; ++a)
      if (b.dg_lo[a] > b.dg_hi[a]) return o.fail(DEM_ERR_ARG, "empty DES-cell box");
    if (!(b.pi_factor > 0.0) && b.pi_count > 0) return o.fail(DEM_ERR_ARG, "PI_FACTOR must be positive");
  }
  o.ibc.clear();
  o.irand.clear();
  o.irng = seed;
  for (int32_t i = 0; i < n; ++i) {
    Oracle::Inflow I;
    I.bc = bcs[i];
    const int occ = bcs[i].pi_count > 0 ? bcs[i].occupants : 0;
    I.p.assign(bcs[i].p, bcs[i].p + occ);
    I.q.assign(bcs[i].q, bcs[i].q + occ);
    I.layout.assign(bcs[i].poly_layout, bcs[i].poly_layout + bcs[i].n_layout);
    I.bc.p = nullptr; I.bc.q = nullptr; I.bc.poly_layout = nullptr; I.bc.w_cell = nullptr; I.bc.h_cell = nullptr;
    o.ibc.push_back(std::move(I));
  }
  return 0;
}

int orc_push_inflow_random(orc_handle* h, const double* r, int64_t n) {
  Oracle& o = h->o;
  if (n < 0 || (n > 0 && !r)) return o.fail(DEM_ERR_ARG, "bad random numbers");
  o.irand.insert(o.irand.end(), r, r + n);
  return 0;
}

int orc_get_inflow_state(orc_handle* h, int32_t bc, int32_t* vacancy, double* mi_time) {
  Oracle& o = h->o;
  if (bc < 0 || bc >= (int32_t)o.ibc.size()) return o.fail(DEM_ERR_ARG, "no such inflow boundary");
  if (vacancy) *vacancy = o.ibc[bc].bc.vacancy;
  if (mi_time) *mi_time = o.ibc[bc].bc.mi_time;
  return 0;
}

int orc_download_cells(orc_handle* h, int32_t* cells, int32_t max_pip) {
  Oracle& o = h->o;
  if (max_pip != o.n) return DEM_ERR_ARG;
  std::copy(o.dg_pijk.begin(), o.dg_pijk.end(), cells);
  return 0;
}

int orc_download_facet_bins(orc_handle* h, int32_t* start, int32_t* ids, int32_t cap, int32_t* nc) {
  Oracle& o = h->o;
  *nc = o.ncell2;
  if (start) for (int c = 0; c <= o.ncell2; ++c) start[c] = o.fbin_start[c];
  if (ids) {
    if (cap < (int32_t)o.fbin.size()) return DEM_ERR_CAPACITY;
    for (size_t q = 0; q < o.fbin.size(); ++q) ids[q] = o.fbin[q].id + 1;
  }
  return 0;
}

int orc_download_edge_flags(orc_handle* h, int8_t* flags) {
  std::copy(h->o.ignore_edge.begin(), h->o.ignore_edge.end(), flags);
  return 0;
}

int orc_desgrid_pic(orc_handle* h) { h->o.desgrid_pic(); return 0; }
int orc_neighbour(orc_handle* h) { h->o.neighbour(); return 0; }
int orc_calc_force(orc_handle* h) { return h->o.calc_force(); }
int orc_cfnewvalues(orc_handle* h) { h->o.cfnewvalues(); return 0; }
int orc_init_neighbors(orc_handle* h) {
  if (!h->o.have_state) return DEM_ERR_STATE;
  h->o.desgrid_pic();
  h->o.row_end.assign(h->o.n, 0); h->o.nbrs.clear(); h->o.pft.clear();
  h->o.neighbour();
  return 0;
}
int orc_step(orc_handle* h, int32_t nn_first, int32_t nsteps) {
  for (int32_t k = 0; k < nsteps; ++k) {
    int rc = h->o.step(nn_first + k);
    if (rc) return rc;
  }
  return 0;
}

int orc_get_stats(orc_handle* h, dem_stats* s) {
  Oracle& o = h->o;
  std::memset(s, 0, sizeof *s);
  double mv[3] = {0, 0, 0}, msum = 0, ysum = 0, ke = 0;
  int64_t nn = 0;
  for (int i = 0; i < o.n; ++i) {
    if (o.state[i] != DEM_STATE_NORMAL) continue;
    nn++;
    for (int c = 0; c < 3; ++c) mv[c] += o.P(o.vel, i, c);
    msum += o.pmass[i]; ysum += o.pmass[i] * o.P(o.pos, i, 1);
    double v2 = 0; for (int c = 0; c < 3; ++c) v2 += o.P(o.vel, i, c) * o.P(o.vel, i, c);
    ke += 0.5 * o.pmass[i] * v2;
  }
  for (int c = 0; c < 3; ++c) mv[c] = nn ? mv[c] / nn : 0.0;
  double gt[3] = {0, 0, 0};
  for (int i = 0; i < o.n; ++i) {
    if (o.state[i] != DEM_STATE_NORMAL) continue;
    for (int c = 0; c < 3; ++c) { double d = o.P(o.vel, i, c) - mv[c]; gt[c] += d * d; }
  }
  for (int c = 0; c < 3; ++c) { s->mean_vel[c] = mv[c]; s->gran_temp[c] = nn ? gt[c] / nn : 0.0; }
  s->n_normal = nn;
  s->n_outflow_removed = o.n_outflow_deleted;
  s->n_inflow_added = o.n_inflow_added;
  s->n_pairs = (int64_t)o.nbrs.size();
  s->n_contacts = o.n_contacts;
  s->n_wall_contacts = o.n_wall_contacts;
  s->n_rogue_removed = o.rogue_removed;
  s->steps_done = o.steps_done;
  s->kinetic_energy = ke;
  s->bed_height = msum > 0 ? ysum / msum : 0.0;
  s->s_time = o.s_time;
  return 0;
}

// Coupling.
int orc_set_gas_fields(orc_handle* h, const dem_fluid_grid* g, const double* ep_g,
                       const double* u_g, const double* v_g, const double* w_g,
                       const double* p_force) {
  Oracle& o = h->o;
  if (!g || !ep_g || !u_g || !v_g || !w_g) return o.fail(DEM_ERR_ARG, "null gas field");
  if (!o.have_state) return o.fail(DEM_ERR_STATE, "upload particles first");
  if (g->interp_scheme != DEM_INTERP_GARG && g->interp_scheme != DEM_INTERP_NONE)
    return o.fail(DEM_ERR_ARG, "unknown interp_scheme");
  if (g->drag_model != DEM_DRAG_GIDASPOW && g->drag_model != DEM_DRAG_SINGLE_SPHERE)
    return o.fail(DEM_ERR_ARG, "unknown drag_model");
  if (g->drag_model == DEM_DRAG_SINGLE_SPHERE && !(g->usr_d_p0 > 0.0))
    return o.fail(DEM_ERR_ARG, "usr_d_p0 must be positive for the single-sphere drag");
  o.g = *g;
  o.gas_setup();
  size_t nc = o.vol_surr.size();
  o.ep_g.assign(ep_g, ep_g + nc);
  o.u_g.assign(u_g, u_g + nc);
  o.v_g.assign(v_g, v_g + nc);
  o.w_g.assign(w_g, w_g + nc);
  if (p_force) o.p_force.assign(p_force, p_force + 3 * nc); else o.p_force.clear();
  for (int m = 0; m < o.p.n_phases; ++m) {
    if (!(g->ro_s[m] > 0.0)) return o.fail(DEM_ERR_ARG, "ro_s must be positive");
    o.ro_s[m] = g->ro_s[m];
  }
  o.have_gas = true;
  o.particles_in_cell();
  return 0;
}
int orc_get_mean_fields(orc_handle* h, double* ep_g, double* rop_s) {
  Oracle& o = h->o;
  if (!o.have_gas) return o.fail(DEM_ERR_STATE, "no gas fields");
  if (ep_g) std::copy(o.ep_g.begin(), o.ep_g.end(), ep_g);
  if (rop_s) {
    if (o.rop_s.empty()) std::fill(rop_s, rop_s + o.vol_surr.size(), 0.0);
    else std::copy(o.rop_s.begin(), o.rop_s.begin() + o.vol_surr.size(), rop_s);
  }
  return 0;
}
// CALC_DES_BEDHEIGHT (des_granular_temperature.f:201-267): the serial loop
// over IJKSTART3..IJKEND3 with EP_S = ROP_S/RO_S and the cell-centre height.
int orc_calc_des_bedheight(orc_handle* h, double* bed_height) {
  Oracle& o = h->o;
  if (!o.have_gas) return o.fail(DEM_ERR_STATE, "no gas fields");
  if (!bed_height) return o.fail(DEM_ERR_ARG, "null output");
  const int M = o.p.n_phases;
  const size_t nc = o.vol_surr.size();
  std::vector<double> num(M, 0.0), den(M, 0.0);
  if (!o.rop_s.empty()) {
    for (size_t ijk = 0; ijk < nc; ++ijk) {
      const int j = (int)((ijk / (size_t)o.gi2) % (size_t)o.gj2) + 1;
      for (int m = 0; m < M; ++m) {
        const double r = o.rop_s[(size_t)m * nc + ijk];
        if (r > 0.0) {
          const double hcell = 0.5 * (o.yn[j] + o.yn[j - 1]);
          const double ep = r / o.ro_s[m];
          num[m] = num[m] + ep * hcell * o.vol();
          den[m] = den[m] + ep * o.vol();
        }
      }
    }
  }
  int pip = 0;
  for (int l = 0; l < o.n; ++l) pip += o.state[l] != DEM_STATE_NONEXISTENT;
  for (int m = 0; m < M; ++m) bed_height[m] = pip > 0 ? num[m] / den[m] : 0.0;
  return 0;
}
int orc_comp_mean_fields(orc_handle* h) {
  if (!h->o.have_gas) return h->o.fail(DEM_ERR_STATE, "no gas fields");
  h->o.comp_mean_fields();
  return 0;
}
int orc_drag_gs_des0(orc_handle* h) {
  if (!h->o.have_gas) return h->o.fail(DEM_ERR_STATE, "no gas fields");
  h->o.drag();
  return 0;
}
int orc_drag_gs_gas0(orc_handle* h, double* f_gds, double* drag_am, double* drag_bm, double* f_gp) {
  Oracle& o = h->o;
  if (!o.have_gas) return o.fail(DEM_ERR_STATE, "no gas fields");
  o.drag_gas();
  if (f_gds) std::copy(o.f_gds.begin(), o.f_gds.end(), f_gds);
  if (drag_am) std::copy(o.drag_am.begin(), o.drag_am.end(), drag_am);
  if (drag_bm) std::copy(o.drag_bm.begin(), o.drag_bm.end(), drag_bm);
  if (f_gp) std::copy(o.f_gp.begin(), o.f_gp.end(), f_gp);
  return 0;
}
int orc_drag_gs_des1(orc_handle* h) {
  if (!h->o.have_gas) return h->o.fail(DEM_ERR_STATE, "no gas fields");
  h->o.drag_des1();
  return 0;
}
int orc_drag_gs_gas1(orc_handle* h, double* f_gds, double* drag_bm, double* f_gp) {
  Oracle& o = h->o;
  if (!o.have_gas) return o.fail(DEM_ERR_STATE, "no gas fields");
  o.drag_gas1();
  if (f_gds) std::copy(o.f_gds.begin(), o.f_gds.end(), f_gds);
  if (drag_bm) std::copy(o.drag_bm.begin(), o.drag_bm.end(), drag_bm);
  if (f_gp) std::copy(o.f_gp.begin(), o.f_gp.end(), f_gp);
  return 0;
}
int orc_step_coupled(orc_handle* h, int32_t nn_first, int32_t nsteps) {
  if (!h->o.have_gas) return h->o.fail(DEM_ERR_STATE, "no gas fields");
  for (int32_t k = 0; k < nsteps; ++k) {
    int rc = h->o.step_coupled(nn_first + k);
    if (rc) return rc;
  }
  return 0;
}

// CHECK_SOLIDS_DEM_COLL_LSD (check_solids_dem.f:519-782) and
// CHECK_SOLIDS_DEM_COLL_HERTZ (798-1122), DEM phases only (MMAX = 0).
int orc_contact_constants(dem_params* p, const double* ref_radius, const double* ref_mass,
                          const double* e_young, const double* v_poisson,
                          const double* en_in, const double* et_in,
                          const double* en_w_in, const double* et_w_in,
                          double ew_young, double vw_poisson,
                          double kt_fac, double kt_w_fac,
                          double des_etat_fac, double des_etat_w_fac,
                          double dtsolid_factor, double* tcoll_out) {
  const int M = p->n_phases, S = DEM_MAX_PHASES;
  const double PI = 4.0 * std::atan(1.0);
  double tcoll = UNDEFINED;
  if (p->coll_model == DEM_COLL_LSD) {
    p->kt = kt_fac * p->kn;
    p->kt_w = kt_w_fac * p->kn_w;
    for (int m = 0; m < M; ++m) {
      double mass_m = ref_mass[m];
      for (int l = m; l < M; ++l) {
        double en = en_in[m * S + l];
        double mass_l = ref_mass[l];
        double mass_eff = mass_m * mass_l / (mass_m + mass_l);
        double etan;
        if (en != 0.0) {
          etan = 2.0 * std::sqrt(p->kn * mass_eff) * std::fabs(std::log(en));
          etan = etan / std::sqrt(PI * PI + (std::log(en) * std::log(en)));
        } else {
          etan = 2.0 * std::sqrt(p->kn * mass_eff);
        }
        double tc;
        if (en != 0.0) tc = PI / std::sqrt(p->kn / mass_eff - ((etan / mass_eff) * (etan / mass_eff)) / 4.0);
        else tc = PI / std::sqrt(p->kn / mass_eff);
        tcoll = std::min(tc, tcoll);
        etan = etan / std::sqrt(mass_eff);
        p->des_etan[m * S + l] = etan; p->des_etat[m * S + l] = des_etat_fac * etan;
        p->des_etan[l * S + m] = p->des_etan[m * S + l]; p->des_etat[l * S + m] = p->des_etat[m * S + l];
      }
      double en = en_w_in[m];
      double mass_eff = mass_m;
      double etan;
      if (en != 0.0) {
        etan = 2.0 * std::sqrt(p->kn_w * mass_eff) * std::fabs(std::log(en));
        etan = etan / std::sqrt(PI * PI + (std::log(en) * std::log(en)));
      } else {
        etan = 2.0 * std::sqrt(p->kn_w * mass_eff);
      }
      etan = etan / std::sqrt(mass_eff);
      p->des_etan_wall[m] = etan;
      p->des_etat_wall[m] = des_etat_w_fac * etan;
    }
  } else {
    double g_wall = 0.5 * ew_young / (1.0 + vw_poisson);
    double gm[DEM_MAX_PHASES];
    for (int m = 0; m < M; ++m) gm[m] = 0.5 * e_young[m] / (1.0 + v_poisson[m]);
    for (int m = 0; m < M; ++m) {
      double mass_m = ref_mass[m];
      for (int l = m; l < M; ++l) {
        double en = en_in[m * S + l], et = et_in[m * S + l];
        double mass_l = ref_mass[l];
        double mass_eff = (mass_m * mass_l) / (mass_m + mass_l);
        double red = (2.0 / 7.0) * mass_eff;
        double r_eff = ref_radius[m] * ref_radius[l] / (ref_radius[m] + ref_radius[l]);
        double e_eff = e_young[m] * e_young[l] /
            (e_young[m] * (1.0 - v_poisson[l] * v_poisson[l]) + e_young[l] * (1.0 - v_poisson[m] * v_poisson[m]));
        double g_eff = gm[m] * gm[l] / (gm[m] * (2.0 - v_poisson[l]) + gm[l] * (2.0 - v_poisson[m]));
        double hkn = (4.0 / 3.0) * std::sqrt(r_eff) * e_eff;
        double hkt = 8.0 * std::sqrt(r_eff) * g_eff;
        double etan, etat;
        if (en != 0.0) {
          etan = std::sqrt(5.0) * std::sqrt(hkn * mass_eff) * std::fabs(std::log(en));
          etan = etan / std::sqrt(PI * PI + (std::log(en) * std::log(en)));
        } else etan = std::sqrt(5.0) * std::sqrt(hkn * mass_eff);
        if (et != 0.0) {
          etat = std::sqrt(5.0) * std::sqrt(hkt * red) * std::fabs(std::log(et));
          etat = etat / std::sqrt(PI * PI + (std::log(et) * std::log(et)));
        } else etat = std::sqrt(5.0) * std::sqrt(hkt * red);
        double tc;
        if (en != 0.0) tc = PI / std::sqrt(hkn / mass_eff - ((etan / mass_eff) * (etan / mass_eff)) / 5.0);
        else tc = PI / std::sqrt(hkn / mass_eff);
        tcoll = std::min(tc, tcoll);
        etan = etan / std::sqrt(hkn * mass_eff);
        etat = etat / std::sqrt(hkt * mass_eff);
        hkn = hkn / std::sqrt(r_eff);
        hkt = hkt / std::sqrt(r_eff);
        p->hert_kn[m * S + l] = p->hert_kn[l * S + m] = hkn;
        p->hert_kt[m * S + l] = p->hert_kt[l * S + m] = hkt;
        p->des_etan[m * S + l] = p->des_etan[l * S + m] = etan;
        p->des_etat[m * S + l] = p->des_etat[l * S + m] = etat;
      }
      double en = en_w_in[m], et = et_w_in[m];
      double mass_eff = mass_m, red = (2.0 / 7.0) * mass_eff;
      double r_eff = ref_radius[m];
      double e_eff = e_young[m] * ew_young /
          (e_young[m] * (1.0 - vw_poisson * vw_poisson) + ew_young * (1.0 - v_poisson[m] * v_poisson[m]));
      double g_eff = gm[m] * g_wall / (gm[m] * (2.0 - vw_poisson) + g_wall * (2.0 - v_poisson[m]));
      double hkwn = (4.0 / 3.0) * std::sqrt(r_eff) * e_eff;
      double hkwt = (double)8.0f * std::sqrt(r_eff) * g_eff;
      double etan, etat;
      if (en != 0.0) {
        etan = std::sqrt(5.0) * std::sqrt(hkwn * mass_eff) * std::fabs(std::log(en));
        etan = etan / std::sqrt(PI * PI + (std::log(en) * std::log(en)));
      } else etan = std::sqrt(5.0) * std::sqrt(hkwn * mass_eff);
      if (et != 0.0) {
        etat = std::sqrt(5.0) * std::sqrt(hkwt * red) * std::fabs(std::log(et));
        etat = etat / std::sqrt(PI * PI + (std::log(et) * std::log(et)));
      } else etat = std::sqrt(5.0) * std::sqrt(hkwt * red);
      p->des_etan_wall[m] = etan / std::sqrt(hkwn * mass_eff);
      p->des_etat_wall[m] = etat / std::sqrt(hkwt * mass_eff);
      p->hert_kwn[m] = hkwn / std::sqrt(r_eff);
      p->hert_kwt[m] = hkwt / std::sqrt(r_eff);
    }
  }
  if (tcoll_out) *tcoll_out = tcoll;
  p->dtsolid = tcoll / dtsolid_factor;
  return 0;
}

}  // extern "C"
