// force.cu -- contact forces and integration, FP64 (K3, K4, K5).
//
// Replaces CALC_FORCE_DEM (model/des/calc_force_dem.f:18-544) with CFRELVEL
// (model/des/cfrelvel.f:54-77), the wall contacts of
// CALC_DEM_FORCE_WITH_WALL_STL (model/des/calc_collision_wall_mod.f:180-629,
// GET/UPDATE/REMOVE_COLLISION 651-792, CFRELVEL_WALL 806-847,
// ClosestPtPointTriangle in stl_functions_des_mod.f:25-160), and
// CFUPDATEOLD + CFNEWVALUES (cfupdateold.f:33-41, cfnewvalues.f:669-812).
//
// The reference loops over owners LL and scatters each pair's force into
// FC(LL) and FC(I).  Here each pair is evaluated once (k_pairs, a thread per
// pair), which updates its tangential history in place and writes the
// terms of both particles into a contact record; then one thread per
// particle gathers (k_gather): walls first, then the records of the pairs
// it appears in as neighbour I owned by lower-index particles (ascending
// owner, from the transpose), its own row, then the remaining incoming
// pairs.  That is exactly the order in which the serial reference adds into
// FC(me)/TOW(me), so every particle's force is bit-identical to the serial
// reference without atomics.
//
// This file is compiled with -fmad=false: every FP64 expression rounds as
// the Fortran does (gfortran emits no FMA without -march).  sqrt and '/' are
// IEEE round-to-nearest in CUDA, as they are on the host.
#include "dem_internal.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace demb {

struct PState {  // one particle's gathered state
  double x[3], v[3], w[3];
  double r, m;
  int ph;
};

__device__ __forceinline__ void load_p(const double4* __restrict__ pos4, const double4* __restrict__ vel4,
                                       const double4* __restrict__ omg4, const uint8_t* __restrict__ phase,
                                       int i, PState& s) {
  double4 a = pos4[i], b = vel4[i], c = omg4[i];
  s.x[0] = a.x; s.x[1] = a.y; s.x[2] = a.z; s.r = a.w;
  s.v[0] = b.x; s.v[1] = b.y; s.v[2] = b.z; s.m = b.w;
  s.w[0] = c.x; s.w[1] = c.y; s.w[2] = c.z;
  s.ph = phase[i];
}

// Contact part of one CC iteration of CALC_FORCE_DEM (calc_force_dem.f:
// 273-363) with CFRELVEL (cfrelvel.f:54-77) for owner L and neighbour I in
// contact; dist = x_I - x_L and d2 = |dist|^2 come from the apart test.
template <int COLL>
__device__ __forceinline__ void contact_force(const DevParams& p, const PState& L, const PState& I,
                                              const double dist[3], double d2, const double pin[3],
                                              double pout[3], PairRec& o) {
  const double rl = L.r, ri = I.r;
  const double r_lm = rl + ri;
  const double dmag = sqrt(d2);
  double nrm[3] = {dist[0] / dmag, dist[1] / dmag, dist[2] / dmag};
  const double overlap_n = r_lm - dmag;
  // CFRELVEL
  double vrel[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) vrel[c] = L.v[c] - I.v[c];
  const double dcl = (dmag * dmag + rl * rl - ri * ri) / (2.0 * dmag);
  const double dci = dmag - dcl;
  double osum[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) osum[c] = L.w[c] * dcl + I.w[c] * dci;
  double vrot[3];
  cross3(osum, nrm, vrot);
#pragma unroll
  for (int c = 0; c < 3; ++c) vrel[c] = vrel[c] + vrot[c];
  const double vrn = dot3(vrel, nrm);
  double vt[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) vt[c] = vrel[c] - vrn * nrm[c];
  const int ix = L.ph * MAXP + I.ph;
  const double rad_eff = (rl * ri) / (rl + ri);
  const double m_eff = (L.m * I.m) / (L.m + I.m);
  double kn, kt, etan, etat;
  if (COLL == DEM_COLL_HERTZ) {
    double so = sqrt(overlap_n);
    kn = p.hkn[ix] * so * sqrt(rad_eff);
    kt = p.hkt[ix] * so * sqrt(rad_eff);
    so = sqrt(so);
    etan = p.etan[ix] * so * sqrt(p.hkn[ix] * sqrt(rad_eff) * m_eff);
    etat = p.etat[ix] * so * sqrt(p.hkt[ix] * sqrt(rad_eff) * m_eff);
  } else {
    kn = p.kn; kt = p.kt;
    etan = p.etan[ix] * sqrt(m_eff);
    etat = p.etat[ix] * sqrt(m_eff);
  }
  double fn[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) fn[c] = -(kn * overlap_n * nrm[c] + etan * vrn * nrm[c]);
  double ot[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) ot[c] = p.dt * vt[c] + pin[c];
  const double mag = sqrt(dot3(ot, ot));
  double ft[3];
  if (mag > 0.0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) ft[c] = -kt * ot[c] - etat * vt[c];
    const double ftmd = sqrt(dot3(ft, ft));
    const double fnmd = p.mew * sqrt(dot3(fn, fn));
    if (ftmd > fnmd) {
      double tg[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) tg[c] = ot[c] / mag;
#pragma unroll
      for (int c = 0; c < 3; ++c) ft[c] = -fnmd * tg[c];
#pragma unroll
      for (int c = 0; c < 3; ++c) ot[c] = (fnmd / kt) * tg[c];
    }
  } else {
    ft[0] = ft[1] = ft[2] = 0.0;
  }
  pout[0] = ot[0]; pout[1] = ot[1]; pout[2] = ot[2];
  o.dcl2 = dmag / 2.0 + (rl * rl - ri * ri) / (2.0 * dmag);
  o.dci2 = dmag - o.dcl2;
  cross3(nrm, ft, o.tf);
#pragma unroll
  for (int c = 0; c < 3; ++c) o.fc[c] = 0.0 + fn[c] + ft[c];
  o.kn = kn;
  o.ov = overlap_n;
}

// ---------------------------------------------------------------------------
// Walls

struct WallCtx {
  const double* __restrict__ vertex;   // [f][v][c]
  const double* __restrict__ norm_face;// [f][c]
  const int8_t* __restrict__ ignore_edge; // [f][4]
  const int* __restrict__ fbin_start;
  const FacetBinEntry* __restrict__ fbin;
  const int* __restrict__ dg_pijk;
  int* __restrict__ wall_fid;          // [i][cmax]
  double* __restrict__ wall_pft;       // [i][cmax][3]
  int nf;
};

__device__ __forceinline__ void closest_pt(const DevParams& p, const WallCtx& w, int f, const double pp[3],
                                           double cpt[3], bool& poe, int& edge) {
  poe = false; edge = 0;
  const double* V = w.vertex + 9 * (size_t)f;
  double a[3], b[3], c[3], ab[3], ac[3], ap[3], bp[3], cp[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) { a[k] = V[k]; b[k] = V[3 + k]; c[k] = V[6 + k]; }
#pragma unroll
  for (int k = 0; k < 3; ++k) { ab[k] = b[k] - a[k]; ac[k] = c[k] - a[k]; ap[k] = pp[k] - a[k]; }
  const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  const int8_t* ig = w.ignore_edge + 4 * (size_t)f;
  if (d1 < 0.0 && d2 < 0.0) {
    for (int k = 0; k < 3; ++k) cpt[k] = a[k];
    poe = true; if (ig[1]) cpt[0] = UNDEFINED_D; edge = 1; return;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) bp[k] = pp[k] - b[k];
  const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 > 0.0 && d4 < d3) {
    for (int k = 0; k < 3; ++k) cpt[k] = b[k];
    poe = true; if (ig[1]) cpt[0] = UNDEFINED_D; edge = 1; return;
  }
  const double vc = d1 * d4 - d3 * d2;
  if (vc < 0.0 && d1 > 0.0 && d3 < 0.0) {
    const double v = d1 / (d1 - d3);
    for (int k = 0; k < 3; ++k) cpt[k] = a[k] + v * ab[k];
    poe = true; if (ig[1]) cpt[0] = UNDEFINED_D; edge = 1; return;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) cp[k] = pp[k] - c[k];
  const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 > 0.0 && d5 < d6) {
    for (int k = 0; k < 3; ++k) cpt[k] = c[k];
    poe = true; if (ig[2]) cpt[0] = UNDEFINED_D; edge = 2; return;
  }
  const double vb = d5 * d2 - d1 * d6;
  if (vb < 0.0 && d2 > 0.0 && d6 < 0.0) {
    const double ww = d2 / (d2 - d6);
    for (int k = 0; k < 3; ++k) cpt[k] = a[k] + ww * ac[k];
    poe = true; if (ig[2]) cpt[0] = UNDEFINED_D; edge = 2; return;
  }
  const double va = d3 * d6 - d5 * d4;
  if (va < 0.0 && (d4 - d3) > 0.0 && (d5 - d6) > 0.0) {
    const double ww = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    for (int k = 0; k < 3; ++k) cpt[k] = b[k] + ww * (c[k] - b[k]);
    poe = true; if (ig[3]) cpt[0] = UNDEFINED_D; edge = 3; return;
  }
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom, ww = vc * denom;
  for (int k = 0; k < 3; ++k) cpt[k] = a[k] + ab[k] * v + ac[k] * ww;
  if (p.no_k) cpt[2] = pp[2];
}

__device__ __forceinline__ void remove_collision(const DevParams& p, const WallCtx& w, int me, int f) {
  int* fid = w.wall_fid + (size_t)me * p.cmax;
  for (int s = 0; s < p.cmax; ++s) if (fid[s] == f) { fid[s] = -1; return; }
}

// returns slot index, or -1 on overflow
__device__ __forceinline__ int get_collision(const DevParams& p, const WallCtx& w, int me, int f, int cell,
                                             double out[3]) {
  int* fid = w.wall_fid + (size_t)me * p.cmax;
  double* wp = w.wall_pft + (size_t)me * p.cmax * 3;
  int free_index = -1;
  for (int s = 0; s < p.cmax; ++s) {
    int v = fid[s];
    if (f == v) { out[0] = wp[3 * s]; out[1] = wp[3 * s + 1]; out[2] = wp[3 * s + 2]; return s; }
    else if (v == -1) free_index = s;
  }
  if (free_index == -1) {
    for (int s = 0; s < p.cmax && free_index == -1; ++s) {
      bool in_cell = false;
      for (int q = w.fbin_start[cell]; q < w.fbin_start[cell + 1]; ++q)
        if (fid[s] == w.fbin[q].id) { in_cell = true; break; }
      if (!in_cell) free_index = s;
    }
  }
  if (free_index == -1) return -1;
  fid[free_index] = f;
  wp[3 * free_index] = 0.0; wp[3 * free_index + 1] = 0.0; wp[3 * free_index + 2] = 0.0;
  out[0] = out[1] = out[2] = 0.0;
  return free_index;
}

// The wall contacts of one particle in a cell with facets.  `live` says
// whether any of its history slots may be in use; when none is, no slot is
// searched for the facets it does not touch (REMOVE_COLLISION would find
// nothing).  The particle's velocity, spin, mass and phase are read at its
// first contact only.
template <int COLL>
__device__ void wall_contacts(const DevParams& p, const WallCtx& w, int me, PState& s, bool live,
                              const double4* __restrict__ vel4, const double4* __restrict__ omg4,
                              const uint8_t* __restrict__ phase, double f[3], double t[3],
                              unsigned long long& nwc, unsigned& eflags) {
  const int cell = p.cell_off + w.dg_pijk[me] - 1;
  const int fs = w.fbin_start[cell], fe = w.fbin_start[cell + 1];
  bool have_kin = false;
  const double r = s.r;
  const double radsq = r * r;
  double pmax[3], pmin[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) { pmax[c] = s.x[c] + r; pmin[c] = s.x[c] - r; }
  for (int q = fs; q < fe; ++q) {
    const FacetBinEntry e = w.fbin[q];
    const int nf = e.id;
    if (e.mn > pmax[e.dir]) { if (live) remove_collision(p, w, me, nf); continue; }
    if (e.mx < pmin[e.dir]) { if (live) remove_collision(p, w, me, nf); continue; }
    const double* V = w.vertex + 9 * (size_t)nf;
    const double* N = w.norm_face + 3 * (size_t)nf;
    double d1[3] = {V[0] - s.x[0], V[1] - s.x[1], V[2] - s.x[2]};
    double nn[3] = {N[0], N[1], N[2]};
    const double line_t = dot3(d1, nn);
    if (line_t <= -1.0001 * r) { if (live) remove_collision(p, w, me, nf); continue; }
    double cpt[3]; bool poe; int edge;
    closest_pt(p, w, nf, s.x, cpt, poe, edge);
    double dist[3] = {cpt[0] - s.x[0], cpt[1] - s.x[1], cpt[2] - s.x[2]};
    const double distsq = dot3(dist, dist);
    if (distsq >= radsq - SMALL_NUMBER) { if (live) remove_collision(p, w, me, nf); continue; }
    if (poe && w.ignore_edge[4 * (size_t)nf + edge]) continue;
    if (!have_kin) {
      const double4 b = vel4[me], c = omg4[me];
      s.v[0] = b.x; s.v[1] = b.y; s.v[2] = b.z; s.m = b.w;
      s.w[0] = c.x; s.w[1] = c.y; s.w[2] = c.z;
      s.ph = phase[me];
      have_kin = true;
    }
    const double distmod = sqrt(distsq);
    double nrm[3] = {dist[0], dist[1], dist[2]};
    if (distsq > 0) { const double sq = sqrt(distsq); for (int c = 0; c < 3; ++c) nrm[c] = dist[c] / sq; }
    const double overlap_n = r - distmod;
    double wxn[3]; cross3(s.w, nrm, wxn);
    double vrel[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) { vrel[c] = s.v[c] + distmod * wxn[c]; vrel[c] = vrel[c] - (0.0 + 0.0); }
    const double vrn = dot3(vrel, nrm);
    double vt[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) vt[c] = vrel[c] - vrn * nrm[c];
    double kn_w, kt_w, etan_w, etat_w;
    const int ph = s.ph;
    if (COLL == DEM_COLL_HERTZ) {
      double so = 0.0;
      if (overlap_n > 0) so = sqrt(overlap_n);
      kn_w = p.hkwn[ph] * so * sqrt(r);
      kt_w = p.hkwt[ph] * so * sqrt(r);
      etan_w = p.etanw[ph] * sqrt(so) * sqrt(p.hkwn[ph] * sqrt(r) * s.m);
      etat_w = p.etatw[ph] * sqrt(so) * sqrt(p.hkwt[ph] * sqrt(r) * s.m);
    } else {
      kn_w = p.kn_w; kt_w = p.kt_w;
      etan_w = p.etanw[ph] * sqrt(s.m);
      etat_w = p.etatw[ph] * sqrt(s.m);
    }
    double fn[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) fn[c] = -(kn_w * overlap_n * nrm[c] + etan_w * vrn * nrm[c]);
    double hist[3];
    const int slot = get_collision(p, w, me, nf, cell, hist);
    if (slot < 0) { eflags |= EF_WALL_SLOTS; continue; }
    double ot[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) ot[c] = p.dt * vt[c] + hist[c];
    const double mag = sqrt(dot3(ot, ot));
    double ft[3];
    if (mag > 0.0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) ft[c] = -kt_w * ot[c] - etat_w * vt[c];
      const double ftmd = sqrt(dot3(ft, ft));
      const double fnmd = p.mew_w * sqrt(dot3(fn, fn));
      if (ftmd > fnmd) {
        double tg[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) tg[c] = ot[c] / mag;
#pragma unroll
        for (int c = 0; c < 3; ++c) ft[c] = -fnmd * tg[c];
#pragma unroll
        for (int c = 0; c < 3; ++c) ot[c] = (fnmd / kt_w) * tg[c];
      }
    } else {
      ft[0] = ft[1] = ft[2] = 0.0;
    }
    double* wp = w.wall_pft + ((size_t)me * p.cmax + slot) * 3;  // UPDATE_COLLISION
    wp[0] = ot[0]; wp[1] = ot[1]; wp[2] = ot[2];
    ++nwc;
#pragma unroll
    for (int c = 0; c < 3; ++c) f[c] = f[c] + fn[c] + ft[c];
    double nxf[3]; cross3(nrm, ft, nxf);
#pragma unroll
    for (int c = 0; c < 3; ++c) t[c] = t[c] + distmod * nxf[c];
    if (p.mew_rw > 0.0) {
      const double om = sqrt(dot3(s.w, s.w));
      if (om > 0.0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) t[c] = t[c] + -(p.mew_rw * (2.0 * r) * kn_w * overlap_n * s.w[c] / om);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Squared distance from x to the closest point of triangle (a, b, c): the
// Voronoi-region walk over vertices, edges and face (C. Ericson, Real-Time
// Collision Detection, 2005, section 5.1.5), with no edge or vertex left out.
__device__ __forceinline__ double tri_dist2(const double* __restrict__ V, const double x[3]) {
  double a[3], ab[3], ac[3], ap[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) { a[k] = V[k]; ab[k] = V[3 + k] - a[k]; ac[k] = V[6 + k] - a[k]; ap[k] = x[k] - a[k]; }
  const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  double q[3];
  auto at = [&](double u, double v) {
#pragma unroll
    for (int k = 0; k < 3; ++k) q[k] = a[k] + u * ab[k] + v * ac[k];
  };
  if (d1 <= 0.0 && d2 <= 0.0) { at(0.0, 0.0); goto done; }
  {
    double bp[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) bp[k] = ap[k] - ab[k];
    const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { at(1.0, 0.0); goto done; }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) { at(d1 / (d1 - d3), 0.0); goto done; }
    double cp[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) cp[k] = ap[k] - ac[k];
    const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) { at(0.0, 1.0); goto done; }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) { at(0.0, d2 / (d2 - d6)); goto done; }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
      const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
      at(1.0 - w, w);
      goto done;
    }
    const double den = 1.0 / (va + vb + vc);
    at(vb * den, vc * den);
  }
done:
  double d[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) d[k] = x[k] - q[k];
  return dot3(d, d);
}

// Clearance of every NORMAL particle in a DES cell with facets from those
// facets at a build (valid while the particle stays in that cell: the
// per-step placement of a periodic system sets it to -1, unknown, when the
// particle changes cell): min over the cell's facets of |x - closest point| - r,
// less a margin of 1e-6 r for the rounding of the closest point, rounded
// down to float.  A particle whose clearance exceeds the displacement bound
// since the build touches none of them (the reference's contact test is
// |x - c|^2 < r^2 - SMALL_NUMBER), so with no history it has no wall work.
template <bool B>
__global__ void k_wall_gaps(DevParams p0, BatchView bv, WallCtx w, const double4* __restrict__ pos4,
                            const int8_t* __restrict__ state, const uint8_t* __restrict__ wall_cand,
                            float* __restrict__ wgap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p0.n) return;
  // a particle that is not NORMAL now may become so before the next build
  // (ENTERING, EXITING): clearance unknown, its walls are checked
  if (state[i] != DEM_STATE_NORMAL) { wgap[i] = -1.0f; return; }
  // no facets in its cell: none to touch while it stays there (a move to
  // another cell before the next build clears the screen, see dg_place users)
  if (!wall_cand[i]) { wgap[i] = FLT_MAX; return; }
  const DevParams& p = sysp<B>(p0, bv, i);
  const int cell = p.cell_off + w.dg_pijk[i] - 1;
  const double4 a = pos4[i];
  const double x[3] = {a.x, a.y, a.z};
  double dmin2 = HUGE_VAL;
  for (int q = w.fbin_start[cell]; q < w.fbin_start[cell + 1]; ++q)
    dmin2 = fmin(dmin2, tri_dist2(w.vertex + 9 * (size_t)w.fbin[q].id, x));
  wgap[i] = __double2float_rd(sqrt(dmin2) - a.w - 1e-6 * a.w);
}

// The particles with wall work this step: NORMAL particles whose DES cell
// holds facets and whose clearance at the last build does not exceed the
// displacement bound since, and NORMAL particles whose history slots may be
// in use (k_walls clears them, or updates them).  A thread screens four
// consecutive particles: their flags arrive in one 32-bit load per array and
// their clearances in one float4, all issued before any is used, so the
// kernel waits on memory about once.  Each block of WALL_LIST_T threads
// appends its particles in index order with one atomic; blocks land in
// arbitrary order, which does not matter: each particle's wall terms depend
// on it alone.
constexpr int WALL_LIST_T = 1024;
static_assert(WALL_LIST_T == 32 * 32, "one warp scans the warp counts");
__device__ __forceinline__ unsigned wall_need(unsigned st, unsigned live, unsigned cand, float gap, double bound) {
  return (st == (unsigned)(uint8_t)DEM_STATE_NORMAL && (live || (cand && !((double)gap > bound)))) ? 1u : 0u;
}
__global__ void __launch_bounds__(WALL_LIST_T)
k_wall_list(int n, const int8_t* __restrict__ state, const uint8_t* __restrict__ wall_cand,
            const uint8_t* __restrict__ wall_live, const float* __restrict__ wgap, const double* __restrict__ skin,
            int* __restrict__ list, int* __restrict__ count) {
  __shared__ int warp_n[WALL_LIST_T / 32];
  const int i0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  const double bound = *skin;
  uint32_t st = 0, lv = 0, cd = 0;
  float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
  if (i0 + 3 < n) {  // the arrays are separate allocations: 256-byte aligned
    st = *reinterpret_cast<const uint32_t*>(state + i0);
    lv = *reinterpret_cast<const uint32_t*>(wall_live + i0);
    cd = *reinterpret_cast<const uint32_t*>(wall_cand + i0);
    g = *reinterpret_cast<const float4*>(wgap + i0);
  } else {
    float gg[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (i0 + j < n) {
        st |= (uint32_t)(uint8_t)state[i0 + j] << (8 * j);
        lv |= (uint32_t)wall_live[i0 + j] << (8 * j);
        cd |= (uint32_t)wall_cand[i0 + j] << (8 * j);
        gg[j] = wgap[i0 + j];
      }
    g = make_float4(gg[0], gg[1], gg[2], gg[3]);
  }
  // bit j: particle i0+j has wall work (bytes past n are zero: state 0 is
  // not NORMAL)
  const unsigned need = wall_need(st & 255u, lv & 255u, cd & 255u, g.x, bound) |
                        (wall_need((st >> 8) & 255u, (lv >> 8) & 255u, (cd >> 8) & 255u, g.y, bound) << 1) |
                        (wall_need((st >> 16) & 255u, (lv >> 16) & 255u, (cd >> 16) & 255u, g.z, bound) << 2) |
                        (wall_need(st >> 24, lv >> 24, cd >> 24, g.w, bound) << 3);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int mine = __popc(need);
  int incl = mine;  // inclusive scan of the counts over the warp
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_n[warp] = incl;
  __syncthreads();
  if (warp == 0) {  // the warps' offsets: a scan of their counts, and one atomic
    const int c = warp_n[lane];
    int wi = c;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    const int tot = __shfl_sync(0xffffffffu, wi, 31);
    int base = 0;
    if (lane == 0 && tot) base = atomicAdd(count, tot);
    base = __shfl_sync(0xffffffffu, base, 0);
    warp_n[lane] = base + wi - c;
  }
  __syncthreads();
  int at = warp_n[warp] + incl - mine;
  for (int j = 0; j < 4; ++j)
    if ((need >> j) & 1u) list[at++] = i0 + j;
}

// Kernel 1 (per listed particle): wall contacts of NORMAL particles whose DES
// cell holds facets.  Writes the particle's wall force and torque, which are
// the first terms of FC/TOW in the reference's order
// (CALC_DEM_FORCE_WITH_WALL_STL runs before the pair loop,
// calc_force_dem.f:113).  Persistent grid over the list built by k_wall_list.
template <int COLL, bool B>
__global__ void __launch_bounds__(128)
k_walls(DevParams p0, BatchView bv, WallCtx w, const int* __restrict__ wlist, const int* __restrict__ wcount,
        const double4* __restrict__ pos4, const double4* __restrict__ vel4,
        const double4* __restrict__ omg4, const uint8_t* __restrict__ phase,
        uint8_t* __restrict__ wall_live, const uint8_t* __restrict__ wall_cand, double* __restrict__ wf,
        uint8_t* __restrict__ wall_hit, DevErr* __restrict__ err) {
  const int nw = *wcount;
  unsigned long long nwc = 0;
  unsigned eflags = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nw; q += gridDim.x * blockDim.x) {
    const int me = wlist[q];
    const DevParams& p = sysp<B>(p0, bv, me);
    if (!wall_cand[me]) {
      // no facet near: clear the history once (calc_collision_wall_mod.f:194-198)
      int* fid = w.wall_fid + (size_t)me * p.cmax;
      double* wp = w.wall_pft + (size_t)me * p.cmax * 3;
      for (int s = 0; s < p.cmax; ++s) fid[s] = -1;
      for (int s = 0; s < 3 * p.cmax; ++s) wp[s] = 0.0;
      wall_live[me] = 0;
      continue;
    }
    PState S;
    const double4 a = pos4[me];
    S.x[0] = a.x; S.x[1] = a.y; S.x[2] = a.z; S.r = a.w;
    double f[3] = {0.0, 0.0, 0.0}, t[3] = {0.0, 0.0, 0.0};
    const bool live = wall_live[me] != 0;
    const unsigned long long nwc0 = nwc;
    wall_contacts<COLL>(p, w, me, S, live, vel4, omg4, phase, f, t, nwc, eflags);
    const bool hit = nwc > nwc0;
    bool used = hit;
    if (!hit && live) {
      const int* fid = w.wall_fid + (size_t)me * p.cmax;
      for (int s = 0; s < p.cmax; ++s) used = used || fid[s] != -1;
    }
    if (used != live) wall_live[me] = used ? 1 : 0;
    if (hit) {
      // the wall terms are the first terms of FC/TOW; the gather reads
      // them only for particles marked here
      double* o = wf + 6 * (size_t)me;
      o[0] = f[0]; o[1] = f[1]; o[2] = f[2]; o[3] = t[0]; o[4] = t[1]; o[5] = t[2];
      wall_hit[me] = 1;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    nwc += __shfl_down_sync(0xffffffffu, nwc, o);
    eflags |= __shfl_down_sync(0xffffffffu, eflags, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (nwc) atomicAdd(&err->n_wall_contacts, nwc);
    if (eflags) atomicOr(&err->flags, eflags);
  }
}

// Kernel 2 (per pair): one CC iteration of CALC_FORCE_DEM, evaluated once
// per pair.  A pair whose gap at the last build is more than twice the
// bound on any particle's displacement since (and whose history is zero) is
// apart without a look at the particles: the reference's apart test would
// find it apart and leave its zero history zero, so it is skipped.  The
// apart test of the others needs only the two positions; velocities, spins
// and masses are gathered only for pairs in contact.  The tangential history
// PFT is updated in place (only this kernel reads it).  pflag keeps, per
// pair, PF_CONTACT (in contact at this pass) and PF_HIST (history nonzero),
// so a pair that stays apart with a zero history costs no history traffic.
// The contact terms go to a record that both particles read back in
// kernel 3, and both particles of a contact are marked in `touched`.
template <int COLL, bool B>
__global__ void __launch_bounds__(256, 2)
k_pairs(DevParams p0, BatchView bv, const int* __restrict__ d_np, long long cap, const int* __restrict__ owner,
        const int* __restrict__ nbrs, const double4* __restrict__ pos4, const double4* __restrict__ vel4,
        const double4* __restrict__ omg4, const int8_t* __restrict__ state, const uint8_t* __restrict__ phase,
        double* __restrict__ pft, uint8_t* __restrict__ pflag, uint8_t* __restrict__ touched,
        const float* __restrict__ pgap, const double* __restrict__ skin, PairRec* __restrict__ prec,
        DevErr* __restrict__ err) {
  // persistent grid-stride loop over the device-side pair count (the grid
  // size does not depend on the list, so the launch can live in a graph)
  const long long np = min((long long)*d_np, cap);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const double reach = 2.0 * skin[0];
  unsigned long long ncont = 0;
  unsigned eflags = 0;
  // four consecutive pairs per iteration: their flags and gaps arrive in
  // one load each, so a run of apart pairs costs few dependent loads
  const long long ng = (np + 3) / 4;
  for (long long g4 = (long long)blockIdx.x * blockDim.x + threadIdx.x; g4 < ng; g4 += stride) {
    const long long c0 = 4 * g4;
    uint32_t fw = 0;  // the four flags, one per byte
    float4 gq = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c0 + 3 < np) {
      fw = *reinterpret_cast<const uint32_t*>(pflag + c0);
      gq = *reinterpret_cast<const float4*>(pgap + c0);
    } else {
      if (c0 < np) { fw |= pflag[c0]; gq.x = pgap[c0]; }
      if (c0 + 1 < np) { fw |= (uint32_t)pflag[c0 + 1] << 8; gq.y = pgap[c0 + 1]; }
      if (c0 + 2 < np) { fw |= (uint32_t)pflag[c0 + 2] << 16; gq.z = pgap[c0 + 2]; }
    }
    // bit j: pair c0+j is provably apart
    const unsigned apart = ((!(fw & PF_HIST) && (double)gq.x > reach) ? 1u : 0u) |
                           ((!((fw >> 8) & PF_HIST) && (double)gq.y > reach) ? 2u : 0u) |
                           ((!((fw >> 16) & PF_HIST) && (double)gq.z > reach) ? 4u : 0u) |
                           ((!((fw >> 24) & PF_HIST) && (double)gq.w > reach) ? 8u : 0u);
    // the particles of the group's pairs in one load each, when any pair
    // needs them (a group past the list's end has fewer than four)
    int4 o4 = make_int4(0, 0, 0, 0), n4 = make_int4(0, 0, 0, 0);
    const unsigned live = c0 + 3 < np ? 15u : (1u << (unsigned)(np - c0)) - 1u;
    if (~apart & live) {
      if (c0 + 3 < np) {
        o4 = *reinterpret_cast<const int4*>(owner + c0);
        n4 = *reinterpret_cast<const int4*>(nbrs + c0);
      } else {
        o4.x = owner[c0]; n4.x = nbrs[c0];
        if (c0 + 1 < np) { o4.y = owner[c0 + 1]; n4.y = nbrs[c0 + 1]; }
        if (c0 + 2 < np) { o4.z = owner[c0 + 2]; n4.z = nbrs[c0 + 2]; }
      }
    }
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
    const long long cc = c0 + j;
    if (cc >= np) break;
    const uint8_t f0 = (uint8_t)(fw >> (8 * j));
    // provably apart: its gap at the build exceeds what the two particles
    // can have closed since, and its history is zero (stays zero)
    if ((apart >> j) & 1u) {
      if (f0) pflag[cc] = 0;
      continue;
    }
    const int ll = j == 0 ? o4.x : (j == 1 ? o4.y : (j == 2 ? o4.z : o4.w));
    const int i = j == 0 ? n4.x : (j == 1 ? n4.y : (j == 2 ? n4.z : n4.w));
    uint8_t f = f0 & PF_HIST;  // NONEXISTENT partner or zero distance: history kept
    double* ph = pft + 3 * cc;
    // the states and the positions in one round of loads (any slot's
    // position can be read; it is used only for existing particles)
    const double4 a = pos4[ll], b = pos4[i];
    const int8_t sl = state[ll], si = state[i];
    if (si != DEM_STATE_NONEXISTENT && sl != DEM_STATE_NONEXISTENT) {
      const DevParams& p = sysp<B>(p0, bv, ll);
      PState L, I;
      L.x[0] = a.x; L.x[1] = a.y; L.x[2] = a.z; L.r = a.w;
      I.x[0] = b.x; I.x[1] = b.y; I.x[2] = b.z; I.r = b.w;
      const double r_lm = L.r + I.r;
      double dist[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double pj = I.x[c];
        double s = periodic_shift(p, c, pj - L.x[c]);
        if (s != 0.0) pj = pj + s;
        dist[c] = pj - L.x[c];
      }
      const double d2 = dot3(dist, dist);
      if (d2 > (r_lm - SMALL_NUMBER) * (r_lm - SMALL_NUMBER)) {
        if (f0 & PF_HIST) { ph[0] = 0.0; ph[1] = 0.0; ph[2] = 0.0; }
        f = 0;
      } else if (d2 == 0.0) {
        eflags |= EF_ZERO_DIST;
        err->zero_a = ll; err->zero_b = i;
      } else {
        const double4 va = vel4[ll], vb = vel4[i], wa = omg4[ll], wb = omg4[i];
        L.v[0] = va.x; L.v[1] = va.y; L.v[2] = va.z; L.m = va.w;
        I.v[0] = vb.x; I.v[1] = vb.y; I.v[2] = vb.z; I.m = vb.w;
        L.w[0] = wa.x; L.w[1] = wa.y; L.w[2] = wa.z;
        I.w[0] = wb.x; I.w[1] = wb.y; I.w[2] = wb.z;
        L.ph = phase[ll]; I.ph = phase[i];
        double pin[3] = {0.0, 0.0, 0.0};
        if (f0 & PF_HIST) { pin[0] = ph[0]; pin[1] = ph[1]; pin[2] = ph[2]; }
        double pout[3];
        PairRec r;
        contact_force<COLL>(p, L, I, dist, d2, pin, pout, r);
        ph[0] = pout[0]; ph[1] = pout[1]; ph[2] = pout[2];
        prec[cc] = r;
        touched[ll] = 1;
        touched[i] = 1;
        f = PF_CONTACT | ((pout[0] != 0.0 || pout[1] != 0.0 || pout[2] != 0.0) ? PF_HIST : 0);
        ++ncont;
      }
    }
    if (f != f0) pflag[cc] = f;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    ncont += __shfl_down_sync(0xffffffffu, ncont, o);
    eflags |= __shfl_down_sync(0xffffffffu, eflags, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (ncont) atomicAdd(&err->n_contacts, ncont);
    if (eflags) atomicOr(&err->flags, eflags);
  }
}

// Rolling-friction torque of one particle in a pair (calc_force_dem.f:491-506):
// -MEW_R*(2*R)*KN_DES*OVERLAP_N*OMEGA/|OMEGA|, evaluated left to right.
__device__ __forceinline__ void add_rolling(const DevParams& p, double r, const double w[3], double om,
                                            const PairRec& q, double t[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) t[c] = t[c] + -(p.mew_r * (2.0 * r) * q.kn * q.ov * w[c] / om);
}

// One pair's terms on one of its particles: the owner adds +FC and DCL2*TF,
// the neighbour -FC and DCI2*TF (calc_force_dem.f:466-506).
template <bool NBR>
__device__ __forceinline__ void add_pair_terms(const DevParams& p, const PairRec& o, bool roll, double r,
                                               const double w[3], double om, double f[3], double t[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) f[c] = NBR ? f[c] - o.fc[c] : f[c] + o.fc[c];
#pragma unroll
  for (int c = 0; c < 3; ++c) t[c] = t[c] + (NBR ? o.dci2 : o.dcl2) * o.tf[c];
  if (roll && om > 0.0) add_rolling(p, r, w, om, o, t);
}

// The records of the set bits of `mask` in ascending order; each record's
// load is issued before the previous record is added.
template <bool NBR, class Idx>
__device__ __forceinline__ void add_flagged(const DevParams& p, unsigned mask, Idx idx,
                                            const PairRec* __restrict__ prec, bool roll, double r,
                                            const double w[3], double om, double f[3], double t[3]) {
  if (!mask) return;
  PairRec cur = prec[idx(__ffs(mask) - 1)];
  mask &= mask - 1u;
  while (true) {
    const bool more = mask != 0u;
    PairRec nxt;
    if (more) {
      nxt = prec[idx(__ffs(mask) - 1)];
      mask &= mask - 1u;
    }
    add_pair_terms<NBR>(p, cur, roll, r, w, om, f, t);
    if (!more) break;
    cur = nxt;
  }
}

// Incoming entries from q on (sorted by owner) whose owner is at most lim,
// 32 at a time: the window's contact flags are read first (independent
// loads), then the flagged records.  Returns the first entry not taken.
__device__ __forceinline__ int add_incoming(const DevParams& p, int q, int ie, int lim,
                                            const int2* __restrict__ in_pair, const uint8_t* __restrict__ pflag,
                                            const PairRec* __restrict__ prec, bool roll, double r,
                                            const double w[3], double om, double f[3], double t[3]) {
  while (q < ie) {
    const int cnt = min(32, ie - q);
    unsigned mask = 0u;
    int stop = cnt;
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      if (k < cnt) {
        const int2 e = in_pair[q + k];
        if (e.x > lim && k < stop) stop = k;
        if (pflag[e.y] & PF_CONTACT) mask |= 1u << k;
      }
    }
    if (stop < 32) mask &= (1u << stop) - 1u;
    const int base = q;
    add_flagged<true>(p, mask, [&](int k) { return in_pair[base + k].y; }, prec, roll, r, w, om, f, t);
    q += stop;
    if (stop < cnt) break;
  }
  return q;
}

// The particle's own row [rs, re), 32 entries at a time.
__device__ __forceinline__ void add_own(const DevParams& p, int rs, int re, const uint8_t* __restrict__ pflag,
                                        const PairRec* __restrict__ prec, bool roll, double r, const double w[3],
                                        double om, double f[3], double t[3]) {
  for (int base = rs; base < re; base += 32) {
    const int cnt = min(32, re - base);
    unsigned mask = 0u;
#pragma unroll 8
    for (int k = 0; k < 32; ++k)
      if (k < cnt && (pflag[base + k] & PF_CONTACT)) mask |= 1u << k;
    add_flagged<false>(p, mask, [&](int k) { return base + k; }, prec, roll, r, w, om, f, t);
  }
}

// Kernel 3 (per particle): sums FC/TOW in the serial reference's order --
// wall terms, pairs owned by lower-index particles (ascending owner), the
// particle's own row, pairs owned by higher-index particles -- and either
// stores them (MODE 0) or integrates them in place of CFNEWVALUES
// (MODE 1 = Euler, MODE 2 = Adams-Bashforth).
template <int MODE, bool B>
__global__ void __launch_bounds__(256, 3)
k_gather(DevParams p0, BatchView bv, const double4* __restrict__ pos_c, const double4* __restrict__ vel_c,
         const double4* __restrict__ omg_c, double4* __restrict__ pos_n, double4* __restrict__ vel_n,
         double4* __restrict__ omg_n, const int8_t* __restrict__ state, const double* __restrict__ wf,
         const int* __restrict__ row_end, const int* __restrict__ in_start, const int2* __restrict__ in_pair,
         const uint8_t* __restrict__ pflag, uint8_t* __restrict__ touched, uint8_t* __restrict__ wall_hit,
         const PairRec* __restrict__ prec,
         double* __restrict__ fc, double* __restrict__ tow, double* __restrict__ acc_old,
         double* __restrict__ rot_acc_old, unsigned* __restrict__ vslot,
         CellOut cells) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= p0.n) return;
  const DevParams& p = sysp<B>(p0, bv, me);
  const int8_t st = state[me];
  // the contacts of this pass; a particle in none has no terms to add
  const bool wh = wall_hit[me] != 0, ph = touched[me] != 0;
  if (wh) wall_hit[me] = 0;
  if (ph) touched[me] = 0;
  // no torque and Euler: the spin stays (OMEGA_NEW = OMEGA_NEW + 0), so it
  // is neither read nor written (the spin array is updated in place)
  const bool keep_w = MODE == 1 && !wh && !ph;
  const double4 W = keep_w ? make_double4(0.0, 0.0, 0.0, 0.0) : omg_c[me];
  const double w[3] = {W.x, W.y, W.z};
  double f[3] = {0.0, 0.0, 0.0}, t[3] = {0.0, 0.0, 0.0};
  if (wh && st == DEM_STATE_NORMAL) {
    const double* o = wf + 6 * (size_t)me;
    f[0] = o[0]; f[1] = o[1]; f[2] = o[2]; t[0] = o[3]; t[1] = o[4]; t[2] = o[5];
  }
  if (st != DEM_STATE_NONEXISTENT && ph) {
    const bool roll = p.mew_r > 0.0;
    const double r = pos_c[me].w;
    double om = 0.0;
    if (roll) om = sqrt(dot3(w, w));
    const int rs = me ? row_end[me - 1] : 0, re = row_end[me];
    const int is = in_start[me], ie = in_start[me + 1];
    const int q = add_incoming(p, is, ie, me, in_pair, pflag, prec, roll, r, w, om, f, t);
    add_own(p, rs, re, pflag, prec, roll, r, w, om, f, t);
    add_incoming(p, q, ie, INT_MAX, in_pair, pflag, prec, roll, r, w, om, f, t);
  }
  const double4 X = pos_c[me], V = vel_c[me];
  const double x[3] = {X.x, X.y, X.z}, v[3] = {V.x, V.y, V.z};
  finish_particle<MODE>(p, me, st, x, v, w, X.w, V.w, W.w, f, t, pos_n, vel_n, omg_n, fc, tow, acc_old,
                        rot_acc_old, vslot, cells, keep_w);
}

// CFUPDATEOLD + CFNEWVALUES from FC/TOW, in place; zeroes FC/TOW.
template <int INTG, bool B>
__global__ void k_integrate(DevParams p0, BatchView bv, double4* __restrict__ pos4, double4* __restrict__ vel4,
                            double4* __restrict__ omg4, const int8_t* __restrict__ state,
                            double* __restrict__ fc, double* __restrict__ tow,
                            double* __restrict__ acc_old, double* __restrict__ rot_acc_old,
                            unsigned* __restrict__ vslot) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= p0.n) return;
  const DevParams& p = sysp<B>(p0, bv, me);
  const size_t n = (size_t)p.n;
  const double4 X = pos4[me], V = vel4[me], W = omg4[me];
  const double x[3] = {X.x, X.y, X.z}, v[3] = {V.x, V.y, V.z}, w[3] = {W.x, W.y, W.z};
  double f[3], t[3];
  for (int c = 0; c < 3; ++c) {
    f[c] = fc[c * n + me]; t[c] = tow[c * n + me];
    fc[c * n + me] = 0.0; tow[c * n + me] = 0.0;
  }
  finish_particle<INTG == DEM_INTG_AB2 ? 2 : 1>(p, me, state[me], x, v, w, X.w, V.w, W.w, f, t, pos4, vel4, omg4,
                                                fc, tow, acc_old, rot_acc_old, vslot);
}

static WallCtx wall_ctx(dem_handle* h) {
  WallCtx w;
  w.vertex = h->vertex; w.norm_face = h->norm_face; w.ignore_edge = h->ignore_edge;
  w.fbin_start = h->fbin_start; w.fbin = h->fbin; w.dg_pijk = h->dg_pijk;
  w.wall_fid = h->wall_fid; w.wall_pft = h->wall_pft; w.nf = h->nf;
  return w;
}

template <int COLL, bool B>
static void launch_walls_t(dem_handle* h) {
  const int c = h->cur;
  const int T = 128;
  cudaMemsetAsync(h->d_nwall, 0, sizeof(int), h->stream);
  const int nq = (h->nl() + 3) / 4;  // four particles per thread
  k_wall_list<<<(nq + WALL_LIST_T - 1) / WALL_LIST_T, WALL_LIST_T, 0, h->stream>>>(
      h->nl(), h->state, h->wall_cand, h->wall_live, h->wgap, h->skin, h->wall_list, h->d_nwall);
  // persistent: the resident blocks of the kernel's register budget
  k_walls<COLL, B><<<h->n_sm * 4, T, 0, h->stream>>>(h->dp, h->bview(), wall_ctx(h), h->wall_list, h->d_nwall,
                                                     h->pos4[c], h->vel4[c], h->omg4[c], h->phase, h->wall_live,
                                                     h->wall_cand, h->wf, h->wall_hit, h->derr);
  h->launches += 2;
}

template <int COLL, bool B>
static void launch_pairs_t(dem_handle* h) {
  const int c = h->cur;
  const int T = h->tune.pair_threads;
  k_pairs<COLL, B><<<(unsigned)(h->n_sm * h->tune.pair_bpsm), T, 0, h->stream>>>(
      h->dp, h->bview(), h->d_np, h->pair_cap, h->pair_owner, h->nbrs[h->rb], h->pos4[c], h->vel4[c], h->omg4[c],
      h->state, h->phase, h->pft[h->pcur], h->pflag(), h->touched, h->pgap, h->skin, h->prec, h->derr);
  DEM_LAUNCH(h);
}

template <int MODE, bool B>
static void launch_gather_t(dem_handle* h) {
  const int T = h->tune.gather_threads, G = (h->nl() + T - 1) / T;
  const int c = h->cur;
  k_gather<MODE, B><<<G, T, 0, h->stream>>>(h->dp, h->bview(), h->pos4[c], h->vel4[c], h->omg4[c], h->pos4[1 - c],
                                            h->vel4[1 - c], h->omg4[1 - c], h->state, h->wf, h->row_end[h->rb], h->in_start, h->in_pair, h->pflag(),
                                            h->touched, h->wall_hit, h->prec, h->fc, h->tow, h->acc_old,
                                            h->rot_acc_old, h->vslot, gather_cells<MODE, B>(h));
  DEM_LAUNCH(h);
}

void launch_wall_gaps(dem_handle* h) {
  if (h->nf <= 0) return;
  const int T = 256, G = (h->nl() + T - 1) / T;
  if (h->batch())
    k_wall_gaps<true><<<G, T, 0, h->stream>>>(h->dp, h->bview(), wall_ctx(h), h->pos4[h->cur], h->state,
                                              h->wall_cand, h->wgap);
  else
    k_wall_gaps<false><<<G, T, 0, h->stream>>>(h->dp, h->bview(), wall_ctx(h), h->pos4[h->cur], h->state,
                                               h->wall_cand, h->wgap);
  DEM_LAUNCH(h);
}

static void launch_walls(dem_handle* h) {
  if (h->nf <= 0) return;
  const bool hz = h->dp.coll == DEM_COLL_HERTZ;
  if (h->batch()) hz ? launch_walls_t<DEM_COLL_HERTZ, true>(h) : launch_walls_t<DEM_COLL_LSD, true>(h);
  else hz ? launch_walls_t<DEM_COLL_HERTZ, false>(h) : launch_walls_t<DEM_COLL_LSD, false>(h);
}

template <bool B>
static void launch_pairs_fp64(dem_handle* h) {
  if (h->dp.coll == DEM_COLL_HERTZ) launch_pairs_t<DEM_COLL_HERTZ, B>(h);
  else launch_pairs_t<DEM_COLL_LSD, B>(h);
}

template <bool B>
static void launch_gather_fp64(dem_handle* h, int mode) {
  if (mode == 0) launch_gather_t<0, B>(h);
  else if (mode == 1) launch_gather_t<1, B>(h);
  else launch_gather_t<2, B>(h);
}

// The two timed parts of the force step for the autotuner.
void launch_pairs_only(dem_handle* h) {
  if (h->dp.prec == DEM_PREC_SPLIT) launch_pairs_split(h);
  else if (h->batch()) launch_pairs_fp64<true>(h);
  else launch_pairs_fp64<false>(h);
}

void launch_gather_only(dem_handle* h) {
  if (h->dp.prec == DEM_PREC_SPLIT) launch_gather_split(h, 0);
  else if (h->batch()) launch_gather_fp64<true>(h, 0);
  else launch_gather_fp64<false>(h, 0);
}

// Contact forces of the current state.  mode: 0 = into FC/TOW, 1/2 = fused
// Euler/AB2 integration into the other state buffer.  The collision model,
// integrator and force precision are common to all systems of a batch.
static void launch_force_kernels(dem_handle* h, int mode, bool split) {
  // The wall kernels and the pair kernel read the same state and write
  // disjoint arrays (walls: wall_hit, wf and the wall histories; pairs: the
  // pair histories, flags, records and touched marks), so the wall work runs
  // on the side stream beside the pair kernel and the gather waits for both
  // (in a captured step, two branches of the graph).  With the parts of the
  // step timed (profiling), they run one after the other.
  const bool side = h->nf > 0 && h->side_stream && !h->prof;
  if (side) {
    cudaEventRecord(h->ev_fork, h->stream);
    cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0);
    cudaStream_t main = h->stream;
    h->stream = h->side_stream;
    launch_walls(h);
    h->stream = main;
    cudaEventRecord(h->ev_join, h->side_stream);
  } else {
    ProfScope ps(h, DEM_PROF_WALLS);
    launch_walls(h);
  }
  {
    ProfScope ps(h, DEM_PROF_PAIRS);
    if (split) launch_pairs_split(h);
    else if (h->batch()) launch_pairs_fp64<true>(h);
    else launch_pairs_fp64<false>(h);
  }
  if (side) cudaStreamWaitEvent(h->stream, h->ev_join, 0);
  ProfScope ps(h, DEM_PROF_GATHER);
  if (split) launch_gather_split(h, mode);
  else if (h->batch()) launch_gather_fp64<true>(h, mode);
  else launch_gather_fp64<false>(h, mode);
}

// Displacement bound since the last build += this step's largest particle
// displacement bound; the slots are cleared for the next step.
__global__ void k_skin(double* __restrict__ skin, unsigned* __restrict__ vslot, CandState* __restrict__ cand) {
  const unsigned m = __reduce_max_sync(0xffffffffu, vslot[threadIdx.x]);
  vslot[threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    skin[0] = skin[0] + (double)__uint_as_float(m);
    if (cand) cand->disp = cand->disp + (double)__uint_as_float(m);  // the candidate list's bound too
  }
}

__global__ void k_set_skin(double* __restrict__ skin, double v) { skin[0] = v; }

void launch_skin(dem_handle* h) {
  k_skin<<<1, 32, 0, h->stream>>>(h->skin, h->vslot, h->cand);
  DEM_LAUNCH(h);
}

void skin_unknown(dem_handle* h) {
  k_set_skin<<<1, 1, 0, h->stream>>>(h->skin, HUGE_VAL);
  DEM_LAUNCH(h);
  // positions (or walls) changed from outside: the candidate list starts over
  if (h->cand) cudaMemsetAsync(&h->cand->have, 0, sizeof(int), h->stream);
}

int run_force(dem_handle* h, bool fused) {
  ProfScope ps(h, DEM_PROF_FORCE);
  h->dp.first_pass = h->first_pass ? 1 : 0;
  const int mode = !fused ? 0 : (h->dp.intg == DEM_INTG_AB2 ? 2 : 1);
  launch_force_kernels(h, mode, h->dp.prec == DEM_PREC_SPLIT);
  if (fused) launch_skin(h);
  if (int rc = check_cuda(h, cudaGetLastError(), "force kernels")) return rc;
  if (fused) { h->cur = 1 - h->cur; h->first_pass = false; }
  return 0;
}

// Per-step force error of the split path: both paths evaluate FC for the
// current state (the wall and pair histories are restored between and after
// them); returns max|F_split - F_fp64| over all components divided by
// max|F_fp64|.
int run_split_force_error(dem_handle* h, double* rel_err) {
  if (!h->have_state || !h->have_pairs) return set_err(h, DEM_ERR_STATE, "state or pair list missing");
  const size_t n = h->n, cm = h->dp.cmax, P = (size_t)host_pairs(h);
  const size_t b_fid = sizeof(int) * cm * n, b_pft = sizeof(double) * 3 * cm * n;
  const size_t b_hist = sizeof(double) * 3 * P;
  // both passes start from the same wall and pair histories (each pass
  // updates them in place)
  char* snap = (char*)stage_buffer(h, b_fid + b_pft + n + b_hist + 2 * P + 64);
  if (!snap) return set_err(h, DEM_ERR_CUDA, "cudaMalloc stage");
  char* s_live = snap + b_fid + b_pft;
  char* s_hist = s_live + n;
  char* s_flag = s_hist + b_hist;
  char* s_inflag = s_flag + P;
  auto save = [&]() {
    cudaMemcpyAsync(snap, h->wall_fid, b_fid, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(snap + b_fid, h->wall_pft, b_pft, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(s_live, h->wall_live, n, cudaMemcpyDeviceToDevice, h->stream);
    if (P) {
      cudaMemcpyAsync(s_hist, h->pft[h->pcur], b_hist, cudaMemcpyDeviceToDevice, h->stream);
      cudaMemcpyAsync(s_flag, h->pflag(), P, cudaMemcpyDeviceToDevice, h->stream);
      cudaMemcpyAsync(s_inflag, h->in_flag, P, cudaMemcpyDeviceToDevice, h->stream);
    }
  };
  auto restore = [&]() {
    cudaMemcpyAsync(h->wall_fid, snap, b_fid, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->wall_pft, snap + b_fid, b_pft, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->wall_live, s_live, n, cudaMemcpyDeviceToDevice, h->stream);
    if (P) {
      cudaMemcpyAsync(h->pft[h->pcur], s_hist, b_hist, cudaMemcpyDeviceToDevice, h->stream);
      cudaMemcpyAsync(h->pflag(), s_flag, P, cudaMemcpyDeviceToDevice, h->stream);
      cudaMemcpyAsync(h->in_flag, s_inflag, P, cudaMemcpyDeviceToDevice, h->stream);
    }
  };
  std::vector<double> f64(3 * n), f32(3 * n);
  h->dp.first_pass = 0;
  save();
  launch_force_kernels(h, 0, false);
  cudaMemcpyAsync(f64.data(), h->fc, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream);
  restore();
  launch_force_kernels(h, 0, true);
  cudaMemcpyAsync(f32.data(), h->fc, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream);
  restore();
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "force error")) return rc;
  double dmax = 0.0, fmax = 0.0;
  for (size_t k = 0; k < 3 * n; ++k) {
    dmax = std::max(dmax, std::fabs(f32[k] - f64[k]));
    fmax = std::max(fmax, std::fabs(f64[k]));
  }
  *rel_err = fmax > 0.0 ? dmax / fmax : dmax;
  return fetch_errors(h);
}

template <int INTG, bool B>
static void launch_integrate_t(dem_handle* h) {
  const int T = 256, G = (h->nl() + T - 1) / T;
  const int c = h->cur;
  k_integrate<INTG, B><<<G, T, 0, h->stream>>>(h->dp, h->bview(), h->pos4[c], h->vel4[c], h->omg4[c], h->state,
                                               h->fc, h->tow, h->acc_old, h->rot_acc_old, h->vslot);
  DEM_LAUNCH(h);
}

int run_cfnewvalues(dem_handle* h) {
  ProfScope ps(h, DEM_PROF_INTEGRATE);
  h->dp.first_pass = h->first_pass ? 1 : 0;
  const bool ab2 = h->dp.intg == DEM_INTG_AB2;
  if (h->batch()) ab2 ? launch_integrate_t<DEM_INTG_AB2, true>(h) : launch_integrate_t<DEM_INTG_EULER, true>(h);
  else ab2 ? launch_integrate_t<DEM_INTG_AB2, false>(h) : launch_integrate_t<DEM_INTG_EULER, false>(h);
  launch_skin(h);
  h->first_pass = false;
  return check_cuda(h, cudaGetLastError(), "k_integrate");
}

}  // namespace demb
