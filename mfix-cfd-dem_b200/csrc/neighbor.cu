// neighbor.cu -- pair-list build and history carry-over (K2).
//
// Replaces NEIGHBOUR (model/des/neighbour.f:21-126) with its
// DESGRID_NEIGH_BUILD (model/des/desgrid_mod.f:1002-1299) and ADD_PAIR
// (model/des/des_allocate_mod.f:555-567), serial build semantics:
//   * rows only for NORMAL particles; a NORMAL particle found in a ghost cell
//     is rogue: it is deleted (REMOVE_ROGUE_PARTICLES) and, as in the
//     reference where the shared do_exit flag stays set, every particle with a
//     larger index gets an empty row in that build;
//   * candidates are visited cell by cell in (lk, lj, li) stencil order,
//     each cell in ascending particle index; coarse grids (cell narrower than
//     2*FACTOR_RLM*MAX_RADIUS) scan only the nearer neighbour cell per axis;
//   * a candidate is kept when it is not the particle itself, not a NORMAL
//     particle of lower index, not NONEXISTENT, and
//     |x_i - x_j|^2 <= (FACTOR_RLM*(r_i + r_j))^2 in FP64.
// The list is built as count -> scan -> fill, so NEIGHBOR_INDEX / NEIGHBORS
// come out bit-identical to the serial reference.  PFT_NEIGHBOR is carried
// over by matching the neighbour id inside the particle's previous row
// (neighbour.f:77-117).  Finally the transpose (incoming pairs per particle,
// ascending owner) is built for the deterministic force gather.  On a
// single system without flow boundaries most builds filter a candidate list
// (pairs within the search radius plus a skin, made by an earlier scan)
// instead of scanning the grid, with the same exact test, so the rows are
// the scan's (section "candidate list" below).
#include "dem_internal.cuh"

namespace demb {

template <bool B>
__global__ void k_find_rogue(DevParams p0, BatchView bv, const int8_t* __restrict__ state,
                             const int* __restrict__ dg_pijk, DevErr* __restrict__ err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p0.n || state[i] != DEM_STATE_NORMAL) return;
  const DevParams& p = sysp<B>(p0, bv, i);
  if constexpr (B) {
    if (!bv.due[bv.sys_of[i]]) return;
  }
  int c = dg_pijk[i];
  int lic = dg_iof(p, c), ljc = dg_jof(p, c), lkc = dg_kof(p, c);
  if (lic < p.istart1 || lic > p.iend1 || ljc < p.jstart1 || ljc > p.jend1 ||
      lkc < p.kstart1 || lkc > p.kend1) {
    if constexpr (B) atomicMin(&bv.first_rogue[bv.sys_of[i]], i);
    else atomicMin(&err->first_rogue, i);
  }
}

__global__ void k_reset_rogue(int nsys, int* __restrict__ first_rogue) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nsys) first_rogue[s] = 0x7fffffff;
}

// DELETE_PARTICLE (mass_outflow_dem.f:241-300) for the rogue particles.
template <bool B>
__global__ void k_delete_rogue(DevParams p0, BatchView bv, int8_t* __restrict__ state,
                               const int* __restrict__ dg_pijk, double4* __restrict__ pos4,
                               double4* __restrict__ vel4, double4* __restrict__ omg4, double* __restrict__ fc,
                               double* __restrict__ tow, int* __restrict__ wall_fid, DevErr* __restrict__ err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p0.n || state[i] != DEM_STATE_NORMAL) return;
  const DevParams& p = sysp<B>(p0, bv, i);
  if constexpr (B) {
    if (!bv.due[bv.sys_of[i]]) return;
  }
  int c = dg_pijk[i];
  int lic = dg_iof(p, c), ljc = dg_jof(p, c), lkc = dg_kof(p, c);
  if (!(lic < p.istart1 || lic > p.iend1 || ljc < p.jstart1 || ljc > p.jend1 ||
        lkc < p.kstart1 || lkc > p.kend1)) return;
  if (!p.remove_rogue) { atomicOr(&err->flags, EF_ROGUE_FATAL); return; }
  pos4[i] = make_double4(0.0, 0.0, 0.0, 0.0);                         // DES_RADIUS = 0
  vel4[i] = make_double4(0.0, 0.0, 0.0, 3.4028234663852886e38);       // PMASS = HUGE(0.0)
  omg4[i] = make_double4(0.0, 0.0, 0.0, 0.0);                         // OMOI = 0
  for (int a = 0; a < 3; ++a) { fc[(size_t)a * p.n + i] = 0.0; tow[(size_t)a * p.n + i] = 0.0; }
  for (int s = 0; s < p.cmax; ++s) wall_fid[(size_t)i * p.cmax + s] = -1;
  state[i] = DEM_STATE_NONEXISTENT;
  atomicAdd(&err->rogue_removed, 1ull);
}

// Count and fill passes of the rows.
//
// Candidates come from the search-grid cells within the particle's reach
// FACTOR_RLM*(r + MAX_RADIUS); the search grid is at least as fine as the
// DES grid, so every pair the reference keeps is among the candidates.  A
// candidate is then tested exactly as the reference tests it: it must lie
// in the particle's DES-grid stencil (the coarse-grid reduction included),
// its periodic image is the one that stencil cell holds, and the FP64
// distance test is the reference's.  Each kept neighbour carries its
// stencil rank ((lk, lj, li) order); the row is sorted by (rank, index),
// which is the order of the reference's cell-by-cell scan.
// The search runs over a cell-sorted copy of the candidate data: sinfo[q] =
// (particle, DES cell as packed (i, j, k), state, search cell) and spos[q] =
// (x, y, z, r) in the order of the search-grid cell lists.  Thread q handles
// particle sinfo[q].x, so a warp holds spatially adjacent particles that scan
// the same cells, and every candidate read is a contiguous run of the sorted
// arrays.
//
// The count pass also keeps the first NSLOT neighbours of each particle as
// (rank << 27 | index) keys in nslot[q]; the fill pass writes them in row
// order, and rescans only the particles with longer rows.
template <bool B>
__global__ void k_sorted_copy(DevParams p0, BatchView bv, int n, const int* __restrict__ n_exist,
                              const int* __restrict__ flist, const double4* __restrict__ pos4,
                              const int8_t* __restrict__ state, const int* __restrict__ dg_pijk,
                              const int* __restrict__ fkey, double4* __restrict__ spos, float4* __restrict__ sposf,
                              int4* __restrict__ sinfo, int* __restrict__ qof) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n || q >= *n_exist) return;
  const int i = flist[q];
  if (qof) qof[i] = q;
  const DevParams& p = sysp<B>(p0, bv, i);
  const int c = dg_pijk[i];
  const double4 x = pos4[i];
  spos[q] = x;
  sposf[q] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)x.w);
  // the DES cell as (i, j, k), unpacked by every particle that scans this one
  sinfo[q] = make_int4(i, pack_ijk(dg_iof(p, c), dg_jof(p, c), dg_kof(p, c)), (int)state[i], fkey[i]);
}

// The scanning particle's frame for the candidate test.
struct NeighFrame {
  int cur;
  int rc[3], s1[3], e1[3], ncl[3], lo_off[3], hi_off[3];
  double4 cp;
  double fr;
  int glo[3], ghi[3];  // search cells within reach, per axis
  double inv_l[3];     // 1 / period length of the periodic axes
  float4 cpf;          // the particle's position and radius rounded to FP32
  float frf, lf[3], inv_lf[3];  // FACTOR_RLM and the periods in FP32 (0: not periodic)
  float tolf;          // rounding allowance of the FP32 pre-check (infinite: check off)
  bool wrap;           // the search range reaches a cell at a periodic boundary
};

// The part of the frame the exact test reads: the particle, its DES cell
// and stencil, and the periods.
__device__ __forceinline__ void neigh_frame_exact(const DevParams& p, const int4& me, const double4& cp,
                                                  NeighFrame& F) {
  F.cur = me.x;
  F.cp = cp;
  F.fr = p.factor_rlm;
  unpack_ijk(me.y, F.rc[0], F.rc[1], F.rc[2]);
  F.s1[0] = p.istart1; F.s1[1] = p.jstart1; F.s1[2] = p.kstart1;
  F.e1[0] = p.iend1; F.e1[1] = p.jend1; F.e1[2] = p.kend1;
  F.ncl[0] = p.iend1 - p.istart1 + 1; F.ncl[1] = p.jend1 - p.jstart1 + 1; F.ncl[2] = p.kend1 - p.kstart1 + 1;
  for (int ax = 0; ax < 3; ++ax) F.inv_l[ax] = (p.per[ax] && !(ax == 2 && p.no_k)) ? p.inv_L[ax] : 0.0;
  const double cpos[3] = {cp.x, cp.y, cp.z};
  const double mr = p.max_radius;
  for (int ax = 0; ax < 3; ++ax) {
    F.lo_off[ax] = 1; F.hi_off[ax] = 1;
    if (ax == 2 && p.no_k) { F.lo_off[2] = 0; F.hi_off[2] = 0; continue; }
    // the reference's stencil is the nearer 2 cells when the DES cells are
    // wider than the search diameter (desgrid_mod.f:1116-1152)
    const bool coarse = 1.0 > 2.0 * mr * F.fr * p.dg_inv[ax];
    if (coarse) {
      const double t = (cpos[ax] - p.dg_start[ax]) * p.dg_inv[ax];
      const double off = t - (double)(long long)floor(t);
      if (off >= 0.5) F.lo_off[ax] = 0; else F.hi_off[ax] = 0;
    }
  }
}

// The whole frame of a particle that scans candidates.
__device__ __forceinline__ void neigh_frame(const DevParams& p, const int4& me, const double4& cp, NeighFrame& F,
                                            double extra = 0.0) {
  neigh_frame_exact(p, me, cp, F);
  F.cpf = make_float4((float)cp.x, (float)cp.y, (float)cp.z, (float)cp.w);
  F.frf = (float)p.factor_rlm;
  // The FP32 pre-check's allowance.  For a neighbour (nearest-image distance
  // at most the search radius sr <= FACTOR_RLM*(r + MAX_RADIUS)) each
  // coordinate of the candidate is within sr of this particle's or of one
  // of its periodic images k*L, so the rounding error of each axis's FP32
  // separation -- the roundings of both coordinates, of the difference and
  // of the image shift -- is below 2^-24 (2|x| + 4|k|L + 3 sr), under
  // 2^-20 (|x| + sr + L) for |k| <= 4 (the wrap of every step keeps the
  // positions within one period of the domain); the sum over the axes
  // bounds the error of the distance.  A period below four search radii
  // could let FP32 pick another image: the check is off there.
  {
    const float srm = (float)(p.factor_rlm * (cp.w + p.max_radius) + extra) * 1.0001f;
    float tol = 0.f;
    bool off = false;
    for (int ax = 0; ax < 3; ++ax) {
      F.lf[ax] = F.inv_l[ax] != 0.0 ? (float)p.L[ax] : 0.f;
      F.inv_lf[ax] = (float)F.inv_l[ax];
      const float c = ax == 0 ? F.cpf.x : (ax == 1 ? F.cpf.y : F.cpf.z);
      tol += 0x1p-20f * (fabsf(c) + srm + F.lf[ax]);
      if (F.inv_l[ax] != 0.0 && p.L[ax] < 4.0 * (double)srm) off = true;
    }
    F.tolf = off ? INFINITY : tol;
  }
  // the search cells within reach FACTOR_RLM*(r + MAX_RADIUS) of the
  // particle, each once: per axis a range of cells, wrapped on a periodic
  // axis (the whole axis when the range covers it); a margin of 1e-4 of the
  // reach covers the rounding of the cell index
  const double cpos[3] = {cp.x, cp.y, cp.z};
  const double reach = F.fr * (cp.w + p.max_radius) + extra;
  F.wrap = false;
  for (int ax = 0; ax < 3; ++ax) {
    F.glo[ax] = 0; F.ghi[ax] = 0;
    if (ax == 2 && p.no_k) continue;
    const double t = (cpos[ax] - p.dg_start[ax]) * p.f_inv[ax], w = reach * p.f_inv[ax] * 1.0001;
    int lo = (int)floor(t - w) + 1, hi = (int)floor(t + w) + 1;
    if (p.per[ax]) {
      if (hi - lo + 1 >= p.fn[ax]) { lo = 1; hi = p.fn[ax]; }
      // Search cells 2..fn-1 of a periodic axis hold particles inside the
      // domain at least one cell from its ends (a particle outside is
      // binned to cell 1 or fn).  When the range lies within them, the
      // particle and every candidate are such, and a candidate's image
      // within reach is its own position: another image would put the
      // particle within reach of a domain end, and the range into cell 1 or
      // fn.  Only a range that reaches cell 1 or fn needs the image shift.
      if (lo <= 1 || hi >= p.fn[ax]) F.wrap = true;
    } else {
      lo = max(lo, 0);
      hi = min(hi, p.fn[ax] + 1);
    }
    F.glo[ax] = lo;
    F.ghi[ax] = hi;
  }
}

__device__ __forceinline__ int search_wrap(const DevParams& p, int g, int ax) {
  if (!p.per[ax] || (ax == 2 && p.no_k)) return g;
  return g < 1 ? g + p.fn[ax] : (g > p.fn[ax] ? g - p.fn[ax] : g);
}

// Calls run(qs, qe) for each run [qs, qe) of the sorted copy that holds the
// frame's candidates: one per (i, k) column of the range, two when the y
// range wraps (y is the fastest key, so a column's cells are contiguous).
// HALF keeps only the candidates after the particle's place q0 in the copy
// (in search cell c_own): a run that ends before c_own is skipped unread.
template <bool HALF, class Run>
__device__ __forceinline__ void for_runs(const DevParams& p, const NeighFrame& F, const int* __restrict__ fstart,
                                         int q0, int c_own, Run&& run) {
  int ylo0 = F.glo[1], yhi0 = F.ghi[1], ylo1 = 0, yhi1 = -1;
  if (p.per[1] && (F.glo[1] < 1 || F.ghi[1] > p.fn[1])) {
    if (F.glo[1] < 1) { ylo0 = F.glo[1] + p.fn[1]; yhi0 = p.fn[1]; ylo1 = 1; yhi1 = F.ghi[1]; }
    else { ylo0 = F.glo[1]; yhi0 = p.fn[1]; ylo1 = 1; yhi1 = F.ghi[1] - p.fn[1]; }
  }
  for (int gk = F.glo[2]; gk <= F.ghi[2]; ++gk) {
    const int bk = p.fcell_off + search_wrap(p, gk, 2) * p.fc2;
    for (int gi = F.glo[0]; gi <= F.ghi[0]; ++gi) {
      const int base = bk + search_wrap(p, gi, 0) * p.fc1;
#pragma unroll
      for (int sg = 0; sg < 2; ++sg) {
        const int lo = sg ? ylo1 : ylo0, hi = sg ? yhi1 : yhi0;
        if (hi < lo) continue;
        const int c0 = base + lo, c1 = base + hi;
        int qs;
        if (HALF) {
          if (c1 < c_own) continue;
          qs = c0 > c_own ? fstart[c0] : q0 + 1;
        } else {
          qs = fstart[c0];
        }
        run(qs, fstart[c1 + 1]);
      }
    }
  }
}

// The runs of for_runs<false> by number, for scans that share them out:
// their count, and run r (column r / rpc of the range in (k, i) order, y
// segment r % rpc).
__device__ __forceinline__ int runs_per_col(const DevParams& p, const NeighFrame& F) {
  return (p.per[1] && (F.glo[1] < 1 || F.ghi[1] > p.fn[1])) ? 2 : 1;
}
__device__ __forceinline__ int run_count(const DevParams& p, const NeighFrame& F) {
  return (F.ghi[2] - F.glo[2] + 1) * (F.ghi[0] - F.glo[0] + 1) * runs_per_col(p, F);
}
__device__ __forceinline__ void run_at(const DevParams& p, const NeighFrame& F, const int* __restrict__ fstart,
                                       int r, int& qs, int& qe) {
  const int rpc = runs_per_col(p, F);
  const int col = r / rpc, sub = r % rpc;
  const int ni = F.ghi[0] - F.glo[0] + 1;
  const int gk = F.glo[2] + col / ni, gi = F.glo[0] + col % ni;
  const int base = p.fcell_off + search_wrap(p, gk, 2) * p.fc2 + search_wrap(p, gi, 0) * p.fc1;
  int lo = F.glo[1], hi = F.ghi[1];
  if (rpc == 2) {
    if (F.glo[1] < 1) { if (sub == 0) { lo = F.glo[1] + p.fn[1]; hi = p.fn[1]; } else { lo = 1; hi = F.ghi[1]; } }
    else { if (sub == 0) { lo = F.glo[1]; hi = p.fn[1]; } else { lo = 1; hi = F.ghi[1] - p.fn[1]; } }
  }
  qs = fstart[base + lo];
  qe = fstart[base + hi + 1];
}

// The FP32 part of a frame as three float4: a = the particle's position
// and radius, b = (FACTOR_RLM, allowance, period x, period y), c = (period
// z, 1/period x, y, z); 0 for an axis that is not periodic.
struct PreFrame {
  float4 a, b, c;
};
__device__ __forceinline__ PreFrame pre_frame(const NeighFrame& F) {
  return {F.cpf, make_float4(F.frf, F.tolf, F.lf[0], F.lf[1]), make_float4(F.lf[2], F.inv_lf[0], F.inv_lf[1], F.inv_lf[2])};
}

// The conservative FP32 pre-check of a candidate at f (see neigh_exact):
// false only for a candidate the exact test rejects.  Most candidates are
// far out of reach, and FP32 copies of the two positions show it: the FP32
// nearest-image distance less the frame's rounding allowance is a lower
// bound of the exact distance for any neighbour, so a candidate beyond the
// search radius by more than the allowance (and a relative 2e-5 for the
// FP32 radius, squares and sum) is no neighbour under any test below.  On
// an axis that is not periodic the image shift is 0 * 0.  A NaN compares
// false and falls through to the exact test.
__device__ __forceinline__ bool pre_test(const PreFrame& G, const float4 f) {
  float e0 = G.a.x - f.x, e1 = G.a.y - f.y, e2 = G.a.z - f.z;
  e0 = e0 - rintf(e0 * G.c.y) * G.b.z;
  e1 = e1 - rintf(e1 * G.c.z) * G.b.w;
  e2 = e2 - rintf(e2 * G.c.w) * G.c.x;
  const float sr = G.b.x * (G.a.w + f.w) + G.b.y;
  return !(e0 * e0 + e1 * e1 + e2 * e2 > sr * sr * 1.00002f);
}
// The same test for a frame whose range needs no image shift (wrap false):
// the separation is the difference of the two positions.  Fused
// multiply-adds round less than the separate operations the margin allows
// for.
__device__ __forceinline__ bool pre_direct(const PreFrame& G, const float4 f) {
  const float e0 = G.a.x - f.x, e1 = G.a.y - f.y, e2 = G.a.z - f.z;
  const float d2 = __fmaf_rn(e2, e2, __fmaf_rn(e1, e1, __fmul_rn(e0, e0)));
  const float sr = __fmaf_rn(G.b.x, G.a.w + f.w, G.b.y);
  return !(d2 > sr * sr * 1.00002f);
}

// Candidate q of the sorted copy (past the pre-check): a neighbour of the
// frame's particle when it is a later or non-NORMAL particle (the half list
// of DESGRID_NEIGH_BUILD), in the reference's DES-grid stencil and within
// FACTOR_RLM*(r_l + r_i); its row key (stencil rank << 27 | index) through
// *key.
__device__ __forceinline__ bool neigh_exact(const DevParams& p, const NeighFrame& F, const int4* __restrict__ sinfo,
                                            const double4* __restrict__ spos, int q, uint32_t* key) {
  const int4 o = sinfo[q];
  const int nb = o.x;
  if (nb == F.cur) return false;
  if (nb < F.cur && o.z == DEM_STATE_NORMAL) return false;
  if (o.z == DEM_STATE_NONEXISTENT) return false;
  const double4 np_ = spos[q];
  const double srad = F.fr * (F.cp.w + np_.w);
  {
    // most candidates are out of reach: the nearest periodic image is at
    // least as close as the one the stencil picks, so a candidate whose
    // nearest image is farther than the search radius (with a margin for
    // rounding) cannot be a neighbour
    double e[3] = {F.cp.x - np_.x, F.cp.y - np_.y, F.cp.z - np_.z};
    for (int ax = 0; ax < 3; ++ax)
      if (F.inv_l[ax] != 0.0) e[ax] = e[ax] - p.L[ax] * rint(e[ax] * F.inv_l[ax]);
    if (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] > srad * srad * (1.0 + 1e-9)) return false;
  }
  // position of the neighbour's DES cell in the reference stencil
  int nc[3];
  unpack_ijk(o.y, nc[0], nc[1], nc[2]);
  int rel[3] = {0, 0, 0};
  double sh[3] = {0.0, 0.0, 0.0};
  for (int ax = 0; ax < 3; ++ax) {
    int r = nc[ax] - F.rc[ax];
    if (p.per[ax] && !(ax == 2 && p.no_k)) {
      if (r > 1) r -= F.ncl[ax];
      else if (r < -1) r += F.ncl[ax];
      const int l = F.rc[ax] + r;
      if (l < F.s1[ax]) sh[ax] = -p.L[ax];
      else if (l > F.e1[ax]) sh[ax] = p.L[ax];
    }
    if (r < -F.lo_off[ax] || r > F.hi_off[ax]) return false;
    rel[ax] = r;
  }
  double px = np_.x, py = np_.y, pz = np_.z;
  if (sh[0] != 0.0) px = px + sh[0];
  if (sh[1] != 0.0) py = py + sh[1];
  if (sh[2] != 0.0) pz = pz + sh[2];
  const double d0 = F.cp.x - px, d1 = F.cp.y - py, d2 = F.cp.z - pz;
  const double dd = d0 * d0 + d1 * d1 + d2 * d2;
  if (dd > srad * srad) return false;
  const int rank = ((rel[2] + 1) * 3 + (rel[1] + 1)) * 3 + (rel[0] + 1);
  *key = ((uint32_t)rank << 27) | (uint32_t)nb;
  return true;
}

constexpr int NSURV = 24;  // pre-checked candidates buffered per thread

// Count pass of the pair build, a half scan: each particle of the sorted
// copy tests only the candidates after it in the copy, so each pair of
// particles within reach of one another is examined once, by the one that
// comes first.  (Each is in the other's search range: a neighbour lies
// within FACTOR_RLM*(r_l + r_i) of the particle, inside the reach
// FACTOR_RLM*(r + MAX_RADIUS) of either.)  The pair goes to the row of its
// owner -- the NORMAL particle of lower index, or the NORMAL one of a
// NORMAL / non-NORMAL pair, as DESGRID_NEIGH_BUILD keeps it -- and is given
// the exact test in the owner's FP64 frame, so the row is the full scan's.
// The owner's count is an atomic add; its first NSLOT keys go to its slots
// nslot[owner] in the order found, and a row that grows past NSLOT enters
// the long-row list (long_rows[0 .. long_rows[n]), sorted-copy places) once.
// Candidates that pass the FP32 pre-check (a few per row) wait in this
// thread's column of s_surv and get the exact test in a second loop, so the
// long exact path runs with every lane holding work instead of one lane at
// a time inside the candidate scan.
template <bool B>
__global__ void __launch_bounds__(128, 8)
k_neigh_count(DevParams p0, BatchView bv, const int* __restrict__ n_exist, const double4* __restrict__ spos,
              const float4* __restrict__ sposf, const int4* __restrict__ sinfo, const int* __restrict__ fstart,
              const DevErr* __restrict__ err, int* __restrict__ row_cnt, uint32_t* __restrict__ nslot,
              int* __restrict__ long_rows, const int* __restrict__ skip) {
  __shared__ int s_surv[NSURV * 128];
  if (skip && *skip) return;  // this build filters the candidate list instead
  const int q0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (q0 >= p0.n || q0 >= *n_exist) return;
  const int4 me = sinfo[q0];
  if (me.z == DEM_STATE_NONEXISTENT) return;
  const int cur = me.x;
  const DevParams& p = sysp<B>(p0, bv, cur);
  const int first_rogue = B ? bv.first_rogue[bv.sys_of[cur]] : err->first_rogue;
  const bool me_normal = me.z == DEM_STATE_NORMAL;
  NeighFrame F;
  neigh_frame(p, me, spos[q0], F);
  auto exact = [&](int q) {
    const int4 o = sinfo[q];
    if (o.z == DEM_STATE_NONEXISTENT) return;
    const bool o_normal = o.z == DEM_STATE_NORMAL;
    bool mine;
    if (me_normal && o_normal) mine = cur < o.x;
    else if (me_normal || o_normal) mine = me_normal;
    else return;  // two non-NORMAL particles: no row holds the pair
    uint32_t key;
    int oq, oi;
    if (mine) {
      if (cur >= first_rogue || !neigh_exact(p, F, sinfo, spos, q, &key)) return;
      oq = q0; oi = cur;
    } else {
      if (o.x >= first_rogue) return;
      NeighFrame Fo;
      neigh_frame_exact(p, o, spos[q], Fo);
      if (!neigh_exact(p, Fo, sinfo, spos, q0, &key)) return;
      oq = q; oi = o.x;
    }
    const int s = atomicAdd(&row_cnt[oi], 1);
    if (s < NSLOT) nslot[(size_t)oi * NSLOT + s] = key;
    else if (s == NSLOT) {
      const int t = atomicAdd(&long_rows[p0.n], 1);
      if (t < p0.n) long_rows[t] = oq;
    }
  };
  int ns = 0;
  auto flush = [&]() {
    for (int s = 0; s < ns; ++s) exact(s_surv[s * blockDim.x + threadIdx.x]);
    ns = 0;
  };
  const PreFrame G = pre_frame(F);
  for_runs<true>(p, F, fstart, q0, me.w, [&](int qs, int qe) {
    if (F.wrap) {
      for (int q = qs; q < qe; ++q) {
        if (!pre_test(G, sposf[q])) continue;
        s_surv[ns * blockDim.x + threadIdx.x] = q;
        if (++ns == NSURV) flush();
      }
    } else {
      for (int q = qs; q < qe; ++q) {
        if (!pre_direct(G, sposf[q])) continue;
        s_surv[ns * blockDim.x + threadIdx.x] = q;
        if (++ns == NSURV) flush();
      }
    }
  });
  flush();
}

// Writes the kept <= R keys of slot at start + (number of smaller keys),
// the keys held in registers.
template <int R>
__device__ __forceinline__ void place_keys(const uint32_t* __restrict__ slot, int kept, long long start,
                                           long long cap, int i, int* __restrict__ nbrs, int* __restrict__ owner) {
  uint32_t k[R];
#pragma unroll
  for (int c = 0; c < R; ++c) k[c] = c < kept ? slot[c] : 0xffffffffu;
#pragma unroll
  for (int c = 0; c < R; ++c) {
    if (c < kept) {
      int r = 0;
#pragma unroll
      for (int d = 0; d < R; ++d) r += k[d] < k[c];
      const long long s = start + r;
      if (s < cap) { nbrs[s] = (int)(k[c] & 0x7ffffffu); owner[s] = i; }
    }
  }
}

// ---- candidate list (single-system handles) --------------------------------
// Between two builds of the list, a build filters it instead of scanning the
// grid.  The list holds, for each particle's row, every particle within the
// search radius FACTOR_RLM*(r_l + r_i) plus the skin at the time it was
// built (nearest image, the half-list rules of DESGRID_NEIGH_BUILD, no
// stencil).  A pair in the reference's list now is within the search radius
// now, and each of its particles has moved at most the displacement bound
// since the list was built, so while twice that bound stays within the skin
// the pair is in the list.  The filter gives each entry the exact test of
// the scan (neigh_exact, in the owner's frame: stencil, periodic image, FP64
// distance, stencil rank), so the rows are the scan's.  The choice is made
// on the device at the start of each build (k_cand_decide), so a captured
// period holds both paths: the count pass and the list build return at once
// when the list is filtered, the filter when it is not.

// A list that expires before any build filtered it (particles moving fast)
// cost two scans for nothing: the next CAND_COOL builds make none.
constexpr int CAND_COOL = 4;
__global__ void k_cand_decide(CandState* __restrict__ cs, DevErr* __restrict__ err, double half_skin) {
  if (cs->have && cs->disp <= half_skin) {
    cs->ok = 1;
    cs->build = 0;
    cs->uses += 1;
    err->cand_filtered += 1;
    return;
  }
  cs->ok = 0;
  if (cs->have && cs->uses == 0) cs->cool = CAND_COOL;
  if (cs->cool > 0) {
    cs->cool -= 1;
    cs->build = 0;
  } else {
    cs->build = 1;
  }
  cs->have = 0;
  cs->uses = 0;
}

// The rows from the candidate list: row count, the first NSLOT keys in the
// slots, longer rows into the long-row list (as the count pass leaves them).
__global__ void __launch_bounds__(128)
k_cand_filter(DevParams p, const int* __restrict__ n_exist, const double4* __restrict__ spos,
              const int4* __restrict__ sinfo, const int* __restrict__ qof, const DevErr* __restrict__ err,
              const int* __restrict__ cand_end, const int* __restrict__ cand_nb, const CandState* __restrict__ cs,
              int* __restrict__ row_cnt, uint32_t* __restrict__ nslot, int* __restrict__ long_rows) {
  if (!cs->ok) return;
  const int q0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (q0 >= p.n || q0 >= *n_exist) return;
  const int4 me = sinfo[q0];
  const int cur = me.x;
  if (me.z != DEM_STATE_NORMAL || cur >= err->first_rogue) return;
  NeighFrame F;
  neigh_frame_exact(p, me, spos[q0], F);
  const int s = cur ? cand_end[cur - 1] : 0, e = cand_end[cur];
  int cnt = 0;
  for (int c = s; c < e; ++c) {
    const int q = qof[cand_nb[c]];
    if (q < 0) continue;  // not in the sorted copy: NONEXISTENT
    uint32_t key;
    if (!neigh_exact(p, F, sinfo, spos, q, &key)) continue;
    if (cnt < NSLOT) nslot[(size_t)cur * NSLOT + cnt] = key;
    ++cnt;
  }
  row_cnt[cur] = cnt;
  if (cnt > NSLOT) {
    const int t = atomicAdd(&long_rows[p.n], 1);
    if (t < p.n) long_rows[t] = q0;
  }
}

// Count (FILL = false) and fill pass of a list build (when k_cand_decide
// asks for one): the half scan of
// k_neigh_count over a reach widened by the skin, each pair within the
// search radius plus the skin of its nearest image entered in its owner's
// row (any NORMAL owner: the rogue limit of a build is applied when the
// list is filtered).  The fill places entries at cand_start[owner] + an
// atomic slot; their order within a row does not matter.
template <bool FILL>
__global__ void __launch_bounds__(128, 8)
k_cand_build(DevParams p, const int* __restrict__ n_exist, const double4* __restrict__ spos,
             const float4* __restrict__ sposf, const int4* __restrict__ sinfo, const int* __restrict__ fstart,
             const CandState* __restrict__ cs, double skin, int* __restrict__ cand_cnt, int* __restrict__ cand_fill,
             const int* __restrict__ cand_start, int* __restrict__ cand_nb, long long cap) {
  __shared__ int s_surv[NSURV * 128];
  if (!cs->build) return;
  const int q0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (q0 >= p.n || q0 >= *n_exist) return;
  const int4 me = sinfo[q0];
  if (me.z == DEM_STATE_NONEXISTENT) return;
  const int cur = me.x;
  const bool me_normal = me.z == DEM_STATE_NORMAL;
  NeighFrame F;
  neigh_frame(p, me, spos[q0], F, skin);
  PreFrame G = pre_frame(F);
  G.b.y = __fadd_ru(G.b.y, __double2float_ru(skin));  // the allowance also covers the skin
  auto enter = [&](int q) {
    const int4 o = sinfo[q];
    if (o.z == DEM_STATE_NONEXISTENT) return;
    const bool o_normal = o.z == DEM_STATE_NORMAL;
    bool mine;
    if (me_normal && o_normal) mine = cur < o.x;
    else if (me_normal || o_normal) mine = me_normal;
    else return;
    const double4 b = spos[q];
    double e[3] = {F.cp.x - b.x, F.cp.y - b.y, F.cp.z - b.z};
    for (int ax = 0; ax < 3; ++ax)
      if (F.inv_l[ax] != 0.0) e[ax] = e[ax] - p.L[ax] * rint(e[ax] * F.inv_l[ax]);
    const double r = F.fr * (F.cp.w + b.w) + skin;
    if (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] > r * r * (1.0 + 1e-9)) return;
    const int oi = mine ? cur : o.x;
    if (!FILL) {
      atomicAdd(&cand_cnt[oi], 1);
    } else {
      const long long at = (long long)cand_start[oi] + atomicAdd(&cand_fill[oi], 1);
      if (at < cap) cand_nb[at] = mine ? o.x : cur;
    }
  };
  int ns = 0;
  auto flush = [&]() {
    for (int s = 0; s < ns; ++s) enter(s_surv[s * blockDim.x + threadIdx.x]);
    ns = 0;
  };
  for_runs<true>(p, F, fstart, q0, me.w, [&](int qs, int qe) {
    if (F.wrap) {
      for (int q = qs; q < qe; ++q) {
        if (!pre_test(G, sposf[q])) continue;
        s_surv[ns * blockDim.x + threadIdx.x] = q;
        if (++ns == NSURV) flush();
      }
    } else {
      for (int q = qs; q < qe; ++q) {
        if (!pre_direct(G, sposf[q])) continue;
        s_surv[ns * blockDim.x + threadIdx.x] = q;
        if (++ns == NSURV) flush();
      }
    }
  });
  flush();
}

// The list's row ends from the counts and the scan; it is complete when its
// entries fit the capacity, and the displacement bound restarts.
__global__ void k_cand_commit(int n, const int* __restrict__ cand_cnt, const int* __restrict__ cand_start,
                              int* __restrict__ cand_end, CandState* __restrict__ cs, DevErr* __restrict__ err,
                              long long cap) {
  if (!cs->build) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) cand_end[i] = cand_start[i] + cand_cnt[i];
  if (i == 0) {
    const int total = cand_start[n];
    cs->total = total;
    cs->have = (long long)total <= cap ? 1 : 0;
    if (!cs->have) cs->cool = CAND_COOL;  // no retry at every build
    else err->cand_lists += 1;
    cs->disp = 0.0;
  }
}

// Fill pass of the rows the count pass kept whole (at most NSLOT
// neighbours, in the order found), a thread per particle: each key goes to
// the place given by the number of smaller keys (the keys of a row are
// distinct), which is (rank, index) order.  Consecutive threads write
// consecutive rows.
template <bool B>
__global__ void k_fill_kept(int n, BatchView bv, const int* __restrict__ row_cnt, int* __restrict__ row_se,
                            int* __restrict__ nbrs, int* __restrict__ owner, const uint32_t* __restrict__ nslot,
                            long long cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if constexpr (B) {
    if (!bv.due[bv.sys_of[i]]) return;
  }
  const int kept = row_cnt[i];
  if (kept == 0 || kept > NSLOT) return;
  const long long start = min((long long)row_se[i], cap);
  const uint32_t* slot = nslot + (size_t)i * NSLOT;
  if (kept <= NSLOT / 2) place_keys<NSLOT / 2>(slot, kept, start, cap, i, nbrs, owner);
  else place_keys<NSLOT>(slot, kept, start, cap, i, nbrs, owner);
  row_se[i] = (int)min(start + kept, cap);   // start -> end pointer
}

// Fill pass of the rows longer than NSLOT (the long-row list), a warp per
// row: the lanes share out the runs of the particle's candidates (a run per
// lane) for a full rescan, collect the row's keys in shared memory and write each key
// at the place given by the number of smaller keys, which is (rank, index)
// order.  A row of more than LONG_KCAP neighbours is written by one lane,
// inserting each neighbour into the row kept sorted.  Warps stride over the
// list.
constexpr int LONG_KCAP = 128;
template <bool B>
__global__ void __launch_bounds__(128)
k_fill_long(DevParams p0, BatchView bv, const double4* __restrict__ spos, const float4* __restrict__ sposf,
            const int4* __restrict__ sinfo, const int* __restrict__ fstart, const int* __restrict__ row_cnt,
            int* __restrict__ row_se, int* __restrict__ nbrs, uint8_t* __restrict__ rank_buf,
            int* __restrict__ owner, const int* __restrict__ long_rows, long long cap) {
  __shared__ uint32_t s_key[4][LONG_KCAP];
  __shared__ int s_n[4];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nl = min(long_rows[p0.n], p0.n);
  for (int t = blockIdx.x * 4 + w; t < nl; t += gridDim.x * 4) {
    const int q0 = long_rows[t];
    const int4 me = sinfo[q0];
    const int cur = me.x;
    const DevParams& p = sysp<B>(p0, bv, cur);
    const long long start = min((long long)row_se[cur], cap);
    NeighFrame F;
    neigh_frame(p, me, spos[q0], F);
    const PreFrame G = pre_frame(F);
    if (row_cnt[cur] <= LONG_KCAP) {
      if (lane == 0) s_n[w] = 0;
      __syncwarp();
      const int nr = run_count(p, F);
      for (int r = lane; r < nr; r += 32) {
        int qs, qe;
        run_at(p, F, fstart, r, qs, qe);
        for (int q = qs; q < qe; ++q) {
          uint32_t key;
          if (!pre_test(G, sposf[q]) || !neigh_exact(p, F, sinfo, spos, q, &key)) continue;
          const int c = atomicAdd(&s_n[w], 1);
          if (c < LONG_KCAP) s_key[w][c] = key;
        }
      }
      __syncwarp();
      const int m = min(s_n[w], LONG_KCAP);
      for (int c = lane; c < m; c += 32) {
        const uint32_t kc = s_key[w][c];
        int r = 0;
        for (int d = 0; d < m; ++d) r += s_key[w][d] < kc;
        const long long sl = start + r;
        if (sl < cap) { nbrs[sl] = (int)(kc & 0x7ffffffu); owner[sl] = cur; }
      }
      if (lane == 0) row_se[cur] = (int)min(start + m, cap);   // start -> end pointer
    } else if (lane == 0) {
      int cnt = 0;
      for_runs<false>(p, F, fstart, q0, me.w, [&](int qs, int qe) {
        for (int q = qs; q < qe; ++q) {
          uint32_t key;
          if (!pre_test(G, sposf[q]) || !neigh_exact(p, F, sinfo, spos, q, &key)) continue;
          const int rank = (int)(key >> 27), nb = (int)(key & 0x7ffffffu);
          const long long sl = start + cnt;
          if (sl < cap) {
            long long b = sl - 1;
            while (b >= start) {
              const int rb = rank_buf[b];
              if (rb < rank || (rb == rank && nbrs[b] < nb)) break;
              nbrs[b + 1] = nbrs[b];
              rank_buf[b + 1] = (uint8_t)rb;
              --b;
            }
            nbrs[b + 1] = nb;
            rank_buf[b + 1] = (uint8_t)rank;
            owner[sl] = cur;
          }
          ++cnt;
        }
      });
      row_se[cur] = (int)min(start + cnt, cap);   // start -> end pointer
    }
    __syncwarp();
  }
}

// Rows of batch systems that do not rebuild now: the count pass takes the
// length of the particle's current row, the fill pass copies the row.  The
// current rows end at n_old, the extent of the build that made them: a
// particle past it has none (a system placed there since is built now, and
// the slots between systems' ranges belong to none).
template <bool FILL>
__global__ void k_keep_rows(int n, int n_old, BatchView bv, const int* __restrict__ old_end,
                            const int* __restrict__ old_nbrs, int* __restrict__ row_cnt, int* __restrict__ row_se,
                            int* __restrict__ nbrs, int* __restrict__ owner, long long cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || i >= n_old || bv.due[bv.sys_of[i]]) return;
  const int s = i ? old_end[i - 1] : 0, e = old_end[i];
  if (!FILL) { row_cnt[i] = e - s; return; }
  const long long start = row_se[i];
  for (int c = s; c < e; ++c) {
    const long long slot = start + (c - s);
    if (slot < cap) { nbrs[slot] = old_nbrs[c]; owner[slot] = i; }
  }
  row_se[i] = (int)min(start + (e - s), cap);
}

// Gap of a pair at a build: |x_i - x_l| - (r_l + r_i), less a margin of
// 1e-9 (r_l + r_i) for the rounding of the distance, rounded down to float;
// -1 for a pair with a NONEXISTENT particle.
template <bool B>
__device__ __forceinline__ float pair_gap(const DevParams& p0, const BatchView& bv, int ll, int i,
                                          const double4* __restrict__ pos4, const int8_t* __restrict__ state) {
  if (state[ll] == DEM_STATE_NONEXISTENT || state[i] == DEM_STATE_NONEXISTENT) return -1.0f;
  const DevParams& p = sysp<B>(p0, bv, ll);
  const double4 a = pos4[ll], b = pos4[i];
  const double xl[3] = {a.x, a.y, a.z}, xi[3] = {b.x, b.y, b.z};
  double d2 = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double pj = xi[c];
    const double s = periodic_shift(p, c, pj - xl[c]);
    if (s != 0.0) pj = pj + s;
    const double d = pj - xl[c];
    d2 += d * d;
  }
  const double r_lm = a.w + b.w;
  return __double2float_rd(sqrt(d2) - r_lm - 1e-9 * r_lm);
}

// neighbour.f:77-117: history of each new pair from the same neighbour id in
// the owner's previous row, zero when the pair is new.  A thread per pair of
// the new list (its owner from pair_owner); a batch system built for the
// first time (due = 2) takes no history from its region.  The same pass sets
// the pair's gap (pair_gap) and restarts the displacement bound.
template <bool B>
__global__ void k_remap(DevParams p0, BatchView bv, const int* __restrict__ d_np, long long cap,
                        const int* __restrict__ nbrs, const int* __restrict__ owner,
                        const int* __restrict__ old_end, const int* __restrict__ old_nbrs,
                        const double* __restrict__ old_pft, double* __restrict__ pft, uint8_t* __restrict__ pflag,
                        int have_old, const double4* __restrict__ pos4, const int8_t* __restrict__ state,
                        float* __restrict__ pgap, double* __restrict__ skin) {
  const long long np = min((long long)*d_np, cap), stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t0 == 0) skin[0] = 0.0;
  for (long long cc = t0; cc < np; cc += stride) {
    const int ll = owner[cc], nb = nbrs[cc];
    bool carry = have_old != 0;
    if constexpr (B) {
      if (bv.due[bv.sys_of[ll]] == 2) carry = false;
    }
    double a = 0.0, b = 0.0, c = 0.0;
    if (carry) {
      const int so = ll ? old_end[ll - 1] : 0, eo = old_end[ll];
      for (int co = so; co < eo; ++co) {
        if (old_nbrs[co] == nb) {
          a = old_pft[3 * (size_t)co]; b = old_pft[3 * (size_t)co + 1]; c = old_pft[3 * (size_t)co + 2];
          break;
        }
      }
    }
    pft[3 * cc] = a; pft[3 * cc + 1] = b; pft[3 * cc + 2] = c;
    pflag[cc] = (a != 0.0 || b != 0.0 || c != 0.0) ? PF_HIST : 0;
    pgap[cc] = pair_gap<B>(p0, bv, ll, nb, pos4, state);
  }
}

// PF_HIST bits of a pair list whose history was set from the host.
__global__ void k_hist_flags(const int* __restrict__ d_np, const double* __restrict__ pft,
                             uint8_t* __restrict__ pflag) {
  const long long np = *d_np, stride = (long long)gridDim.x * blockDim.x;
  for (long long cc = (long long)blockIdx.x * blockDim.x + threadIdx.x; cc < np; cc += stride) {
    const double* q = pft + 3 * cc;
    pflag[cc] = (q[0] != 0.0 || q[1] != 0.0 || q[2] != 0.0) ? PF_HIST : 0;
  }
}



void set_hist_flags(dem_handle* h) {
  const int T = 256;
  k_hist_flags<<<pair_grid(h, T), T, 0, h->stream>>>(h->d_np, h->pft[h->pcur], h->pflag());
  DEM_LAUNCH(h);
}

__global__ void k_set_int(int* __restrict__ p, int v) { *p = v; }

// Keeps every pair-indexed kernel inside the allocation when a build needed
// more than the capacity (only possible inside a captured step, which cannot
// grow the arrays); the overflow is reported as DEM_ERR_PAIR_OVERFLOW.
__global__ void k_clamp_np(int* __restrict__ d_np, long long cap, DevErr* __restrict__ err) {
  if (*d_np > cap) { *d_np = (int)cap; atomicOr(&err->flags, EF_PAIR_CAP); }
}

__global__ void k_in_count(const int* __restrict__ d_np, const int* __restrict__ nbrs, int* __restrict__ in_cnt) {
  const long long np = *d_np, stride = (long long)gridDim.x * blockDim.x;
  for (long long cc = (long long)blockIdx.x * blockDim.x + threadIdx.x; cc < np; cc += stride)
    atomicAdd(&in_cnt[nbrs[cc]], 1);
}

__global__ void k_in_fill(const int* __restrict__ d_np, const int* __restrict__ nbrs, const int* __restrict__ owner,
                          const int* __restrict__ in_start, int* __restrict__ in_fill, int2* __restrict__ in_pair) {
  const long long np = *d_np, stride = (long long)gridDim.x * blockDim.x;
  for (long long cc = (long long)blockIdx.x * blockDim.x + threadIdx.x; cc < np; cc += stride) {
    const int j = nbrs[cc];
    const int slot = atomicAdd(&in_fill[j], 1);
    in_pair[in_start[j] + slot] = make_int2(owner[cc], (int)cc);
  }
}

// incoming pairs of each particle in ascending pair index (= owner order);
// each pair's slot in the list (in_pos) and a cleared contact flag of the
// slot (in_flag: no pair of a new list is in contact before its first force
// pass)
__global__ void k_in_sort(int n, const int* __restrict__ in_start, int2* __restrict__ in_pair,
                          int* __restrict__ in_pos, uint8_t* __restrict__ in_flag) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int s = in_start[j], e = in_start[j + 1], m = e - s;
  constexpr int R = 16;  // lists up to R long are sorted in registers
  if (m <= R) {
    // each entry goes to the place given by the number of smaller pair
    // indices (distinct within a list)
    int2 v[R];
#pragma unroll
    for (int c = 0; c < R; ++c) v[c] = c < m ? in_pair[s + c] : make_int2(0, 0x7fffffff);
#pragma unroll
    for (int c = 0; c < R; ++c) {
      if (c < m) {
        int r = 0;
#pragma unroll
        for (int d = 0; d < R; ++d) r += v[d].y < v[c].y;
        in_pair[s + r] = v[c];
        in_pos[v[c].y] = s + r;
        in_flag[s + r] = 0;
      }
    }
    return;
  }
  for (int a = s + 1; a < e; ++a) {
    int2 v = in_pair[a];
    int b = a - 1;
    while (b >= s && in_pair[b].y > v.y) { in_pair[b + 1] = in_pair[b]; --b; }
    in_pair[b + 1] = v;
  }
  for (int a = s; a < e; ++a) {
    in_pos[in_pair[a].y] = a;
    in_flag[a] = 0;
  }
}

// Transpose of the current list (buffer nb, pair count in d_np): incoming
// pairs of every particle in ascending owner order.
int build_transpose(dem_handle* h, int nb) {
  const int n = h->nl();
  const int T = 256, B = (n + T - 1) / T;
  const unsigned BP = pair_grid(h, T);
  if (int rc = check_cuda(h, cudaMemsetAsync(h->in_cnt, 0, sizeof(int) * n, h->stream), "memset")) return rc;
  k_in_count<<<BP, T, 0, h->stream>>>(h->d_np, h->nbrs[nb], h->in_cnt);
  DEM_LAUNCH(h);
  if (int rc = exclusive_scan(h, h->in_cnt, h->in_start, n, h->in_start + n)) return rc;
  if (int rc = check_cuda(h, cudaMemsetAsync(h->in_fill, 0, sizeof(int) * n, h->stream), "memset")) return rc;
  k_in_fill<<<BP, T, 0, h->stream>>>(h->d_np, h->nbrs[nb], h->pair_owner, h->in_start, h->in_fill, h->in_pair);
  DEM_LAUNCH(h);
  k_in_sort<<<B, T, 0, h->stream>>>(n, h->in_start, h->in_pair, h->in_pos, h->in_flag);
  DEM_LAUNCH(h);
  return check_cuda(h, cudaGetLastError(), "transpose");
}

long long pair_array_bytes(long long cap) {
  // nbrs, pft and pflag double-buffered; in_pair, pair_owner, the contact
  // records, gaps, in_pos and in_flag (the flag arrays padded by 16 bytes)
  return 2 * ((long long)sizeof(int) * cap + (long long)sizeof(double) * 3 * cap + cap + 16) +
         (long long)(sizeof(int2) + sizeof(int) + sizeof(PairRec) + sizeof(float) + sizeof(int)) * cap + cap + 16;
}

// The candidate list's array for at least `need` entries, a quarter over
// so that a list that grows a little does not reallocate at every build.
static int ensure_cand_capacity(dem_handle* h, long long need) {
  if (need <= h->cand_cap) return 0;
  const long long cap = need + need / 4 + 1024;
  int* cnb = nullptr;
  if (int rc = check_cuda(h, cudaMalloc(&cnb, sizeof(int) * cap), "cudaMalloc candidates")) return rc;
  cudaStreamSynchronize(h->stream);
  cudaFree(h->cand_nb);
  h->cand_nb = cnb;
  h->cand_cap = cap;
  invalidate_graphs(h);  // captured builds point at the old array
  return check_cuda(h, cudaGetLastError(), "grow candidates");
}

// Pair-list arrays for at least `need` pairs: the first allocation takes
// exactly `need`, a later one doubles the capacity until it fits.
int ensure_pair_capacity(dem_handle* h, long long need) {
  if (need <= h->pair_cap) return 0;
  long long cap = h->pair_cap > 0 ? h->pair_cap : need;
  while (cap < need) cap *= 2;
  const long long old = h->pair_cap;  // the whole old allocation (the count may be stale)
  int* nb[2]; double* pf[2]; int2* inp; int* own; uint8_t* pfl[2]; PairRec* prc; float* gap;
  int* ipos; uint8_t* ifl;
  for (int b = 0; b < 2; ++b) {
    if (int rc = check_cuda(h, cudaMalloc(&nb[b], sizeof(int) * cap), "cudaMalloc nbrs")) return rc;
    if (int rc = check_cuda(h, cudaMalloc(&pf[b], sizeof(double) * 3 * cap), "cudaMalloc pft")) return rc;
    // flag arrays carry 16 bytes of padding: the gather reads them as aligned words
    if (int rc = check_cuda(h, cudaMalloc(&pfl[b], cap + 16), "cudaMalloc pflag")) return rc;
  }
  if (int rc = check_cuda(h, cudaMalloc(&inp, sizeof(int2) * cap), "cudaMalloc in_pair")) return rc;
  if (int rc = check_cuda(h, cudaMalloc(&own, sizeof(int) * cap), "cudaMalloc owner")) return rc;
  if (int rc = check_cuda(h, cudaMalloc(&prc, sizeof(PairRec) * cap), "cudaMalloc prec")) return rc;
  if (int rc = check_cuda(h, cudaMalloc(&gap, sizeof(float) * cap), "cudaMalloc pgap")) return rc;
  if (int rc = check_cuda(h, cudaMalloc(&ipos, sizeof(int) * cap), "cudaMalloc in_pos")) return rc;
  if (int rc = check_cuda(h, cudaMalloc(&ifl, cap + 16), "cudaMalloc in_flag")) return rc;
  if (old > 0) {
    // keep the current list and history (the rebuild reads them)
    cudaMemcpyAsync(nb[h->rb], h->nbrs[h->rb], sizeof(int) * old, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(pf[h->pcur], h->pft[h->pcur], sizeof(double) * 3 * old, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(inp, h->in_pair, sizeof(int2) * old, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(own, h->pair_owner, sizeof(int) * old, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(pfl[h->pcur], h->pflag(), old, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(gap, h->pgap, sizeof(float) * old, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(ipos, h->in_pos, sizeof(int) * old, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(ifl, h->in_flag, old, cudaMemcpyDeviceToDevice, h->stream);
  }
  cudaStreamSynchronize(h->stream);
  for (int b = 0; b < 2; ++b) {
    cudaFree(h->nbrs[b]); cudaFree(h->pft[b]); cudaFree(h->pflagb[b]);
    h->nbrs[b] = nb[b]; h->pft[b] = pf[b]; h->pflagb[b] = pfl[b];
  }
  cudaFree(h->in_pair); cudaFree(h->pair_owner); cudaFree(h->prec); cudaFree(h->pgap);
  cudaFree(h->in_pos); cudaFree(h->in_flag);
  h->in_pair = inp; h->pair_owner = own; h->prec = prc; h->pgap = gap;
  h->in_pos = ipos; h->in_flag = ifl;
  h->pair_cap = cap;
  invalidate_graphs(h);  // captured steps point at the old arrays
  return check_cuda(h, cudaGetLastError(), "grow pairs");
}

// Count pass of the pair build over the current cell-sorted copy: row_cnt
// and the long-row list start from zero, so the pass can be launched again
// on its own (the autotuner times it).
void launch_neigh_count(dem_handle* h, const int* skip) {
  const int n = h->nl(), T = h->tune.neigh_threads, B = (n + T - 1) / T;
  const bool bt = h->batch();
  const int* n_exist = h->fcell_start + (bt ? h->nfcell_total : h->dp.nfcell);
  cudaMemsetAsync(h->row_cnt, 0, sizeof(int) * n, h->stream);
  cudaMemsetAsync(h->long_rows + h->n, 0, sizeof(int), h->stream);  // the count, at [capacity]
  if (bt)
    k_neigh_count<true><<<B, T, 0, h->stream>>>(h->dp, h->bview(), n_exist, h->spos, h->sposf, h->sinfo,
                                                h->fcell_start, h->derr, h->row_cnt, h->nslot, h->long_rows, skip);
  else
    k_neigh_count<false><<<B, T, 0, h->stream>>>(h->dp, h->bview(), n_exist, h->spos, h->sposf, h->sinfo,
                                                 h->fcell_start, h->derr, h->row_cnt, h->nslot, h->long_rows, skip);
  DEM_LAUNCH(h);
}

int run_neighbour(dem_handle* h, bool carry_history) {
  ProfScope ps(h, DEM_PROF_NEIGHBOR);
  const DevParams& p = h->dp;
  const int n = h->nl(), T = 128, B = (n + T - 1) / T;
  const bool bt = h->batch();
  const BatchView bv = h->bview();
  DevErr* e = h->derr;
  // first_rogue := none
  if (bt) k_reset_rogue<<<((int)h->sys.size() + 127) / 128, 128, 0, h->stream>>>((int)h->sys.size(), h->d_first_rogue);
  else k_set_int<<<1, 1, 0, h->stream>>>(&e->first_rogue, n);
  DEM_LAUNCH(h);
  if (bt) k_find_rogue<true><<<B, T, 0, h->stream>>>(p, bv, h->state, h->dg_pijk, e);
  else k_find_rogue<false><<<B, T, 0, h->stream>>>(p, bv, h->state, h->dg_pijk, e);
  DEM_LAUNCH(h);
  const int nb = 1 - h->rb;  // new list goes into the other buffer
  const int* n_exist = h->fcell_start + (bt ? h->nfcell_total : p.nfcell);
  // the candidate list serves single systems without flow boundaries (their
  // seeding and deletion change particle states, and with them the rules of
  // the half list); with them it is dropped
  const bool cand = !bt && h->cand && h->obc.empty() && h->ibc.empty();
  const double skin_c = 0.3 * p.factor_rlm * p.max_radius;
  if (cand) {
    k_cand_decide<<<1, 1, 0, h->stream>>>(h->cand, e, 0.5 * skin_c);
    DEM_LAUNCH(h);
  } else if (h->cand) {
    cudaMemsetAsync(&h->cand->have, 0, sizeof(int), h->stream);
  }
  if (h->qof) cudaMemsetAsync(h->qof, 0xff, sizeof(int) * n, h->stream);
  if (bt)
    k_sorted_copy<true><<<B, T, 0, h->stream>>>(p, bv, n, n_exist, h->fcell_list, h->pos4[h->cur], h->state,
                                                h->dg_pijk, h->fcell_key, h->spos, h->sposf, h->sinfo, nullptr);
  else
    k_sorted_copy<false><<<B, T, 0, h->stream>>>(p, bv, n, n_exist, h->fcell_list, h->pos4[h->cur], h->state,
                                                 h->dg_pijk, h->fcell_key, h->spos, h->sposf, h->sinfo, h->qof);
  DEM_LAUNCH(h);
  launch_neigh_count(h, cand ? &h->cand->ok : nullptr);
  if (cand) {
    k_cand_filter<<<B, T, 0, h->stream>>>(p, n_exist, h->spos, h->sinfo, h->qof, e, h->cand_end, h->cand_nb, h->cand,
                                          h->row_cnt, h->nslot, h->long_rows);
    DEM_LAUNCH(h);
  }
  if (bt) {
    k_keep_rows<false><<<B, T, 0, h->stream>>>(n, h->n_built, bv, h->row_end[h->rb], h->nbrs[h->rb], h->row_cnt, nullptr,
                                               nullptr, nullptr, 0);
    DEM_LAUNCH(h);
  }
  if (int rc = exclusive_scan(h, h->row_cnt, h->row_end[nb], n, h->d_np)) return rc;
  if (!h->capturing) {
    // eager steps read the count back and grow the arrays when needed
    int P = 0;
    if (int rc = check_cuda(h, cudaMemcpyAsync(&P, h->d_np, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "copy P")) return rc;
    if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sync")) return rc;
    if (int rc = ensure_pair_capacity(h, (long long)P + 1)) return rc;
    h->n_pairs = P;
    h->np_stale = false;
  } else {
    h->np_stale = true;
  }
  // rows kept whole by the count pass, then the long rows (a fixed grid
  // striding over the list, whose length is on the device)
  const int BL = 4 * 148;
  if (bt) {
    k_fill_kept<true><<<B, T, 0, h->stream>>>(n, bv, h->row_cnt, h->row_end[nb], h->nbrs[nb], h->pair_owner,
                                              h->nslot, h->pair_cap);
    DEM_LAUNCH(h);
    k_fill_long<true><<<BL, 128, 0, h->stream>>>(p, bv, h->spos, h->sposf, h->sinfo, h->fcell_start, h->row_cnt,
                                                 h->row_end[nb],
                                                 h->nbrs[nb], h->pflagb[1 - h->pcur], h->pair_owner, h->long_rows,
                                                 h->pair_cap);
    DEM_LAUNCH(h);
    k_keep_rows<true><<<B, T, 0, h->stream>>>(n, h->n_built, bv, h->row_end[h->rb], h->nbrs[h->rb], nullptr, h->row_end[nb],
                                              h->nbrs[nb], h->pair_owner, h->pair_cap);
  } else {
    k_fill_kept<false><<<B, T, 0, h->stream>>>(n, bv, h->row_cnt, h->row_end[nb], h->nbrs[nb], h->pair_owner,
                                               h->nslot, h->pair_cap);
    DEM_LAUNCH(h);
    k_fill_long<false><<<BL, 128, 0, h->stream>>>(p, bv, h->spos, h->sposf, h->sinfo, h->fcell_start,
                                                  h->row_cnt, h->row_end[nb], h->nbrs[nb], h->pflagb[1 - h->pcur], h->pair_owner,
                                                  h->long_rows, h->pair_cap);
  }
  DEM_LAUNCH(h);
  k_clamp_np<<<1, 1, 0, h->stream>>>(h->d_np, h->pair_cap, e);
  DEM_LAUNCH(h);
  if (bt)
    k_delete_rogue<true><<<B, T, 0, h->stream>>>(p, bv, h->state, h->dg_pijk, h->pos4[h->cur], h->vel4[h->cur],
                                                  h->omg4[h->cur], h->fc, h->tow, h->wall_fid, e);
  else
    k_delete_rogue<false><<<B, T, 0, h->stream>>>(p, bv, h->state, h->dg_pijk, h->pos4[h->cur], h->vel4[h->cur],
                                                   h->omg4[h->cur], h->fc, h->tow, h->wall_fid, e);
  DEM_LAUNCH(h);
  if (cand) {
    // a new candidate list when k_cand_decide asks for one (each kernel
    // returns at once otherwise)
    cudaMemsetAsync(h->cand_cnt, 0, sizeof(int) * n, h->stream);
    k_cand_build<false><<<B, T, 0, h->stream>>>(p, n_exist, h->spos, h->sposf, h->sinfo, h->fcell_start, h->cand,
                                                skin_c, h->cand_cnt, h->cand_fill, h->cand_start, h->cand_nb,
                                                h->cand_cap);
    DEM_LAUNCH(h);
    if (int rc = exclusive_scan(h, h->cand_cnt, h->cand_start, n, h->cand_start + n)) return rc;
    if (!h->capturing) {
      // eager builds read the list's length back (0 when none is made) and
      // grow its array when needed; a captured build that overflows leaves
      // the list incomplete, unused
      int total = 0;
      if (int rc = check_cuda(h, cudaMemcpyAsync(&total, h->cand_start + n, sizeof(int), cudaMemcpyDeviceToHost,
                                                 h->stream), "copy candidates")) return rc;
      if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sync")) return rc;
      if (int rc = ensure_cand_capacity(h, total)) return rc;
    }
    const long long cap = h->cand_cap;
    cudaMemsetAsync(h->cand_fill, 0, sizeof(int) * n, h->stream);
    k_cand_build<true><<<B, T, 0, h->stream>>>(p, n_exist, h->spos, h->sposf, h->sinfo, h->fcell_start, h->cand,
                                               skin_c, h->cand_cnt, h->cand_fill, h->cand_start, h->cand_nb, cap);
    DEM_LAUNCH(h);
    k_cand_commit<<<B, T, 0, h->stream>>>(n, h->cand_cnt, h->cand_start, h->cand_end, h->cand, e, cap);
    DEM_LAUNCH(h);
  }
  // The transpose of the new list and the history carry-over with the gaps
  // read the list and write disjoint arrays: the transpose runs on the side
  // stream beside them and is joined before the build returns (in sequence
  // when the kernel classes are timed).  Its scan uses the handle's scan
  // scratch, so nothing on this stream between the fork and the join scans
  // (the candidate list above is made before the fork).
  const bool side = h->side_stream && !h->prof;
  int trc = 0;
  if (side) {
    cudaEventRecord(h->ev_fork, h->stream);
    cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0);
    cudaStream_t main = h->stream;
    h->stream = h->side_stream;
    trc = build_transpose(h, nb);
    h->stream = main;
    cudaEventRecord(h->ev_join, h->side_stream);
  }
  // history carry-over into the other pft buffer
  const int pn = 1 - h->pcur;
  const int have_old = (carry_history && h->have_pairs) ? 1 : 0;
  if (bt)
    k_remap<true><<<pair_grid(h, 256), 256, 0, h->stream>>>(p, bv, h->d_np, h->pair_cap, h->nbrs[nb],
                                                            h->pair_owner, h->row_end[h->rb], h->nbrs[h->rb],
                                                            h->pft[h->pcur], h->pft[pn], h->pflagb[pn], have_old,
                                                            h->pos4[h->cur], h->state, h->pgap, h->skin);
  else
    k_remap<false><<<pair_grid(h, 256), 256, 0, h->stream>>>(p, bv, h->d_np, h->pair_cap, h->nbrs[nb],
                                                             h->pair_owner, h->row_end[h->rb], h->nbrs[h->rb],
                                                             h->pft[h->pcur], h->pft[pn], h->pflagb[pn], have_old,
                                                             h->pos4[h->cur], h->state, h->pgap, h->skin);
  DEM_LAUNCH(h);
  h->rb = nb;
  h->n_built = n;
  h->pcur = pn;
  h->have_pairs = true;
  launch_wall_gaps(h);
  if (side) {
    cudaStreamWaitEvent(h->stream, h->ev_join, 0);
    return trc;
  }
  return build_transpose(h, nb);
}

long long host_pairs(dem_handle* h) {
  if (h->np_stale) {
    int P = 0;
    cudaMemcpyAsync(&P, h->d_np, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    cudaStreamSynchronize(h->stream);
    h->n_pairs = P;
    h->np_stale = false;
  }
  return h->n_pairs;
}

}  // namespace demb
