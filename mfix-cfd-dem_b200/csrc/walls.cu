// walls.cu -- wall facets binned to the DES grid (set-up, runs once).
//
// Replaces BIN_FACETS_TO_DG, ADD_FACET_FOR_DES and ADD_FACET
// (model/des/stl_preproc_des_mod.f:135-349) with TRI_BOX_OVERLAP
// (model/des/stl_functions_des_mod.f:280-536, the Akenine-Moller
// triangle/box test), and FLAG_FACETS_WHERE_EDGE_COLLISION_IS_IGNORED
// (stl_preproc_des_mod.f:361-490).  One thread per DES cell tests every
// facet whose index range covers the cell, so each cell's list comes out in
// ascending facet order, the order of the reference's outer facet loop.
#include "dem_internal.cuh"

#include <cfloat>
#include <cmath>

namespace demb {

constexpr double TOL_STL = 1.0e-6;   // cartesian_grid_init_namelist.f:748
constexpr double TOL_EDGE = 1.0e-9;  // stl_preproc_des_mod.f:383

__device__ bool tri_box_overlap(const double ctr[3], const double hs[3], const double* V /*[v][c]*/) {
  double v0[3], v1[3], v2[3], e0[3], e1[3], e2[3];
  for (int c = 0; c < 3; ++c) { v0[c] = V[c] - ctr[c]; v1[c] = V[3 + c] - ctr[c]; v2[c] = V[6 + c] - ctr[c]; }
  for (int c = 0; c < 3; ++c) { e0[c] = v1[c] - v0[c]; e1[c] = v2[c] - v1[c]; e2[c] = v0[c] - v2[c]; }
  auto axtest = [](double pa, double pb, double rad) {
    double lmin = pa < pb ? pa : pb, lmax = pa < pb ? pb : pa;
    return (lmin > rad || lmax < -rad);
  };
  auto z12 = [](double pa1, double pa2, double rad) {
    double lmin, lmax;
    if (pa2 < pa1) { lmin = pa2; lmax = pa1; } else { lmin = pa1; lmax = pa2; }
    return (lmin > rad || lmax < -rad);
  };
  double fex, fey, fez, a, b;
  fex = fabs(e0[0]); fey = fabs(e0[1]); fez = fabs(e0[2]);
  a = e0[2]; b = e0[1]; if (axtest(a * v0[1] - b * v0[2], a * v2[1] - b * v2[2], fez * hs[1] + fey * hs[2])) return false;
  a = e0[2]; b = e0[0]; if (axtest(-a * v0[0] + b * v0[2], -a * v2[0] + b * v2[2], fez * hs[0] + fex * hs[2])) return false;
  a = e0[1]; b = e0[0]; if (z12(a * v1[0] - b * v1[1], a * v2[0] - b * v2[1], fey * hs[0] + fex * hs[1])) return false;
  fex = fabs(e1[0]); fey = fabs(e1[1]); fez = fabs(e1[2]);
  a = e1[2]; b = e1[1]; if (axtest(a * v0[1] - b * v0[2], a * v2[1] - b * v2[2], fez * hs[1] + fey * hs[2])) return false;
  a = e1[2]; b = e1[0]; if (axtest(-a * v0[0] + b * v0[2], -a * v2[0] + b * v2[2], fez * hs[0] + fex * hs[2])) return false;
  a = e1[1]; b = e1[0]; if (axtest(a * v0[0] - b * v0[1], a * v1[0] - b * v1[1], fey * hs[0] + fex * hs[1])) return false;
  fex = fabs(e2[0]); fey = fabs(e2[1]); fez = fabs(e2[2]);
  a = e2[2]; b = e2[1]; if (axtest(a * v0[1] - b * v0[2], a * v1[1] - b * v1[2], fez * hs[1] + fey * hs[2])) return false;
  a = e2[2]; b = e2[0]; if (axtest(-a * v0[0] + b * v0[2], -a * v1[0] + b * v1[2], fez * hs[0] + fex * hs[2])) return false;
  a = e2[1]; b = e2[0]; if (z12(a * v1[0] - b * v1[1], a * v2[0] - b * v2[1], fey * hs[0] + fex * hs[1])) return false;
  for (int c = 0; c < 3; ++c) {
    double mn = v0[c]; if (v1[c] < mn) mn = v1[c]; if (v2[c] < mn) mn = v2[c];
    double mx = v0[c]; if (v1[c] > mx) mx = v1[c]; if (v2[c] > mx) mx = v2[c];
    if (mn > hs[c] || mx < -hs[c]) return false;
  }
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

// Cell range of facet f (BIN_FACETS_TO_DG lines 160-186).
__device__ void facet_range(const DevParams& p, const double* V, int rng[6]) {
  double lo[3], hi[3];
  for (int c = 0; c < 3; ++c) {
    double a = V[c], b = V[3 + c], d = V[6 + c];
    lo[c] = fmin(a, fmin(b, d));
    hi[c] = fmax(a, fmax(b, d));
  }
  const int s2[3] = {p.istart2, p.jstart2, p.kstart2}, e2[3] = {p.iend2, p.jend2, p.kend2};
  const int s1[3] = {p.istart1, p.jstart1, p.kstart1};
  for (int c = 0; c < 3; ++c) {
    rng[2 * c] = e2[c];
    rng[2 * c + 1] = s2[c];
    if (c == 2 && p.no_k) continue;
    if (hi[c] >= p.lo[c] - TOL_STL && lo[c] <= p.hi[c] + TOL_STL) {
      rng[2 * c] = max(dg_ofpos(p, c, lo[c], s1[c]) - 1, s2[c]);
      rng[2 * c + 1] = min(dg_ofpos(p, c, hi[c], s1[c]) + 1, e2[c]);
    }
  }
}

template <bool FILL>
__global__ void k_bin_facets(DevParams p, int nf, const double* __restrict__ vertex, double buffer, int fac_off,
                             int* __restrict__ cnt, const int* __restrict__ start, FacetBinEntry* __restrict__ out) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;  // 0-based
  if (cell >= p.ncell2) return;
  const int ijk = cell + 1;
  const int ii = dg_iof(p, ijk), jj = dg_jof(p, ijk), kk = dg_kof(p, ijk);
  const double ldx = 1.0 / p.dg_inv[0], ldy = 1.0 / p.dg_inv[1], ldz = 1.0 / p.dg_inv[2];
  double ctr[3], hs[3];
  ctr[0] = p.dg_start[0] + ((double)(ii - p.istart1) + 0.5) * ldx; hs[0] = 0.5 * ldx + buffer;
  ctr[1] = p.dg_start[1] + ((double)(jj - p.jstart1) + 0.5) * ldy; hs[1] = 0.5 * ldy + buffer;
  if (!p.no_k) { ctr[2] = p.dg_start[2] + ((double)(kk - p.kstart1) + 0.5) * ldz; hs[2] = 0.5 * ldz + buffer; }
  else { ctr[2] = 0.5 * ldz; hs[2] = 0.5 * ldz; }
  int k = 0;
  const int base = FILL ? start[cell] : 0;
  for (int f = 0; f < nf; ++f) {
    const double* V = vertex + 9 * (size_t)f;
    int rng[6];
    facet_range(p, V, rng);
    if (ii < rng[0] || ii > rng[1] || jj < rng[2] || jj > rng[3] || kk < rng[4] || kk > rng[5]) continue;
    if (!tri_box_overlap(ctr, hs, V)) continue;
    if (FILL) {
      FacetBinEntry e;
      e.id = fac_off + f; e.dir = 0; e.mn = 0.0; e.mx = 0.0;
      double smallest = (double)FLT_MAX;  // HUGE(0.0)
      for (int c = 0; c < 3; ++c) {
        double a = V[c], b = V[3 + c], d = V[6 + c];
        double mn = fmin(a, fmin(b, d)), mx = fmax(a, fmax(b, d));
        if (fabs(mx - mn) < smallest) { e.dir = c; e.mn = mn; e.mx = mx; smallest = fabs(mx - mn); }
      }
      out[base + k] = e;
    }
    ++k;
  }
  if (!FILL) cnt[cell] = k;
}

__global__ void k_edge_flags(int ncell, const int* __restrict__ start, const FacetBinEntry* __restrict__ bins,
                             const double* __restrict__ vertex, const double* __restrict__ norm, double cos_nb,
                             int8_t* __restrict__ flags) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= ncell) return;
  const int s = start[cell], e = start[cell + 1];
  for (int a = s; a < e; ++a) {
    const int fa = bins[a].id;
    const double* Va = vertex + 9 * (size_t)fa;
    double ec[3][3];
    for (int c = 0; c < 3; ++c) {
      ec[0][c] = 0.5 * (Va[c] + Va[3 + c]);
      ec[1][c] = 0.5 * (Va[c] + Va[6 + c]);
      ec[2][c] = 0.5 * (Va[3 + c] + Va[6 + c]);
    }
    for (int ed = 0; ed < 3; ++ed)
      for (int b = s; b < e; ++b) {
        if (a == b) continue;
        const int fb = bins[b].id;
        const double* Vb = vertex + 9 * (size_t)fb;
        for (int ned = 0; ned < 3; ++ned) {
          const int i0 = ned == 2 ? 3 : 0, i1 = ned == 0 ? 3 : 6;
          double d[3];
          for (int c = 0; c < 3; ++c) d[c] = 0.5 * (Vb[i0 + c] + Vb[i1 + c]) - ec[ed][c];
          if (dot3(d, d) < TOL_EDGE) {
            const double* na = norm + 3 * (size_t)fa;
            const double* nb = norm + 3 * (size_t)fb;
            const double dp = na[0] * nb[0] + na[1] * nb[1] + na[2] * nb[2];
            if (dp > cos_nb) {
              flags[4 * (size_t)fa + ed + 1] = 1;
              flags[4 * (size_t)fb + ned + 1] = 1;
            }
          }
        }
      }
  }
}

int run_bin_facets(dem_handle* h, const double* vf, const double* nfort, int nf) {
  const DevParams& p = h->dp;
  invalidate_graphs(h);
  cudaFree(h->vertex); cudaFree(h->norm_face); cudaFree(h->ignore_edge); cudaFree(h->fbin);
  h->vertex = nullptr; h->norm_face = nullptr; h->ignore_edge = nullptr; h->fbin = nullptr;
  h->nf = nf;
  h->n_fbin = 0;
  if (int rc = check_cuda(h, cudaMemsetAsync(h->fbin_start, 0, sizeof(int) * (p.ncell2 + 1), h->stream), "memset")) return rc;
  if (nf == 0) {
    launch_wall_cand(h);
    return check_cuda(h, cudaStreamSynchronize(h->stream), "sync");
  }
  // Fortran VERTEX(3,3,F) [v + 3c + 9f] -> device [f][v][c]
  std::vector<double> vx((size_t)9 * nf), nx((size_t)3 * nf);
  for (int f = 0; f < nf; ++f)
    for (int v = 0; v < 3; ++v)
      for (int c = 0; c < 3; ++c) vx[(size_t)9 * f + 3 * v + c] = vf[v + 3 * c + 9 * (size_t)f];
  for (size_t q = 0; q < nx.size(); ++q) nx[q] = nfort[q];
  if (int rc = check_cuda(h, cudaMalloc(&h->vertex, sizeof(double) * vx.size()), "cudaMalloc")) return rc;
  if (int rc = check_cuda(h, cudaMalloc(&h->norm_face, sizeof(double) * nx.size()), "cudaMalloc")) return rc;
  if (int rc = check_cuda(h, cudaMalloc(&h->ignore_edge, (size_t)4 * nf), "cudaMalloc")) return rc;
  cudaMemcpyAsync(h->vertex, vx.data(), sizeof(double) * vx.size(), cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(h->norm_face, nx.data(), sizeof(double) * nx.size(), cudaMemcpyHostToDevice, h->stream);
  cudaMemsetAsync(h->ignore_edge, 0, (size_t)4 * nf, h->stream);
  const int T = 128, B = (p.ncell2 + T - 1) / T;
  const double buffer = 1.1 * p.max_radius;
  k_bin_facets<false><<<B, T, 0, h->stream>>>(p, nf, h->vertex, buffer, 0, h->cell_cnt, nullptr, nullptr);
  DEM_LAUNCH(h);
  int* total = h->cell_fill;
  if (int rc = exclusive_scan(h, h->cell_cnt, h->fbin_start, p.ncell2, total)) return rc;
  int nb = 0;
  cudaMemcpyAsync(&nb, total, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sync")) return rc;
  cudaMemcpyAsync(h->fbin_start + p.ncell2, &nb, sizeof(int), cudaMemcpyHostToDevice, h->stream);
  if (int rc = check_cuda(h, cudaMalloc(&h->fbin, sizeof(FacetBinEntry) * (size_t)(nb > 0 ? nb : 1)), "cudaMalloc")) return rc;
  h->n_fbin = nb;
  k_bin_facets<true><<<B, T, 0, h->stream>>>(p, nf, h->vertex, buffer, 0, nullptr, h->fbin_start, h->fbin);
  DEM_LAUNCH(h);
  // COS_STL_NB_ANGLE = DCOS(STL_NB_ANGLE/180*PI) + 1e-6, STL_NB_ANGLE = 5.0 (REAL)
  const double pi = 4.0 * std::atan(1.0);
  const double cos_nb = std::cos((double)5.0f / 180.0 * pi) + 1.0e-6;
  k_edge_flags<<<B, T, 0, h->stream>>>(p.ncell2, h->fbin_start, h->fbin, h->vertex, h->norm_face, cos_nb,
                                       h->ignore_edge);
  DEM_LAUNCH(h);
  launch_wall_cand(h);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "bin facets");
}

__global__ void k_add_int(int n, int* __restrict__ a, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] += v;
}

// Facets of one system of a batch handle.  The system owns the facet range
// [fac_off, fac_off + nf), the bin range [bin_off, bin_off + nbin) and the
// ncell2 + 1 entries of fbin_start from its cell_off (its own end pointer
// included), so binning one system leaves the others untouched.  Facet ids
// in the bins and in the wall history are handle-wide.
int run_bin_facets_sys(dem_handle* h, int sys, const double* vf, const double* nfort, int nf) {
  SysSlot& S = h->sys[sys];
  const DevParams& p = S.dp;
  invalidate_graphs(h);
  if (S.nf > 0) h->fac_alloc.give(S.fac_off, S.nf);
  if (S.nbin > 0) h->bin_alloc.give(S.bin_off, S.nbin);
  S.nf = 0; S.nbin = 0; S.fac_off = 0; S.bin_off = 0;
  int* fs = h->fbin_start + p.cell_off;
  if (int rc = check_cuda(h, cudaMemsetAsync(fs, 0, sizeof(int) * (p.ncell2 + 1), h->stream), "memset")) return rc;
  if (nf == 0) {
    launch_wall_cand(h);
    return check_cuda(h, cudaStreamSynchronize(h->stream), "sync");
  }
  const int fo = h->fac_alloc.take(nf, 1);
  if (fo < 0) return set_err(h, DEM_ERR_CAPACITY, "batch facet capacity exhausted");
  S.fac_off = fo; S.nf = nf;
  std::vector<double> vx((size_t)9 * nf), nx((size_t)3 * nf);
  for (int f = 0; f < nf; ++f)
    for (int v = 0; v < 3; ++v)
      for (int c = 0; c < 3; ++c) vx[(size_t)9 * f + 3 * v + c] = vf[v + 3 * c + 9 * (size_t)f];
  for (size_t q = 0; q < nx.size(); ++q) nx[q] = nfort[q];
  cudaMemcpyAsync(h->vertex + 9 * (size_t)fo, vx.data(), sizeof(double) * vx.size(), cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(h->norm_face + 3 * (size_t)fo, nx.data(), sizeof(double) * nx.size(), cudaMemcpyHostToDevice, h->stream);
  cudaMemsetAsync(h->ignore_edge + 4 * (size_t)fo, 0, (size_t)4 * nf, h->stream);
  const int T = 128, B = (p.ncell2 + T - 1) / T;
  const double buffer = 1.1 * p.max_radius;
  const double* V = h->vertex + 9 * (size_t)fo;
  k_bin_facets<false><<<B, T, 0, h->stream>>>(p, nf, V, buffer, fo, h->cell_cnt, nullptr, nullptr);
  DEM_LAUNCH(h);
  if (int rc = exclusive_scan(h, h->cell_cnt, fs, p.ncell2, fs + p.ncell2)) return rc;
  int nb = 0;
  cudaMemcpyAsync(&nb, fs + p.ncell2, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sync")) return rc;
  const int bo = nb > 0 ? h->bin_alloc.take(nb, 1) : 0;
  if (bo < 0) return set_err(h, DEM_ERR_CAPACITY, "batch facet-bin capacity exhausted");
  S.bin_off = bo; S.nbin = nb;
  k_add_int<<<(p.ncell2 + 1 + T - 1) / T, T, 0, h->stream>>>(p.ncell2 + 1, fs, bo);
  k_bin_facets<true><<<B, T, 0, h->stream>>>(p, nf, V, buffer, fo, nullptr, fs, h->fbin);
  h->launches += 2;
  const double pi = 4.0 * std::atan(1.0);
  const double cos_nb = std::cos((double)5.0f / 180.0 * pi) + 1.0e-6;
  k_edge_flags<<<B, T, 0, h->stream>>>(p.ncell2, fs, h->fbin, h->vertex, h->norm_face, cos_nb, h->ignore_edge);
  DEM_LAUNCH(h);
  launch_wall_cand(h);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "bin facets");
}

}  // namespace demb
