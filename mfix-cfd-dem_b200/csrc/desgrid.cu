// desgrid.cu -- DES grid binning (K1).
//
// Replaces DESGRID_PIC(.TRUE.) (model/des/desgrid_mod.f:877-995) with the
// cell functions IofPOS/JofPOS/KofPOS (391-419) and DG_FUNIJK (184-188):
//   dg_pijk = dg_funijk(clamp(iofpos(x)), clamp(jofpos(y)), clamp(kofpos(z)))
// On neighbour-search steps the particles are also binned (count -> scan
// -> scatter) to the finer search grid of the pair build; the order inside a
// search cell does not matter there because every row is put into the
// reference's stencil order when it is filled.
//
// For periodic axes the same pass wraps particles that crossed a periodic
// face by one period, which is what the serial self-exchange of
// DES_PAR_EXCHANGE (mpi_funs_des_mod.f:38-160) does for crossing particles.
#include "dem_internal.cuh"

namespace demb {

__global__ void k_cell_keys(DevParams p, double4* __restrict__ pos4, const int8_t* __restrict__ state,
                            int* __restrict__ dg_pijk, int* __restrict__ cell_cnt, int do_wrap) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  if (state[i] == DEM_STATE_NONEXISTENT) { dg_pijk[i] = 0; return; }
  double4 x = pos4[i];
  if (do_wrap) {
    bool moved = false;
    if (p.per[0]) {
      int ci = dg_ofpos(p, 0, x.x, p.istart1);
      if (ci > p.iend1) { x.x = x.x - p.L[0]; moved = true; }
      else if (ci < p.istart1) { x.x = x.x + p.L[0]; moved = true; }
    }
    if (p.per[1]) {
      int cj = dg_ofpos(p, 1, x.y, p.jstart1);
      if (cj > p.jend1) { x.y = x.y - p.L[1]; moved = true; }
      else if (cj < p.jstart1) { x.y = x.y + p.L[1]; moved = true; }
    }
    if (p.per[2] && !p.no_k) {
      int ck = dg_ofpos(p, 2, x.z, p.kstart1);
      if (ck > p.kend1) { x.z = x.z - p.L[2]; moved = true; }
      else if (ck < p.kstart1) { x.z = x.z + p.L[2]; moved = true; }
    }
    if (moved) pos4[i] = x;
  }
  int li = min(p.iend2, max(p.istart2, dg_ofpos(p, 0, x.x, p.istart1)));
  int lj = min(p.jend2, max(p.jstart2, dg_ofpos(p, 1, x.y, p.jstart1)));
  int lk = p.no_k ? 1 : min(p.kend2, max(p.kstart2, dg_ofpos(p, 2, x.z, p.kstart1)));
  int c = dg_funijk(p, li, lj, lk);
  dg_pijk[i] = c;
  if (cell_cnt) atomicAdd(&cell_cnt[c - 1], 1);
}

// Search-grid cell of every existing particle (for the pair build).
__global__ void k_fine_keys(DevParams p, const double4* __restrict__ pos4, const int8_t* __restrict__ state,
                            int* __restrict__ fkey, int* __restrict__ fcnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n || state[i] == DEM_STATE_NONEXISTENT) return;
  const double4 x = pos4[i];
  const double xx[3] = {x.x, x.y, x.z};
  int g[3] = {0, 0, 0};
  for (int a = 0; a < 3; ++a) {
    if (a == 2 && p.no_k) break;
    int v = (int)floor((xx[a] - p.dg_start[a]) * p.f_inv[a]) + 1;
    const int lo = p.per[a] ? 1 : 0, hi = p.per[a] ? p.fn[a] : p.fn[a] + 1;
    g[a] = min(hi, max(lo, v));
  }
  const int key = g[2] * p.fc2 + g[0] * p.fc1 + g[1];
  fkey[i] = key;
  atomicAdd(&fcnt[key], 1);
}

__global__ void k_fine_scatter(int n, const int8_t* __restrict__ state, const int* __restrict__ fkey,
                               const int* __restrict__ fstart, int* __restrict__ ffill, int* __restrict__ flist) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || state[i] == DEM_STATE_NONEXISTENT) return;
  const int c = fkey[i];
  const int slot = atomicAdd(&ffill[c], 1);
  flist[fstart[c] + slot] = i;
}

// DESGRID_PIC: cell of every particle (and the periodic wrap).  When
// `bin_search` is set (neighbour-search steps) the particles are also binned
// to the search grid of the pair build.
int run_desgrid_pic(dem_handle* h, bool bin_search) {
  ProfScope ps(h, DEM_PROF_DESGRID);
  const DevParams& p = h->dp;
  const int n = h->n, T = 256, B = (n + T - 1) / T;
  const bool anyper = p.per[0] || p.per[1] || (p.per[2] && !p.no_k);
  k_cell_keys<<<B, T, 0, h->stream>>>(p, h->pos4[h->cur], h->state, h->dg_pijk, nullptr, anyper ? 1 : 0);
  DEM_LAUNCH(h);
  if (!bin_search) return check_cuda(h, cudaGetLastError(), "k_cell_keys");
  if (int rc = check_cuda(h, cudaMemsetAsync(h->fcell_cnt, 0, sizeof(int) * p.nfcell, h->stream), "memset")) return rc;
  k_fine_keys<<<B, T, 0, h->stream>>>(p, h->pos4[h->cur], h->state, h->fcell_key, h->fcell_cnt);
  DEM_LAUNCH(h);
  if (int rc = exclusive_scan(h, h->fcell_cnt, h->fcell_start, p.nfcell, h->fcell_start + p.nfcell)) return rc;
  if (int rc = check_cuda(h, cudaMemsetAsync(h->fcell_cnt, 0, sizeof(int) * p.nfcell, h->stream), "memset")) return rc;
  k_fine_scatter<<<B, T, 0, h->stream>>>(n, h->state, h->fcell_key, h->fcell_start, h->fcell_cnt, h->fcell_list);
  DEM_LAUNCH(h);
  return check_cuda(h, cudaGetLastError(), "desgrid_pic");
}

}  // namespace demb
