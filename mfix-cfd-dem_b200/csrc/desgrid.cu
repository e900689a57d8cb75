// desgrid.cu -- DES grid binning (K1).
//
// Replaces DESGRID_PIC(.TRUE.) (model/des/desgrid_mod.f:877-995) with the
// cell functions IofPOS/JofPOS/KofPOS (391-419) and DG_FUNIJK (184-188):
//   dg_pijk = dg_funijk(clamp(iofpos(x)), clamp(jofpos(y)), clamp(kofpos(z)))
// followed by a counting sort of particle indices into per-cell lists whose
// order is ascending particle index, the order of the serial reference.
// The sort is: count (atomics) -> exclusive scan -> scatter (atomics) ->
// per-cell rank sort (one warp per cell, shared memory), so the result does
// not depend on the order in which atomics were served.
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

__global__ void k_cell_scatter(int n, const int8_t* __restrict__ state, const int* __restrict__ dg_pijk,
                               const int* __restrict__ cell_start, int* __restrict__ cell_fill,
                               int* __restrict__ cell_list) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || state[i] == DEM_STATE_NONEXISTENT) return;
  int c = dg_pijk[i] - 1;
  int slot = atomicAdd(&cell_fill[c], 1);
  cell_list[cell_start[c] + slot] = i;
}

constexpr int SORT_WARPS = 4;
constexpr int SORT_CAP = 1024;  // particles per cell sorted in shared memory

// One warp per cell: each lane ranks its elements by counting smaller ones
// (indices are distinct), then writes them to their sorted slot.
__global__ void k_cell_sort(int ncell, const int* __restrict__ cell_start, int* __restrict__ cell_list) {
  __shared__ int buf[SORT_WARPS][SORT_CAP];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * SORT_WARPS + w;
  if (c >= ncell) return;
  const int s = cell_start[c], e = cell_start[c + 1];
  const int k = e - s;
  if (k <= 1) return;
  if (k <= SORT_CAP) {
    for (int t = lane; t < k; t += 32) buf[w][t] = cell_list[s + t];
    __syncwarp();
    for (int t = lane; t < k; t += 32) {
      int v = buf[w][t], r = 0;
      for (int u = 0; u < k; ++u) r += (buf[w][u] < v);
      cell_list[s + r] = v;
    }
  } else if (lane == 0) {
    // rare overfull cell: insertion sort in global memory
    for (int a = s + 1; a < e; ++a) {
      int v = cell_list[a], b = a - 1;
      while (b >= s && cell_list[b] > v) { cell_list[b + 1] = cell_list[b]; --b; }
      cell_list[b + 1] = v;
    }
  }
}

int run_desgrid_pic(dem_handle* h, bool sort_cells) {
  ProfScope ps(h, DEM_PROF_DESGRID);
  const DevParams& p = h->dp;
  const int n = h->n, T = 256, B = (n + T - 1) / T;
  const bool anyper = p.per[0] || p.per[1] || (p.per[2] && !p.no_k);
  if (sort_cells) {
    if (int rc = check_cuda(h, cudaMemsetAsync(h->cell_cnt, 0, sizeof(int) * p.ncell2, h->stream), "memset")) return rc;
  }
  k_cell_keys<<<B, T, 0, h->stream>>>(p, h->pos4[h->cur], h->state, h->dg_pijk,
                                      sort_cells ? h->cell_cnt : nullptr, anyper ? 1 : 0);
  DEM_LAUNCH(h);
  if (!sort_cells) return check_cuda(h, cudaGetLastError(), "k_cell_keys");
  if (int rc = exclusive_scan(h, h->cell_cnt, h->cell_start, p.ncell2, h->cell_start + p.ncell2)) return rc;
  if (int rc = check_cuda(h, cudaMemsetAsync(h->cell_fill, 0, sizeof(int) * p.ncell2, h->stream), "memset")) return rc;
  k_cell_scatter<<<B, T, 0, h->stream>>>(n, h->state, h->dg_pijk, h->cell_start, h->cell_fill, h->cell_list);
  DEM_LAUNCH(h);
  k_cell_sort<<<(p.ncell2 + SORT_WARPS - 1) / SORT_WARPS, 32 * SORT_WARPS, 0, h->stream>>>(
      p.ncell2, h->cell_start, h->cell_list);
  DEM_LAUNCH(h);
  return check_cuda(h, cudaGetLastError(), "desgrid_pic");
}

}  // namespace demb
