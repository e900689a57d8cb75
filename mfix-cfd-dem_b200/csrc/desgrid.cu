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

// Cell of every existing particle; in a batch only for systems that rebuild
// now or have periodic axes (the others keep the cells of their last build,
// as the reference does between rebuilds).
template <bool B>
__global__ void k_cell_keys(DevParams p0, BatchView bv, double4* __restrict__ pos4,
                            const int8_t* __restrict__ state, int* __restrict__ dg_pijk,
                            const int* __restrict__ fbin_start, uint8_t* __restrict__ wall_cand,
                            float* __restrict__ wgap) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p0.n) return;
  const DevParams& p = sysp<B>(p0, bv, i);
  const bool per = p.per[0] || p.per[1] || (p.per[2] && !p.no_k);
  if constexpr (B) {
    if (!bv.due[bv.sys_of[i]] && !per) return;
  }
  // the position is read with the state (both loads in flight at once)
  double4 x = pos4[i];
  if (state[i] == DEM_STATE_NONEXISTENT) { dg_pijk[i] = 0; wall_cand[i] = 0; return; }
  int c;
  if (dg_place(p, per, x, c)) pos4[i] = x;
  // the facet clearance of the last build holds for that build's cell only
  if (dg_pijk[i] != c) wgap[i] = -1.0f;
  dg_pijk[i] = c;
  const int fc = p.cell_off + c - 1;
  wall_cand[i] = fbin_start[fc + 1] > fbin_start[fc] ? 1 : 0;
}

// The facet-cell flag of every particle from its current DES cell (after
// the walls change).
template <bool B>
__global__ void k_wall_cand(DevParams p0, BatchView bv, const int8_t* __restrict__ state,
                            const int* __restrict__ dg_pijk, const int* __restrict__ fbin_start,
                            uint8_t* __restrict__ wall_cand) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p0.n) return;
  const DevParams& p = sysp<B>(p0, bv, i);
  const int c = dg_pijk[i];
  if (state[i] == DEM_STATE_NONEXISTENT || c < 1) { wall_cand[i] = 0; return; }
  const int fc = p.cell_off + c - 1;
  wall_cand[i] = fbin_start[fc + 1] > fbin_start[fc] ? 1 : 0;
}

void launch_wall_cand(dem_handle* h) {
  const int T = 256, B = (h->nl() + T - 1) / T;
  if (h->batch())
    k_wall_cand<true><<<B, T, 0, h->stream>>>(h->dp, h->bview(), h->state, h->dg_pijk, h->fbin_start, h->wall_cand);
  else
    k_wall_cand<false><<<B, T, 0, h->stream>>>(h->dp, h->bview(), h->state, h->dg_pijk, h->fbin_start, h->wall_cand);
  DEM_LAUNCH(h);
  skin_unknown(h);  // the walls changed: no particle is known clear of them until the next build
}

// Search-grid cell of every existing particle (for the pair build), as an
// index into the handle-wide search-cell arrays; -1 for particles of batch
// systems that do not rebuild now.
template <bool B>
__global__ void k_fine_keys(DevParams p0, BatchView bv, const double4* __restrict__ pos4,
                            const int8_t* __restrict__ state, int* __restrict__ fkey, int* __restrict__ fcnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p0.n) return;
  const DevParams& p = sysp<B>(p0, bv, i);
  if constexpr (B) {
    if (!bv.due[bv.sys_of[i]]) { fkey[i] = -1; return; }
  }
  if (state[i] == DEM_STATE_NONEXISTENT) return;
  const double4 x = pos4[i];
  const double xx[3] = {x.x, x.y, x.z};
  int g[3] = {0, 0, 0};
  for (int a = 0; a < 3; ++a) {
    if (a == 2 && p.no_k) break;
    int v = (int)floor((xx[a] - p.dg_start[a]) * p.f_inv[a]) + 1;
    const int lo = p.per[a] ? 1 : 0, hi = p.per[a] ? p.fn[a] : p.fn[a] + 1;
    g[a] = min(hi, max(lo, v));
  }
  const int key = p.fcell_off + g[2] * p.fc2 + g[0] * p.fc1 + g[1];
  fkey[i] = key;
  atomicAdd(&fcnt[key], 1);
}

__global__ void k_fine_scatter(int n, const int8_t* __restrict__ state, const int* __restrict__ fkey,
                               const int* __restrict__ fstart, int* __restrict__ ffill, int* __restrict__ flist) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || state[i] == DEM_STATE_NONEXISTENT) return;
  const int c = fkey[i];
  if (c < 0) return;
  const int slot = atomicAdd(&ffill[c], 1);
  flist[fstart[c] + slot] = i;
}

// DESGRID_PIC: cell of every particle (and the periodic wrap).  When
// `bin_search` is set (neighbour-search steps) the particles are also binned
// to the search grid of the pair build.
int run_desgrid_pic(dem_handle* h, bool bin_search) {
  ProfScope ps(h, DEM_PROF_DESGRID);
  const DevParams& p = h->dp;
  const int n = h->nl(), T = 256, B = (n + T - 1) / T;
  const bool bt = h->batch();
  const BatchView bv = h->bview();
  // the live systems' cells (one more, empty, ends the last range); the
  // count of binned particles also goes to the end of the cell arrays,
  // where the pair build reads it
  const int nfc = h->nfl() + 1;
  int* n_binned = h->fcell_start + (bt ? h->nfcell_total : p.nfcell);
  if (bt)
    k_cell_keys<true><<<B, T, 0, h->stream>>>(p, bv, h->pos4[h->cur], h->state, h->dg_pijk, h->fbin_start,
                                              h->wall_cand, h->wgap);
  else
    k_cell_keys<false><<<B, T, 0, h->stream>>>(p, bv, h->pos4[h->cur], h->state, h->dg_pijk, h->fbin_start,
                                               h->wall_cand, h->wgap);
  DEM_LAUNCH(h);
  // particles seeded since the last DESGRID_PIC are in its cell lists now
  if (h->pic_fresh && !h->ibc.empty()) cudaMemsetAsync(h->pic_fresh, 0, (size_t)n, h->stream);
  if (!bin_search) return check_cuda(h, cudaGetLastError(), "k_cell_keys");
  if (int rc = check_cuda(h, cudaMemsetAsync(h->fcell_cnt, 0, sizeof(int) * nfc, h->stream), "memset")) return rc;
  if (bt) k_fine_keys<true><<<B, T, 0, h->stream>>>(p, bv, h->pos4[h->cur], h->state, h->fcell_key, h->fcell_cnt);
  else k_fine_keys<false><<<B, T, 0, h->stream>>>(p, bv, h->pos4[h->cur], h->state, h->fcell_key, h->fcell_cnt);
  DEM_LAUNCH(h);
  if (int rc = exclusive_scan(h, h->fcell_cnt, h->fcell_start, nfc, n_binned)) return rc;
  if (int rc = check_cuda(h, cudaMemsetAsync(h->fcell_cnt, 0, sizeof(int) * nfc, h->stream), "memset")) return rc;
  k_fine_scatter<<<B, T, 0, h->stream>>>(n, h->state, h->fcell_key, h->fcell_start, h->fcell_cnt, h->fcell_list);
  DEM_LAUNCH(h);
  return check_cuda(h, cudaGetLastError(), "desgrid_pic");
}

}  // namespace demb
