// batch.cu -- many independent DEM systems in one handle.
//
// No counterpart in the reference, which runs one system per process.  A
// batch handle owns handle-wide arrays (particles, DES cells, search cells,
// wall facets and their bins, pair list) and gives every system a range of
// each: its particles [p_begin, p_end), its DES cells (plus one end entry of
// the facet bins) from cell_off, its search cells from fcell_off, its facets
// and bins.  Every kernel runs once over the whole handle and reads a
// particle's parameters from the system table (BatchView), so one launch
// steps all systems, whatever their sizes.
//
// Each system keeps its own DES_TIME_STEP numbering NN and rebuilds its pair
// list when NN == 1 or mod(NN, NEIGHBOR_SEARCH_N) == 0, as it would alone:
// at a rebuild event the systems that are not due keep their rows (copied
// with their history), so a system's results do not depend on which other
// systems share the handle.  A system's ranges never move while it lives.
#include "dem_internal.cuh"

#include <algorithm>
#include <cstring>

using namespace demb;

namespace demb {

int RangeAlloc::take(int len, int align) {
  if (len <= 0) return 0;
  for (size_t k = 0; k < free_.size(); ++k) {
    const long long b = free_[k].first, l = free_[k].second;
    const long long a = (b + align - 1) / align * align;
    if (a + len > b + l) continue;
    std::vector<std::pair<int, int>> keep;
    if (a > b) keep.push_back({(int)b, (int)(a - b)});
    if (a + len < b + l) keep.push_back({(int)(a + len), (int)(b + l - a - len)});
    free_.erase(free_.begin() + k);
    free_.insert(free_.begin() + k, keep.begin(), keep.end());
    return (int)a;
  }
  return -1;
}

void RangeAlloc::give(int begin, int len) {
  if (len <= 0) return;
  auto it = std::lower_bound(free_.begin(), free_.end(), std::make_pair(begin, 0));
  size_t k = it - free_.begin();
  free_.insert(it, {begin, len});
  if (k + 1 < free_.size() && free_[k].first + free_[k].second == free_[k + 1].first) {
    free_[k].second += free_[k + 1].second;
    free_.erase(free_.begin() + k + 1);
  }
  if (k > 0 && free_[k - 1].first + free_[k - 1].second == free_[k].first) {
    free_[k - 1].second += free_[k].second;
    free_.erase(free_.begin() + k);
  }
}

__global__ void k_fill_u16(int n, uint16_t* __restrict__ a, uint16_t v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

// Rows [i0, i0 + cnt) of the current list as 1-based end pointers of the
// system's own CSR (first entry = the pairs before its first row).
__global__ void k_rows_local(int i0, int cnt, const int* __restrict__ row_end, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  const int base = i0 ? row_end[i0 - 1] : 0;
  out[i] = row_end[i0 + i] - base + 1;
}

__global__ void k_nbrs_local(int cnt, const int* __restrict__ nbrs, int shift, int* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < cnt) out[c] = nbrs[c] - shift + 1;
}

static bool same_kind(const dem_params& a, const dem_params& b) {
  const int ca = a.collision_array_max > 0 ? a.collision_array_max : 8;
  const int cb = b.collision_array_max > 0 ? b.collision_array_max : 8;
  return a.coll_model == b.coll_model && a.intg_method == b.intg_method &&
         (a.force_precision == DEM_PREC_SPLIT) == (b.force_precision == DEM_PREC_SPLIT) && ca == cb;
}

static int upload_table(dem_handle* h, int s) {
  // pageable source: the copy is staged before the call returns, so the
  // host block can change afterwards
  return check_cuda(h, cudaMemcpyAsync(h->d_sys + s, &h->sys[s].dp, sizeof(DevParams), cudaMemcpyHostToDevice,
                                       h->stream), "system table");
}

// Rebuild mask of the next event: started systems by their own NN rule, the
// systems starting now 2 (first build, no history), and every slot without a
// running system 2 as well (its rows are rebuilt from scratch: empty for an
// empty slot, never carried over from an earlier occupant of its range).
static bool due_mask(dem_handle* h, std::vector<uint8_t>& m, const std::vector<int>* starting) {
  const int S = (int)h->sys.size();
  m.assign(S, 0);
  bool any = false;
  for (int s = 0; s < S; ++s) {
    const SysSlot& q = h->sys[s];
    if (!q.live || !q.started) { m[s] = 2; continue; }
    if (starting) continue;
    const int nsn = q.prm.neighbor_search_n;
    if (q.nn == 1 || q.nn % nsn == 0) { m[s] = 1; any = true; }
  }
  if (starting)
    for (int s : *starting) { m[s] = 2; any = true; }
  return any;
}

static int upload_due(dem_handle* h, const std::vector<uint8_t>& m) {
  return check_cuda(h, cudaMemcpyAsync(h->d_due, m.data(), m.size(), cudaMemcpyHostToDevice, h->stream), "due mask");
}

// After a rebuild event every empty slot's rows are gone (its particles are
// NONEXISTENT and it was rebuilt), so its id can be given out again.
static void mark_clean(dem_handle* h) {
  for (SysSlot& q : h->sys)
    if (!q.live) q.clean = true;
}

// Rebuild event of the empty slots only (the running systems keep their
// rows), to free the ids of removed systems.
static int clean_slots(dem_handle* h) {
  std::vector<uint8_t> m;
  due_mask(h, m, nullptr);
  for (size_t s = 0; s < m.size(); ++s)
    if (h->sys[s].live && h->sys[s].started) m[s] = 0;
  if (int rc = upload_due(h, m)) return rc;
  if (int rc = run_desgrid_pic(h, true)) return rc;
  if (int rc = run_neighbour(h, true)) return rc;
  mark_clean(h);
  return 0;
}

static int total_facets(const dem_handle* h) {
  int nf = 0;
  for (const SysSlot& q : h->sys) if (q.live) nf += q.nf;
  return nf;
}

#define SYS_GUARD(h, s)                                                                   \
  do {                                                                                    \
    if (!(h)) return DEM_ERR_ARG;                                                         \
    cudaSetDevice((h)->dev);                                                              \
    if (!(h)->batch()) return set_err((h), DEM_ERR_ARG, "not a batch handle");            \
    if ((s) < 0 || (s) >= (int)(h)->sys.size() || !(h)->sys[(s)].live)                    \
      return set_err((h), DEM_ERR_ARG, "no such system in the batch");                    \
  } while (0)

// The extent of the live systems' particle and search-cell ranges, which the
// step kernels cover (ranges are taken first-fit from the low end, so the
// extent follows what is running, not the capacity).
static void update_extent(dem_handle* h) {
  int np = 0, nf = 0;
  for (const SysSlot& S : h->sys) {
    if (!S.live) continue;
    np = std::max(np, S.dp.p_end);
    nf = std::max(nf, S.dp.fcell_off + S.dp.nfcell);
  }
  h->n_act = std::min(h->n, std::max(np, 64));
  h->nfc_act = std::min(h->nfcell_total, std::max(nf, 1));
}

// The tables of a batch handle past handle_arrays, each given to
// A(&pointer, bytes) as in handle_arrays.
template <class F>
static void batch_arrays(dem_handle* h, const dem_batch_limits* lim, F&& A) {
  A((void**)&h->d_sys, sizeof(DevParams) * lim->max_systems);
  A((void**)&h->sys_of, sizeof(uint16_t) * (size_t)lim->max_particles);
  A((void**)&h->d_due, 3 * (size_t)lim->max_systems);
  A((void**)&h->d_first_rogue, sizeof(int) * lim->max_systems);
  A((void**)&h->vertex, sizeof(double) * 9 * (size_t)lim->max_facets);
  A((void**)&h->norm_face, sizeof(double) * 3 * (size_t)lim->max_facets);
  A((void**)&h->ignore_edge, (size_t)4 * lim->max_facets);
  A((void**)&h->fbin, sizeof(FacetBinEntry) * (size_t)lim->max_facet_bins);
}

static bool limits_ok(const dem_params* q, const dem_batch_limits* lim) {
  return lim->max_particles > 0 && lim->max_particles <= MAX_PARTICLES && lim->max_systems > 0 &&
         lim->max_systems <= 65535 && lim->max_cells > 0 && lim->max_search_cells > 0 && lim->max_facets >= 0 &&
         lim->max_facet_bins >= 0 && lim->pairs_per_particle >= 0 && q->n_phases >= 1 &&
         q->n_phases <= DEM_MAX_PHASES && q->dtsolid > 0.0;
}

// Pair-list room a batch handle starts with.
static long long batch_pair_reserve(const dem_batch_limits* lim) {
  const long long per = lim->pairs_per_particle > 0 ? lim->pairs_per_particle : 6;
  return per * (long long)lim->max_particles + 1024;
}

}  // namespace demb

extern "C" {

int dem_params_cells(const dem_params* q, int32_t* des_cells, int32_t* search_cells) {
  if (!q || !des_cells || !search_cells) return DEM_ERR_ARG;
  if (!des_grid_ok(*q)) return DEM_ERR_ARG;
  DevParams dp;
  fill_devparams(*q, 1, dp);
  *des_cells = dp.ncell2 + 1;
  *search_cells = dp.nfcell;
  return 0;
}

int dem_batch_footprint(const dem_params* q, const dem_batch_limits* lim, dem_memory* out) {
  if (!q || !lim || !out) return DEM_ERR_ARG;
  if (!limits_ok(q, lim)) return DEM_ERR_ARG;
  dem_handle tmp;
  tmp.prm = *q;
  tmp.n = lim->max_particles;
  tmp.sys.resize(lim->max_systems);  // a batch: its arrays, not a single handle's
  fill_devparams(tmp.prm, tmp.n, tmp.dp);
  long long bytes = 0;
  auto S = [&](void**, size_t b) { bytes += (long long)(b > 0 ? b : 8); };
  handle_arrays(&tmp, (size_t)tmp.n, (size_t)lim->max_cells, (size_t)lim->max_search_cells, S);
  batch_arrays(&tmp, lim, S);
  memset(out, 0, sizeof *out);
  out->array_bytes = bytes;
  out->pair_capacity = batch_pair_reserve(lim);
  out->pair_bytes = pair_array_bytes(out->pair_capacity);
  return 0;
}

int dem_batch_create(const dem_params* q, const dem_batch_limits* lim, dem_handle** out) {
  if (!q || !lim || !out) return DEM_ERR_ARG;
  if (!limits_ok(q, lim)) return DEM_ERR_ARG;
  dem_handle* h = new dem_handle();
  h->prm = *q;
  h->n = lim->max_particles;
  cudaGetDevice(&h->dev);
  fill_devparams(h->prm, h->n, h->dp);
  h->sys.resize(lim->max_systems);
  h->ncell_total = lim->max_cells;
  h->nfcell_total = lim->max_search_cells;
  h->max_facets = lim->max_facets;
  h->max_bins = lim->max_facet_bins;
  int rc = alloc_handle(h, lim->max_cells, lim->max_search_cells, batch_pair_reserve(lim));
  auto A = [&](void** p, size_t bytes) {
    if (rc) return;
    if (cudaMalloc(p, bytes > 0 ? bytes : 8) != cudaSuccess) rc = DEM_ERR_CUDA;
    else cudaMemset(*p, 0, bytes > 0 ? bytes : 8);
    h->arr_bytes += (long long)(bytes > 0 ? bytes : 8);
  };
  batch_arrays(h, lim, A);
  if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = DEM_ERR_CUDA;
  if (rc) {
    dem_destroy(h);
    return rc;
  }
  // every slot starts empty (due 1, table entry of the common kind)
  for (int s = 0; s < lim->max_systems; ++s) {
    h->sys[s].prm = *q;
    h->sys[s].dp = h->dp;
  }
  for (int s = 0; s < lim->max_systems; ++s) upload_table(h, s);
  std::vector<uint8_t> m(lim->max_systems, 1);
  upload_due(h, m);
  h->due_cur = h->d_due;
  h->part_alloc.reset(h->n);
  h->cell_alloc.reset(lim->max_cells);
  h->fcell_alloc.reset(lim->max_search_cells);
  h->fac_alloc.reset(lim->max_facets);
  h->bin_alloc.reset(lim->max_facet_bins);
  update_extent(h);
  h->have_state = true;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
    dem_destroy(h);
    return DEM_ERR_CUDA;
  }
  *out = h;
  return 0;
}

int dem_sys_add(dem_handle* h, const dem_params* q, int32_t max_pip, int32_t* sys) {
  if (!h) return DEM_ERR_ARG;
  cudaSetDevice(h->dev);
  if (!h->batch()) return set_err(h, DEM_ERR_ARG, "not a batch handle");
  if (!q || !sys || max_pip <= 0) return set_err(h, DEM_ERR_ARG, "bad system");
  if (!same_kind(*q, h->prm))
    return set_err(h, DEM_ERR_ARG, "collision model, integrator, force precision and COLLISION_ARRAY_MAX "
                                   "must be the same for all systems of a batch");
  if (q->n_phases < 1 || q->n_phases > DEM_MAX_PHASES || !des_grid_ok(*q) || q->neighbor_search_n < 1 ||
      !(q->dtsolid > 0.0))
    return set_err(h, DEM_ERR_ARG, "bad system parameters");
  for (int a = 0; a < 3; ++a) {
    const int cells = a == 0 ? q->dg_imax : (a == 1 ? q->dg_jmax : q->dg_kmax);
    if (q->periodic[a] && !(a == 2 && q->no_k) && cells < 3) return set_err(h, DEM_ERR_ARG, "periodic axis needs 3 cells");
  }
  // a slot whose id may still label rows of a removed system is reused only
  // after a rebuild event has emptied those rows
  auto find_slot = [&]() {
    for (int s = 0; s < (int)h->sys.size(); ++s)
      if (!h->sys[s].live && (h->sys[s].clean || !h->have_pairs)) return s;
    return -1;
  };
  int id = find_slot();
  if (id < 0) {
    bool any_free = false;
    for (const SysSlot& q : h->sys) any_free = any_free || !q.live;
    if (!any_free) return set_err(h, DEM_ERR_CAPACITY, "all system slots of the batch are in use");
    if (int rc = clean_slots(h)) return rc;
    id = find_slot();
    if (id < 0) return set_err(h, DEM_ERR_STATE, "no clean system slot");
  }
  DevParams dp;
  fill_devparams(*q, h->n, dp);
  const int pb = h->part_alloc.take(max_pip, 64);
  const int cb = pb < 0 ? -1 : h->cell_alloc.take(dp.ncell2 + 1, 1);
  const int fb = cb < 0 ? -1 : h->fcell_alloc.take(dp.nfcell, 1);
  if (pb < 0 || cb < 0 || fb < 0) {
    if (pb >= 0) h->part_alloc.give(pb, max_pip);
    if (cb >= 0) h->cell_alloc.give(cb, dp.ncell2 + 1);
    return set_err(h, DEM_ERR_CAPACITY, "batch particle or cell capacity exhausted");
  }
  dp.p_begin = pb;
  dp.p_end = pb + max_pip;
  dp.cell_off = cb;
  dp.fcell_off = fb;
  SysSlot& S = h->sys[id];
  S = SysSlot();
  S.live = true;
  S.prm = *q;
  S.dp = dp;
  S.cap = max_pip;
  const size_t n = (size_t)max_pip, cm = (size_t)h->dp.cmax;
  const int T = 256;
  k_fill_u16<<<(max_pip + T - 1) / T, T, 0, h->stream>>>(max_pip, h->sys_of + pb, (uint16_t)id);
  h->launches++;
  cudaMemsetAsync(h->state + pb, 0, n, h->stream);
  cudaMemsetAsync(h->wall_live + pb, 0, n, h->stream);
  cudaMemsetAsync(h->wall_fid + pb * cm, 0xff, sizeof(int) * cm * n, h->stream);
  cudaMemsetAsync(h->wall_pft + pb * cm * 3, 0, sizeof(double) * 3 * cm * n, h->stream);
  cudaMemsetAsync(h->fbin_start + cb, 0, sizeof(int) * (dp.ncell2 + 1), h->stream);
  if (int rc = upload_table(h, id)) return rc;
  update_extent(h);
  invalidate_graphs(h);
  *sys = id;
  return check_cuda(h, cudaStreamSynchronize(h->stream), "add system");
}

int dem_sys_remove(dem_handle* h, int32_t s) {
  SYS_GUARD(h, s);
  SysSlot& S = h->sys[s];
  cudaMemsetAsync(h->state + S.dp.p_begin, 0, (size_t)S.cap, h->stream);
  h->part_alloc.give(S.dp.p_begin, S.cap);
  h->cell_alloc.give(S.dp.cell_off, S.dp.ncell2 + 1);
  h->fcell_alloc.give(S.dp.fcell_off, S.dp.nfcell);
  if (S.nf > 0) h->fac_alloc.give(S.fac_off, S.nf);
  if (S.nbin > 0) h->bin_alloc.give(S.bin_off, S.nbin);
  S = SysSlot();
  S.prm = h->prm;
  S.dp = h->dp;
  S.clean = false;
  if (int rc = upload_table(h, s)) return rc;
  h->nf = total_facets(h);
  update_extent(h);
  invalidate_graphs(h);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "remove system");
}

int dem_sys_set_walls(dem_handle* h, int32_t s, const double* vertex, const double* norm_face, int32_t nf) {
  SYS_GUARD(h, s);
  if (nf < 0 || (nf > 0 && (!vertex || !norm_face))) return set_err(h, DEM_ERR_ARG, "bad facet arrays");
  const int rc = run_bin_facets_sys(h, s, vertex, norm_face, nf);
  h->nf = total_facets(h);
  return rc;
}

int dem_sys_upload_state(dem_handle* h, int32_t s, const double* pos, const double* vel, const double* omega,
                         const double* radius, const double* pmass, const double* omoi, const int8_t* state,
                         const int32_t* phase, int32_t max_pip) {
  SYS_GUARD(h, s);
  SysSlot& S = h->sys[s];
  if (max_pip < 0 || max_pip > S.cap) return set_err(h, DEM_ERR_ARG, "more particles than the system reserved");
  if (!radius || !pmass || !omoi || !state || !phase) return set_err(h, DEM_ERR_ARG, "null array");
  cudaMemsetAsync(h->state + S.dp.p_begin, 0, (size_t)S.cap, h->stream);
  if (int rc = upload_range(h, S.dp.p_begin, max_pip, S.prm.n_phases, pos, vel, omega, radius, pmass, omoi,
                            state, phase))
    return rc;
  skin_unknown(h);
  S.have_state = true;
  return 0;
}

int dem_sys_download_state(dem_handle* h, int32_t s, double* pos, double* vel, double* omega, int8_t* state,
                           int32_t max_pip) {
  SYS_GUARD(h, s);
  SysSlot& S = h->sys[s];
  if (max_pip < 0 || max_pip > S.cap) return set_err(h, DEM_ERR_ARG, "more particles than the system reserved");
  return download_range(h, S.dp.p_begin, max_pip, pos, vel, omega, state);
}

// First pair list of the given systems (the tail of MAKE_ARRAYS_DES); the
// running systems keep theirs.  The systems then step from NN = 1.
int dem_sys_start(dem_handle* h, const int32_t* ids, int32_t k) {
  if (!h) return DEM_ERR_ARG;
  cudaSetDevice(h->dev);
  if (!h->batch()) return set_err(h, DEM_ERR_ARG, "not a batch handle");
  if (k < 0 || (k > 0 && !ids)) return set_err(h, DEM_ERR_ARG, "bad system list");
  std::vector<int> starting;
  for (int j = 0; j < k; ++j) {
    const int s = ids[j];
    if (s < 0 || s >= (int)h->sys.size() || !h->sys[s].live) return set_err(h, DEM_ERR_ARG, "no such system in the batch");
    if (!h->sys[s].have_state) return set_err(h, DEM_ERR_STATE, "upload the system's particles first");
    if (h->sys[s].started) return set_err(h, DEM_ERR_STATE, "system already started");
    starting.push_back(s);
  }
  if (starting.empty()) return 0;
  std::vector<uint8_t> m;
  due_mask(h, m, &starting);
  if (int rc = upload_due(h, m)) return rc;
  if (int rc = run_desgrid_pic(h, true)) return rc;
  if (int rc = run_neighbour(h, true)) return rc;
  mark_clean(h);
  for (int s : starting) {
    SysSlot& S = h->sys[s];
    S.started = true;
    S.nn = 1;
    S.first_pass = true;
    S.steps_done = 0;
    S.s_time = 0.0;
  }
  invalidate_graphs(h);
  return fetch_errors(h);
}

// One DES_TIME_STEP of every running system: force + integration in one pass
// over the handle, then the cell binning and the rebuild of the systems that
// are due (each by its own NN).
static int batch_step_once(dem_handle* h, std::vector<uint8_t>& last_due) {
  // FIRST_PASS of the Adams-Bashforth start is per system
  for (int s = 0; s < (int)h->sys.size(); ++s) {
    SysSlot& S = h->sys[s];
    const int fp = (S.live && S.started && S.first_pass) ? 1 : 0;
    if (S.dp.first_pass != fp) {
      S.dp.first_pass = fp;
      if (int rc = upload_table(h, s)) return rc;
    }
  }
  cudaMemsetAsync(&h->derr->n_contacts, 0, 2 * sizeof(unsigned long long), h->stream);
  if (int rc = run_force(h, true)) return rc;
  std::vector<uint8_t> m;
  const bool any_due = due_mask(h, m, nullptr);
  bool anyper = false;
  for (const SysSlot& S : h->sys)
    if (S.live && S.started)
      anyper = anyper || S.dp.per[0] || S.dp.per[1] || (S.dp.per[2] && !S.dp.no_k);
  if (any_due || anyper) {
    if (m != last_due) {
      if (int rc = upload_due(h, m)) return rc;
      last_due = m;
    }
    if (int rc = run_desgrid_pic(h, any_due)) return rc;
    if (any_due) {
      if (int rc = run_neighbour(h, true)) return rc;
      mark_clean(h);
    }
  }
  for (SysSlot& S : h->sys) {
    if (!S.live || !S.started) continue;
    S.s_time = S.s_time + S.prm.dtsolid;
    S.steps_done++;
    S.first_pass = false;
    S.nn++;
  }
  h->steps_done++;
  return 0;
}

// A whole NEIGHBOR_SEARCH_N period of a batch whose running systems are all
// at a period boundary (same NEIGHBOR_SEARCH_N, each at its own NN = m*N + 1
// with m >= 1, past the first Adams-Bashforth step) is the same sequence
// every time: N force passes with the periodic rebinning, the rebuild of all
// of them after the last -- the systems' own step counts do not enter it.
// It is captured once per combination of buffer parities and replayed; the
// two rebuild masks it uses (idle steps, rebuild step) stay in device memory.
static bool period_aligned(const dem_handle* h, int* nsn) {
  int N = -1;
  bool any = false;
  for (const SysSlot& S : h->sys) {
    if (!S.live) continue;
    if (!S.started || S.first_pass) return false;
    if (N < 0) N = S.prm.neighbor_search_n;
    if (S.prm.neighbor_search_n != N || S.nn <= 1 || (S.nn - 1) % N != 0) return false;
    any = true;
  }
  if (!any) return false;
  *nsn = N;
  return true;
}

static int graph_step(dem_handle* h, bool rebuild, bool anyper) {
  cudaMemsetAsync(&h->derr->n_contacts, 0, 2 * sizeof(unsigned long long), h->stream);
  if (int rc = run_force(h, true)) return rc;
  if (rebuild || anyper) {
    const size_t S = h->sys.size();
    h->due_cur = h->d_due + (rebuild ? 2 * S : S);
    int rc = run_desgrid_pic(h, rebuild);
    if (!rc && rebuild) rc = run_neighbour(h, true);
    h->due_cur = h->d_due;
    if (rc) return rc;
  }
  return 0;
}

static int batch_replay_period(dem_handle* h, int N) {
  const long long P = host_pairs(h);
  if (2 * P + 1024 > h->pair_cap) {
    if (int rc = ensure_pair_capacity(h, 2 * P + 1024)) return rc;
    invalidate_graphs(h);
  }
  bool anyper = false;
  for (const SysSlot& S : h->sys)
    if (S.live) anyper = anyper || S.dp.per[0] || S.dp.per[1] || (S.dp.per[2] && !S.dp.no_k);
  const int key = (h->cur << 2) | (h->pcur << 1) | h->rb;
  if (!h->graphs[key]) {
    // the idle-step and rebuild-step masks of this membership
    const size_t S = h->sys.size();
    std::vector<uint8_t> m(2 * S);
    for (size_t s = 0; s < S; ++s) {
      const bool run = h->sys[s].live && h->sys[s].started;
      m[s] = run ? 0 : 2;
      m[S + s] = run ? 1 : 2;
    }
    if (int rc = check_cuda(h, cudaMemcpyAsync(h->d_due + S, m.data(), 2 * S, cudaMemcpyHostToDevice, h->stream),
                            "period masks")) return rc;
    if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sync")) return rc;
    cudaGraph_t graph;
    h->capturing = true;
    if (int rc = check_cuda(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "begin capture")) {
      h->capturing = false;
      return rc;
    }
    const int cur0 = h->cur, pcur0 = h->pcur, rb0 = h->rb;
    const long long l0 = h->launches;
    int rc = 0;
    for (int j = 0; j < N && !rc; ++j) rc = graph_step(h, j == N - 1, anyper);
    cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
    h->capturing = false;
    h->cur = cur0; h->pcur = pcur0; h->rb = rb0;
    const long long kernels = h->launches - l0;
    h->launches = l0;
    if (rc) return rc;
    if (int r2 = check_cuda(h, ce, "end capture")) return r2;
    cudaGraphExec_t exec;
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (int r2 = check_cuda(h, ce, "graph instantiate")) return r2;
    h->graphs[key] = exec;
    h->graph_kernels[key] = kernels;
  }
  if (int rc = check_cuda(h, cudaGraphLaunch(h->graphs[key], h->stream), "graph launch")) return rc;
  h->launches += h->graph_kernels[key];
  for (int j = 0; j < N; ++j) h->cur = 1 - h->cur;
  h->pcur = 1 - h->pcur;
  h->rb = 1 - h->rb;
  h->np_stale = true;
  h->steps_done += N;
  for (SysSlot& S : h->sys) {
    if (!S.live) continue;
    for (int j = 0; j < N; ++j) S.s_time = S.s_time + S.prm.dtsolid;
    S.steps_done += N;
    S.nn += N;
  }
  mark_clean(h);
  return 0;
}

int dem_batch_step(dem_handle* h, int32_t nsteps) {
  if (!h) return DEM_ERR_ARG;
  cudaSetDevice(h->dev);
  if (!h->batch()) return set_err(h, DEM_ERR_ARG, "not a batch handle");
  if (nsteps < 0) return set_err(h, DEM_ERR_ARG, "bad step count");
  for (const SysSlot& S : h->sys)
    if (S.live && S.have_state && !S.started)
      return set_err(h, DEM_ERR_STATE, "a system with particles has not been started");
  if (!h->have_pairs) return set_err(h, DEM_ERR_STATE, "no system started");
  const bool graphs_ok = h->stream != nullptr && !h->prof && !h->no_graphs;
  std::vector<uint8_t> last_due;
  int k = 0;
  while (k < nsteps) {
    int N = 0;
    if (graphs_ok && period_aligned(h, &N) && nsteps - k >= N) {
      if (int rc = batch_replay_period(h, N)) return rc;
      last_due.clear();
      k += N;
    } else {
      if (int rc = batch_step_once(h, last_due)) return rc;
      ++k;
    }
  }
  return fetch_errors(h);
}

int dem_sys_get_stats(dem_handle* h, int32_t s, dem_stats* st) {
  SYS_GUARD(h, s);
  if (!st) return DEM_ERR_ARG;
  SysSlot& S = h->sys[s];
  memset(st, 0, sizeof *st);
  if (int rc = stats_range(h, S.dp.p_begin, S.cap, st)) return rc;
  if (S.started) {
    int e[2] = {0, 0};
    const int* re = h->row_end[h->rb];
    if (S.dp.p_begin > 0) cudaMemcpyAsync(&e[0], re + S.dp.p_begin - 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(&e[1], re + S.dp.p_end - 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "system pairs")) return rc;
    st->n_pairs = e[1] - e[0];
  }
  st->steps_done = S.steps_done;
  st->s_time = S.s_time;
  return 0;
}

int dem_sys_download_pairs(dem_handle* h, int32_t s, int32_t* ni, int32_t* nb, double* pf, int64_t cap,
                           int32_t max_pip) {
  SYS_GUARD(h, s);
  SysSlot& S = h->sys[s];
  if (!S.started) return set_err(h, DEM_ERR_STATE, "system not started");
  if (max_pip < 0 || max_pip > S.cap) return set_err(h, DEM_ERR_ARG, "more particles than the system reserved");
  if (max_pip == 0) return 0;
  const int* re = h->row_end[h->rb];
  int e[2] = {0, 0};
  if (S.dp.p_begin > 0) cudaMemcpyAsync(&e[0], re + S.dp.p_begin - 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(&e[1], re + S.dp.p_begin + max_pip - 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "system pairs")) return rc;
  const long long P = e[1] - e[0];
  if ((nb || pf) && cap < P) return set_err(h, DEM_ERR_CAPACITY, "pair capacity too small");
  int* tmp = (int*)stage_buffer(h, sizeof(int) * ((size_t)max_pip + (size_t)P) + 64);
  if (!tmp) return set_err(h, DEM_ERR_CUDA, "cudaMalloc stage");
  const int T = 256;
  k_rows_local<<<(max_pip + T - 1) / T, T, 0, h->stream>>>(S.dp.p_begin, max_pip, re, tmp);
  h->launches++;
  if (P > 0) {
    k_nbrs_local<<<(unsigned)((P + T - 1) / T), T, 0, h->stream>>>((int)P, h->nbrs[h->rb] + e[0], S.dp.p_begin,
                                                                   tmp + max_pip);
    h->launches++;
  }
  if (ni) cudaMemcpyAsync(ni, tmp, sizeof(int) * max_pip, cudaMemcpyDeviceToHost, h->stream);
  if (nb && P) cudaMemcpyAsync(nb, tmp + max_pip, sizeof(int) * P, cudaMemcpyDeviceToHost, h->stream);
  if (pf && P) cudaMemcpyAsync(pf, h->pft[h->pcur] + 3 * (size_t)e[0], sizeof(double) * 3 * P, cudaMemcpyDeviceToHost, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "download system pairs");
}

int dem_sys_info(dem_handle* h, int32_t s, dem_sys_status* out) {
  SYS_GUARD(h, s);
  if (!out) return DEM_ERR_ARG;
  const SysSlot& S = h->sys[s];
  memset(out, 0, sizeof *out);
  out->capacity = S.cap;
  out->started = S.started ? 1 : 0;
  out->next_nn = S.nn;
  out->particle_offset = S.dp.p_begin;
  out->steps_done = S.steps_done;
  out->s_time = S.s_time;
  return 0;
}

}  // extern "C"
