// capi.cu -- the C ABI of include/dem_b200.h.
//
// Owns device allocation, host<->device conversion between the Fortran
// layouts of the DES arrays and the packed device layout, and the
// DES_TIME_STEP sequence (model/des/des_time_march.f:342-432).
#include "dem_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

using namespace demb;

namespace demb {

int set_err(dem_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int check_cuda(dem_handle* h, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return 0;
  char b[256];
  snprintf(b, sizeof b, "%s: %s", what, cudaGetErrorString(e));
  return set_err(h, DEM_ERR_CUDA, b);
}

// Packs Fortran (n,3) columns + scalars into double4 arrays.
__global__ void k_pack(int n, const double* __restrict__ v3, const double* __restrict__ s, double4* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_double4(v3[i], v3[(size_t)n + i], v3[2 * (size_t)n + i], s ? s[i] : 0.0);
}
__global__ void k_pack_keepw(int n, const double* __restrict__ v3, double4* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 o = out[i];
  out[i] = make_double4(v3[i], v3[(size_t)n + i], v3[2 * (size_t)n + i], o.w);
}
// Positions of a motion-only upload: as k_pack_keepw, and each existing
// particle's move notes its length in the displacement bound's slots, so
// the bound (pair and wall gaps, candidate list) stays valid without a
// rebuild.
__global__ void k_pack_moved(int n, const double* __restrict__ v3, double4* __restrict__ out,
                             const int8_t* __restrict__ state, unsigned* __restrict__ vslot) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 o = out[i];
  const double x = v3[i], y = v3[(size_t)n + i], z = v3[2 * (size_t)n + i];
  out[i] = make_double4(x, y, z, o.w);
  if (state[i] != DEM_STATE_NONEXISTENT) {
    const double dx = x - o.x, dy = y - o.y, dz = z - o.z;
    note_displacement(vslot, sqrt(dx * dx + dy * dy + dz * dz));
  }
}
__global__ void k_unpack(int n, const double4* __restrict__ in, double* __restrict__ v3) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 a = in[i];
  v3[i] = a.x; v3[(size_t)n + i] = a.y; v3[2 * (size_t)n + i] = a.z;
}
__global__ void k_phase_in(int n, const int* __restrict__ ph, const int8_t* __restrict__ st, uint8_t* __restrict__ out,
                           int nph, unsigned* __restrict__ bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int p = ph[i] - 1;
  if (st[i] != DEM_STATE_NONEXISTENT && (p < 0 || p >= nph)) { atomicOr(bad, 1u); p = 0; }
  out[i] = (uint8_t)(p < 0 ? 0 : p);
}

// Per-block partial sums for statistics; the host adds the partials in
// block order, so the result is deterministic.
constexpr int STAT_T = 256;
__global__ void k_stats1(int n, const double4* __restrict__ pos4, const double4* __restrict__ vel4,
                         const int8_t* __restrict__ state, double* __restrict__ part) {
  __shared__ double sh[8][STAT_T];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (i < n && state[i] == DEM_STATE_NORMAL) {
    double4 p = pos4[i], u = vel4[i];
    v[0] = 1.0; v[1] = u.x; v[2] = u.y; v[3] = u.z;
    v[4] = u.w; v[5] = u.w * p.y;
    v[6] = 0.5 * u.w * (u.x * u.x + u.y * u.y + u.z * u.z);
    v[7] = 0.0;
  }
  for (int k = 0; k < 8; ++k) sh[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int s = STAT_T / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) for (int k = 0; k < 8; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) for (int k = 0; k < 8; ++k) part[(size_t)blockIdx.x * 8 + k] = sh[k][0];
}
__global__ void k_stats2(int n, const double4* __restrict__ vel4, const int8_t* __restrict__ state,
                         double mx, double my, double mz, double* __restrict__ part) {
  __shared__ double sh[3][STAT_T];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[3] = {0, 0, 0};
  if (i < n && state[i] == DEM_STATE_NORMAL) {
    double4 u = vel4[i];
    v[0] = (u.x - mx) * (u.x - mx); v[1] = (u.y - my) * (u.y - my); v[2] = (u.z - mz) * (u.z - mz);
  }
  for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int s = STAT_T / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) for (int k = 0; k < 3; ++k) part[(size_t)blockIdx.x * 3 + k] = sh[k][0];
}

int fetch_errors(dem_handle* h) {
  if (int rc = check_cuda(h, cudaMemcpyAsync(h->herr, h->derr, sizeof(DevErr), cudaMemcpyDeviceToHost, h->stream), "copy err")) return rc;
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sync")) return rc;
  unsigned f = h->herr->flags;
  if (!f) return 0;
  // clear the flags for the next call
  unsigned z = 0;
  cudaMemcpyAsync(&h->derr->flags, &z, sizeof(unsigned), cudaMemcpyHostToDevice, h->stream);
  cudaStreamSynchronize(h->stream);
  char b[200];
  if (f & EF_ZERO_DIST) {
    snprintf(b, sizeof b, "distance between particles is zero: %d %d", h->herr->zero_a + 1, h->herr->zero_b + 1);
    return set_err(h, DEM_ERR_ZERO_DISTANCE, b);
  }
  if (f & EF_WALL_SLOTS) return set_err(h, DEM_ERR_WALL_SLOTS, "Error: COLLISION_ARRAY_MAX too small.");
  if (f & EF_ROGUE_FATAL) return set_err(h, DEM_ERR_ROGUE, "NORMAL particle found in GHOST cell (remove_rogue = 0)");
  if (f & EF_PAIR_CAP) return set_err(h, DEM_ERR_PAIR_OVERFLOW, "pair list capacity exceeded");
  if (f & EF_INFLOW_CAP) return set_err(h, DEM_ERR_CAPACITY, "no NONEXISTENT slot left for an inflow particle (MAX_PIP)");
  return set_err(h, DEM_ERR_STATE, "device error flags set");
}

void invalidate_graphs(dem_handle* h) {
  for (auto& g : h->graphs) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

void* stage_buffer(dem_handle* h, size_t bytes) {
  if (bytes > h->stage_bytes) {
    if (h->stage) cudaFree(h->stage);
    h->stage = nullptr;
    h->stage_bytes = 0;
    if (cudaMalloc(&h->stage, bytes) != cudaSuccess) return nullptr;
    h->stage_bytes = bytes;
  }
  return h->stage;
}

static cudaEvent_t pool_event(dem_handle* h) {
  if (!h->ev_pool.empty()) { cudaEvent_t e = h->ev_pool.back(); h->ev_pool.pop_back(); return e; }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

ProfScope::ProfScope(dem_handle* hh, int cls) : h(hh) {
  if (!h->prof || (cls >= DEM_PROF_WALLS && h->prof < 2)) return;
  dem_handle::ProfEv ev{cls, pool_event(h), pool_event(h)};
  cudaEventRecord(ev.a, h->stream);
  h->prof_pending.push_back(ev);
  idx = (int)h->prof_pending.size() - 1;
}
ProfScope::~ProfScope() {
  if (idx < 0) return;
  cudaEventRecord(h->prof_pending[idx].b, h->stream);
}

static void prof_collect(dem_handle* h) {
  if (h->prof_pending.empty()) return;
  cudaStreamSynchronize(h->stream);
  for (auto& e : h->prof_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
      h->prof_ms[e.cls] += ms;
      h->prof_n[e.cls] += 1;
    }
    h->ev_pool.push_back(e.a);
    h->ev_pool.push_back(e.b);
  }
  h->prof_pending.clear();
}


// Particles [off, off + cnt) from Fortran-layout host arrays with cnt rows.
int upload_range(dem_handle* h, int off, int cnt, int nph, const double* pos, const double* vel,
                 const double* omega, const double* radius, const double* pmass, const double* omoi,
                 const int8_t* state, const int32_t* phase, bool note_moves) {
  // radius, pmass, omoi, state and phase may be NULL: the device keeps its
  // values of those (the callers check that there are some); note_moves
  // (with radius and state NULL) notes the moves in the displacement slots
  if (!pos || !vel || !omega) return set_err(h, DEM_ERR_ARG, "null array");
  if (cnt <= 0) return 0;
  const size_t n = (size_t)cnt;
  // one staging block: pos(3n) vel(3n) omega(3n) r(n) m(n) omoi(n) + phase(n ints) + flag
  double* st = (double*)stage_buffer(h, sizeof(double) * 12 * n + sizeof(int) * n + 64);
  if (!st) return set_err(h, DEM_ERR_CUDA, "cudaMalloc stage");
  const int T = 256, B = (int)((n + T - 1) / T);
  const int c = h->cur;
  const double* src[3] = {pos, vel, omega};
  const double* scal[3] = {radius, pmass, omoi};
  double4* dst[3] = {h->pos4[c] + off, h->vel4[c] + off, h->omg4[c] + off};
  for (int a = 0; a < 3; ++a) {
    cudaMemcpyAsync(st + 3 * n * a, src[a], sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream);
    if (scal[a]) {
      cudaMemcpyAsync(st + 9 * n + n * a, scal[a], sizeof(double) * n, cudaMemcpyHostToDevice, h->stream);
      k_pack<<<B, T, 0, h->stream>>>(cnt, st + 3 * n * a, st + 9 * n + n * a, dst[a]);
    } else if (a == 0 && note_moves && !state) {
      k_pack_moved<<<B, T, 0, h->stream>>>(cnt, st, dst[0], h->state + off, h->vslot);
    } else {
      k_pack_keepw<<<B, T, 0, h->stream>>>(cnt, st + 3 * n * a, dst[a]);
    }
    h->launches++;
  }
  if (state) cudaMemcpyAsync(h->state + off, state, n, cudaMemcpyHostToDevice, h->stream);
  unsigned hb = 0;
  if (phase) {
    int* ph = (int*)(st + 12 * n);
    unsigned* bad = (unsigned*)(ph + n);
    cudaMemcpyAsync(ph, phase, sizeof(int) * n, cudaMemcpyHostToDevice, h->stream);
    cudaMemsetAsync(bad, 0, sizeof(unsigned), h->stream);
    k_phase_in<<<B, T, 0, h->stream>>>(cnt, ph, h->state + off, h->phase + off, nph, bad);
    h->launches++;
    cudaMemcpyAsync(&hb, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream);
  }
  // the host arrays may be reused when the call returns
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "upload")) return rc;
  if (hb) return set_err(h, DEM_ERR_ARG, "phase out of range");
  return 0;
}

// Particles [off, off + cnt) into Fortran-layout host arrays with cnt rows.
int download_range(dem_handle* h, int off, int cnt, double* pos, double* vel, double* omega, int8_t* state) {
  if (cnt <= 0) return 0;
  const size_t n = (size_t)cnt;
  double* st = (double*)stage_buffer(h, sizeof(double) * 12 * n + sizeof(int) * n + 64);
  if (!st) return set_err(h, DEM_ERR_CUDA, "cudaMalloc stage");
  const int T = 256, B = (int)((n + T - 1) / T);
  const int c = h->cur;
  k_unpack<<<B, T, 0, h->stream>>>(cnt, h->pos4[c] + off, st);
  k_unpack<<<B, T, 0, h->stream>>>(cnt, h->vel4[c] + off, st + 3 * n);
  k_unpack<<<B, T, 0, h->stream>>>(cnt, h->omg4[c] + off, st + 6 * n);
  h->launches += 3;
  if (pos) cudaMemcpyAsync(pos, st, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream);
  if (vel) cudaMemcpyAsync(vel, st + 3 * n, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream);
  if (omega) cudaMemcpyAsync(omega, st + 6 * n, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream);
  if (state) cudaMemcpyAsync(state, h->state + off, n, cudaMemcpyDeviceToHost, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "download");
}

// Kinematic statistics of particles [off, off + cnt): NORMAL count, mean
// velocity, granular temperature, kinetic energy and bed height.
int stats_range(dem_handle* h, int off, int cnt, dem_stats* s) {
  const int T = STAT_T, B = (cnt + T - 1) / T;
  if (B > 0 && h->red_elems < 8 * B) {
    if (h->red) cudaFree(h->red);
    h->red = nullptr;
    h->red_elems = 0;
    if (int rc = check_cuda(h, cudaMalloc(&h->red, sizeof(double) * 8 * B), "cudaMalloc")) return rc;
    h->red_elems = 8 * B;
  }
  std::vector<double> part((size_t)8 * B);
  double sum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (B > 0) {
    k_stats1<<<B, T, 0, h->stream>>>(cnt, h->pos4[h->cur] + off, h->vel4[h->cur] + off, h->state + off, h->red);
    h->launches++;
    cudaMemcpyAsync(part.data(), h->red, sizeof(double) * 8 * B, cudaMemcpyDeviceToHost, h->stream);
    if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "stats")) return rc;
    for (int b = 0; b < B; ++b) for (int k = 0; k < 8; ++k) sum[k] += part[(size_t)8 * b + k];
  }
  const double nn = sum[0];
  double mv[3] = {0, 0, 0};
  if (nn > 0) for (int c = 0; c < 3; ++c) mv[c] = sum[1 + c] / nn;
  double gt[3] = {0, 0, 0};
  if (B > 0) {
    k_stats2<<<B, T, 0, h->stream>>>(cnt, h->vel4[h->cur] + off, h->state + off, mv[0], mv[1], mv[2], h->red);
    h->launches++;
    cudaMemcpyAsync(part.data(), h->red, sizeof(double) * 3 * B, cudaMemcpyDeviceToHost, h->stream);
    if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "stats")) return rc;
    for (int b = 0; b < B; ++b) for (int k = 0; k < 3; ++k) gt[k] += part[(size_t)3 * b + k];
  }
  s->n_normal = (int64_t)nn;
  for (int c = 0; c < 3; ++c) { s->mean_vel[c] = mv[c]; s->gran_temp[c] = nn > 0 ? gt[c] / nn : 0.0; }
  s->kinetic_energy = sum[6];
  s->bed_height = sum[4] > 0 ? sum[5] / sum[4] : 0.0;
  return 0;
}

}  // namespace demb

// Interior DES cells per axis at least 1 and, with the ghost layers, within
// the packed (i, j, k) of the pair build; at most MAX_GRID_CELLS cells in
// all, so that every cell index fits an int.
bool demb::des_grid_ok(const dem_params& q) {
  if (q.dg_imax < 1 || q.dg_jmax < 1 || (!q.no_k && q.dg_kmax < 1)) return false;
  if (!(q.dg_imax + 2 <= DG_MAX_IK && q.dg_jmax + 2 <= DG_MAX_J && (q.no_k || q.dg_kmax + 2 <= DG_MAX_IK)))
    return false;
  const long long cells = (long long)(q.dg_imax + 2) * (q.dg_jmax + 2) * (q.no_k ? 1 : q.dg_kmax + 2);
  return cells <= MAX_GRID_CELLS;
}

void demb::fill_devparams(const dem_params& q, int n, DevParams& p) {
  memset(&p, 0, sizeof p);
  p.n = n;
  p.coll = q.coll_model; p.intg = q.intg_method; p.nph = q.n_phases; p.no_k = q.no_k;
  p.cmax = q.collision_array_max > 0 ? q.collision_array_max : 8;
  p.remove_rogue = q.remove_rogue;
  p.prec = q.force_precision == DEM_PREC_SPLIT ? DEM_PREC_SPLIT : DEM_PREC_FP64;
  for (int a = 0; a < 3; ++a) {
    p.per[a] = q.periodic[a] ? 1 : 0;
    p.grav[a] = q.grav[a];
    p.lo[a] = q.domain_lo[a]; p.hi[a] = q.domain_hi[a];
    p.L[a] = q.domain_hi[a] - q.domain_lo[a];
    p.inv_L[a] = 1.0 / p.L[a];
  }
  // desgrid_init for one rank (desgrid_mod.f:571-604, 780-850)
  p.istart1 = 2; p.iend1 = q.dg_imax + 1; p.istart2 = 1; p.iend2 = q.dg_imax + 2;
  p.jstart1 = 2; p.jend1 = q.dg_jmax + 1; p.jstart2 = 1; p.jend2 = q.dg_jmax + 2;
  if (q.no_k) { p.kstart1 = p.kend1 = p.kstart2 = p.kend2 = 1; }
  else { p.kstart1 = 2; p.kend1 = q.dg_kmax + 1; p.kstart2 = 1; p.kend2 = q.dg_kmax + 2; }
  p.c1 = p.jend2 - p.jstart2 + 1;
  p.c2 = p.c1 * (p.iend2 - p.istart2 + 1);
  p.c3 = -p.c1 * p.istart2 - p.c2 * p.kstart2 - p.jstart2 + 1;
  p.ncell2 = (p.iend2 - p.istart2 + 1) * (p.jend2 - p.jstart2 + 1) * (p.kend2 - p.kstart2 + 1);
  p.dt = q.dtsolid;
  p.kn = q.kn; p.kt = q.kt; p.kn_w = q.kn_w; p.kt_w = q.kt_w;
  p.mew = q.mew; p.mew_w = q.mew_w; p.mew_r = q.mew_r; p.mew_rw = q.mew_rw;
  p.factor_rlm = q.factor_rlm; p.max_radius = q.max_radius;
  p.dg_start[0] = q.dg_xstart; p.dg_start[1] = q.dg_ystart; p.dg_start[2] = q.dg_zstart;
  p.dg_inv[0] = q.dg_dxinv; p.dg_inv[1] = q.dg_dyinv; p.dg_inv[2] = q.dg_dzinv;
  for (int k = 0; k < MAXP * MAXP; ++k) {
    p.etan[k] = q.des_etan[k]; p.etat[k] = q.des_etat[k]; p.hkn[k] = q.hert_kn[k]; p.hkt[k] = q.hert_kt[k];
  }
  for (int k = 0; k < MAXP; ++k) {
    p.etanw[k] = q.des_etan_wall[k]; p.etatw[k] = q.des_etat_wall[k];
    p.hkwn[k] = q.hert_kwn[k]; p.hkwt[k] = q.hert_kwt[k];
  }
  for (int k = 0; k < MAXP * MAXP; ++k) {
    p.hkn32[k] = (float)p.hkn[k]; p.hkt32[k] = (float)p.hkt[k];
    p.etan_sq32[k] = (float)(p.etan[k] * std::sqrt(std::max(p.hkn[k], 0.0)));
    p.etat_sq32[k] = (float)(p.etat[k] * std::sqrt(std::max(p.hkt[k], 0.0)));
    p.etan32[k] = (float)p.etan[k]; p.etat32[k] = (float)p.etat[k];
  }
  p.kn32 = (float)p.kn; p.kt32 = (float)p.kt; p.mew32 = (float)p.mew;
  // Search grid for the pair build: cells about half the largest search
  // diameter 2*FACTOR_RLM*MAX_RADIUS wide (1 % margin); each particle scans
  // the cells within its own reach FACTOR_RLM*(r + MAX_RADIUS), so a small
  // particle among large ones scans few.  The reference's own DES-grid
  // stencil (reduced to the nearer cells when the DES cells are wider than
  // the search diameter) is applied to the candidates afterwards.  An axis
  // keeps the DES grid's division when that is not coarser.  The grid is an
  // acceleration structure, so it may be coarser than that and stay exact:
  // its cell count is held to max(DES cells, SEARCH_CELLS_CAP) (small
  // spheres in a large box would otherwise ask for billions of cells),
  // scaling every refined axis down together.  The bound depends on the
  // system's grid alone, so batch limits sized from the parameters
  // (dem_params_cells) fit the system when it is added.
  const int dgn[3] = {q.dg_imax, q.dg_jmax, q.no_k ? 1 : q.dg_kmax};
  const double target = q.factor_rlm * q.max_radius * 1.01;
  double len[3], want[3];
  for (int a = 0; a < 3; ++a) {
    len[a] = (double)dgn[a] / p.dg_inv[a];
    want[a] = (a == 2 && q.no_k) ? (double)dgn[a] : std::max((double)dgn[a], std::floor(len[a] / target));
  }
  const long long ndes = (long long)(dgn[0] + 2) * (dgn[1] + 2) * (q.no_k ? 1 : dgn[2] + 2);
  const long long cap = std::min<long long>(MAX_GRID_CELLS, std::max<long long>(ndes, SEARCH_CELLS_CAP));
  for (int it = 0; it < 64; ++it) {
    const double cells = (want[0] + 2) * (want[1] + 2) * (q.no_k ? 1.0 : want[2] + 2);
    if (cells <= (double)cap) break;
    const double sc = std::max(0.5, std::cbrt((double)cap / cells) * 0.99);
    bool shrunk = false;
    for (int a = 0; a < 3; ++a) {
      if ((a == 2 && q.no_k) || want[a] <= dgn[a]) continue;
      want[a] = std::max((double)dgn[a], std::floor(want[a] * sc));
      shrunk = true;
    }
    if (!shrunk) break;
  }
  for (int a = 0; a < 3; ++a) {
    int nfa = (int)want[a];
    if (nfa <= dgn[a] || (a == 2 && q.no_k)) nfa = dgn[a];
    if (nfa < 1) nfa = 1;
    p.fn[a] = nfa;
    // same division as the DES grid -> the same inverse width, bit for bit
    p.f_inv[a] = nfa == dgn[a] ? p.dg_inv[a] : (double)nfa / len[a];
  }
  p.fc1 = p.fn[1] + 2;
  p.fc2 = p.fc1 * (p.fn[0] + 2);
  p.nfcell = p.fc2 * (q.no_k ? 1 : p.fn[2] + 2);
}

// ---- scratch of dem_get_stats_noalloc --------------------------------------
// Per-block partial sums of the two statistics passes (8 columns for the
// first, 3 for the second), followed by the 8 block-ordered totals.  The
// array is static device memory of the library: every GPU that loads it
// holds STATS_SCRATCH_DOUBLES * 8 bytes (2 MiB for 2^23 particles) until the
// process exits.  All calls on a device share it and it keeps what the last
// call left there; nothing in it has to start at zero, because each call
// writes every element it reads earlier on the same stream.
constexpr int STATS_NOALLOC_BLOCKS = (DEM_STATS_NOALLOC_MAX_PARTICLES + STAT_T - 1) / STAT_T;
constexpr size_t STATS_TOTAL_OFF = (size_t)8 * STATS_NOALLOC_BLOCKS;
constexpr size_t STATS_SCRATCH_DOUBLES = STATS_TOTAL_OFF + 8;
static __device__ __align__(256) double g_stats_scratch[STATS_SCRATCH_DOUBLES];

// Adds the partials of nb blocks in block order (the order dem_get_stats
// adds them on the host), one thread per column.
__global__ void k_stats_total(int nb, int ncol, const double* __restrict__ part, double* __restrict__ total) {
  const int k = threadIdx.x;
  if (k >= ncol) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += part[(size_t)ncol * b + k];
  total[k] = s;
}

// Device address of g_stats_scratch on each device.  In host code the name
// g_stats_scratch is only a stand-in for the symbol, not a device address;
// the address is looked up with cudaGetSymbolAddress, once per device, with
// that device current, on the first call made for it.
constexpr int STATS_MAX_DEVICES = 64;
static std::mutex g_stats_mu;
static double* g_stats_ptr[STATS_MAX_DEVICES] = {};

static int stats_scratch(dem_handle* h, double** out) {
  if (h->dev < 0 || h->dev >= STATS_MAX_DEVICES) return set_err(h, DEM_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_stats_mu);
  if (!g_stats_ptr[h->dev]) {
    void* p = nullptr;
    if (int rc = check_cuda(h, cudaGetSymbolAddress(&p, g_stats_scratch), "cudaGetSymbolAddress(stats scratch)")) return rc;
    g_stats_ptr[h->dev] = static_cast<double*>(p);
  }
  *out = g_stats_ptr[h->dev];
  return 0;
}

// Device arrays of a handle for h->n particles, nc DES cells and nfc search
// cells, its error word, stream and an initial pair capacity.
int demb::alloc_handle(dem_handle* h, int nc, int nfc, long long pairs) {
  const size_t n = (size_t)h->n;
  const int cmax = h->dp.cmax;
  bool ok = true;
  auto A = [&](void** p, size_t bytes) {
    if (!ok) return;
    if (cudaMalloc(p, bytes > 0 ? bytes : 8) != cudaSuccess) ok = false;
    else cudaMemset(*p, 0, bytes > 0 ? bytes : 8);
    h->arr_bytes += (long long)(bytes > 0 ? bytes : 8);
  };
  handle_arrays(h, n, (size_t)nc, (size_t)nfc, A);
  if (!ok) return DEM_ERR_CUDA;
  cudaMemset(h->wall_fid, 0xff, sizeof(int) * cmax * n);  // -1 = free slot
  if (cudaMallocHost((void**)&h->herr, sizeof(DevErr)) != cudaSuccess) return DEM_ERR_CUDA;
  memset(h->herr, 0, sizeof(DevErr));
  h->herr->first_rogue = h->n;
  cudaMemcpy(h->derr, h->herr, sizeof(DevErr), cudaMemcpyHostToDevice);
  cudaDeviceGetAttribute(&h->n_sm, cudaDevAttrMultiProcessorCount, h->dev);
  // a stream of its own, so that whole rebuild periods can be captured as
  // CUDA graphs (the legacy default stream cannot be captured)
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) return DEM_ERR_CUDA;
  h->stream = h->own_stream;
  if (cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return DEM_ERR_CUDA;
  if (ensure_pair_capacity(h, pairs)) return DEM_ERR_CUDA;
  if (cudaDeviceSynchronize() != cudaSuccess) return DEM_ERR_CUDA;
  return 0;
}

#define API_GUARD(h) do { if (!(h)) return DEM_ERR_ARG; cudaSetDevice((h)->dev); } while (0)
// entry points of a single-system handle (a batch handle has dem_sys_* calls)
#define SINGLE_GUARD(h)                                                                       \
  do {                                                                                        \
    API_GUARD(h);                                                                             \
    if ((h)->batch()) return set_err((h), DEM_ERR_ARG, "batch handle: use the dem_sys_ calls"); \
  } while (0)

extern "C" {

int dem_abi_version(void) { return DEM_ABI_VERSION; }

int dem_memory_info(dem_handle* h, dem_memory* out) {
  API_GUARD(h);
  if (!out) return DEM_ERR_ARG;
  memset(out, 0, sizeof *out);
  out->array_bytes = h->arr_bytes;
  out->pair_capacity = h->pair_cap;
  out->pair_bytes = pair_array_bytes(h->pair_cap) + (long long)sizeof(int) * h->cand_cap;
  out->scratch_bytes = (int64_t)(h->scan_tmp_elems * sizeof(int) + h->stage_bytes);
  out->pairs = host_pairs(h);
  return fetch_errors(h);
}

const char* dem_last_error(const dem_handle* h) { return h ? h->err.c_str() : "null handle"; }

int dem_create(const dem_params* q, int32_t max_pip, dem_handle** out) {
  if (!q || !out || max_pip <= 0 || max_pip > MAX_PARTICLES) return DEM_ERR_ARG;
  if (q->n_phases < 1 || q->n_phases > DEM_MAX_PHASES) return DEM_ERR_ARG;
  if (!des_grid_ok(*q)) return DEM_ERR_ARG;
  if (q->neighbor_search_n < 1 || !(q->dtsolid > 0.0)) return DEM_ERR_ARG;
  for (int a = 0; a < 3; ++a) {
    int cells = a == 0 ? q->dg_imax : (a == 1 ? q->dg_jmax : q->dg_kmax);
    if (q->periodic[a] && !(a == 2 && q->no_k) && cells < 3) return DEM_ERR_ARG;
  }
  dem_handle* h = new dem_handle();
  h->prm = *q;
  h->n = max_pip;
  cudaGetDevice(&h->dev);
  fill_devparams(h->prm, h->n, h->dp);
  if (int rc = alloc_handle(h, h->dp.ncell2, h->dp.nfcell, 16 * (long long)max_pip + 1024)) {
    dem_destroy(h);
    return rc;
  }
  *out = h;
  return 0;
}

int dem_destroy(dem_handle* h) {
  if (!h) return 0;
  cudaSetDevice(h->dev);
  cudaStreamSynchronize(h->stream);
  free_gas(h);
  invalidate_graphs(h);
  void* ptrs[] = {h->pos4[0], h->pos4[1], h->vel4[0], h->vel4[1], h->omg4[0],
                  h->state, h->phase, h->fc, h->tow, h->acc_old, h->rot_acc_old, h->dg_pijk,
                  h->cell_cnt, h->cell_start, h->cell_fill, h->cell_list, h->row_cnt,
                  h->row_end[0], h->row_end[1], h->nbrs[0], h->nbrs[1], h->pft[0], h->pft[1],
                  h->in_cnt, h->in_start, h->in_fill, h->in_pair, h->pair_owner, h->vertex,
                  h->norm_face, h->ignore_edge, h->fbin_start, h->fbin, h->wall_fid, h->wall_pft,
                  h->scan_tmp, h->derr, h->red, h->stage, h->wall_live, h->wf, h->pflagb[0], h->pflagb[1], h->in_pos, h->in_flag, h->prec, h->touched, h->wall_hit, h->wall_cand, h->wall_list, h->d_nwall, h->wgap, h->d_obc, h->d_ibc, h->pic_fresh, h->d_seed, h->skin, h->vslot, h->pgap,
                  h->fcell_key, h->fcell_cnt, h->fcell_start, h->fcell_list, h->spos, h->sposf, h->sinfo, h->nslot, h->long_rows, h->cand_end, h->cand_cnt, h->cand_start, h->cand_fill, h->qof, h->cand_nb, h->cand, h->slipfix, h->d_np,
                  h->d_sys, h->sys_of, h->d_due, h->d_first_rogue};
  for (void* p : ptrs) if (p) cudaFree(p);
  for (auto& e : h->prof_pending) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
  for (auto e : h->ev_pool) cudaEventDestroy(e);
  if (h->herr) cudaFreeHost(h->herr);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  if (h->side_stream) cudaStreamDestroy(h->side_stream);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  delete h;
  return 0;
}

int dem_set_stream(dem_handle* h, void* stream) {
  API_GUARD(h);
  cudaStreamSynchronize(h->stream);
  invalidate_graphs(h);
  h->stream = (cudaStream_t)stream;
  return 0;
}

int dem_launch_count(const dem_handle* h, int64_t* count) {
  if (!h || !count) return DEM_ERR_ARG;
  *count = h->launches;
  return 0;
}

int dem_set_dtsolid(dem_handle* h, double dtsolid) {
  SINGLE_GUARD(h);
  if (!(dtsolid > 0.0) || !std::isfinite(dtsolid)) return set_err(h, DEM_ERR_ARG, "DTSOLID must be positive");
  if (h->prm.dtsolid != dtsolid) {
    h->prm.dtsolid = dtsolid;
    h->dp.dt = dtsolid;
    invalidate_graphs(h);  // captured steps hold the old DTSOLID
  }
  return 0;
}

int dem_set_walls(dem_handle* h, const double* vertex, const double* norm_face, int32_t nf) {
  SINGLE_GUARD(h);
  if (nf < 0 || (nf > 0 && (!vertex || !norm_face))) return set_err(h, DEM_ERR_ARG, "bad facet arrays");
  return run_bin_facets(h, vertex, norm_face, nf);
}

// Upload goes through a device staging buffer so that the layout change is a
// kernel, not a host loop.
int dem_upload_state(dem_handle* h, const double* pos, const double* vel, const double* omega,
                     const double* radius, const double* pmass, const double* omoi,
                     const int8_t* state, const int32_t* phase, int32_t max_pip) {
  SINGLE_GUARD(h);
  if (max_pip != h->n) return set_err(h, DEM_ERR_ARG, "max_pip does not match dem_create");
  if ((!radius || !pmass || !omoi || !state || !phase) && !h->have_state)
    return set_err(h, DEM_ERR_ARG, "the first upload needs every array");
  // A motion-only upload (radius, mass, inertia, state and phase kept) adds
  // the largest move to the displacement bound; any other upload leaves no
  // pair known apart until the next build.
  const bool motion = h->have_state && !radius && !pmass && !omoi && !state && !phase;
  if (int rc = upload_range(h, 0, h->n, h->dp.nph, pos, vel, omega, radius, pmass, omoi, state, phase, motion))
    return rc;
  if (motion) launch_skin(h);
  else skin_unknown(h);
  h->have_state = true;
  return 0;
}

int dem_download_state(dem_handle* h, double* pos, double* vel, double* omega, int8_t* state, int32_t max_pip) {
  SINGLE_GUARD(h);
  if (max_pip != h->n) return set_err(h, DEM_ERR_ARG, "max_pip mismatch");
  return download_range(h, 0, h->n, pos, vel, omega, state);
}

int dem_download_forces(dem_handle* h, double* fc, double* tow, int32_t max_pip) {
  API_GUARD(h);
  if (max_pip != h->n) return set_err(h, DEM_ERR_ARG, "max_pip mismatch");
  const size_t n = h->n;
  if (fc) cudaMemcpyAsync(fc, h->fc, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream);
  if (tow) cudaMemcpyAsync(tow, h->tow, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "download forces");
}

int dem_set_ab2_history(dem_handle* h, const double* acc_old, const double* rot_acc_old,
                        int32_t first_pass, int32_t max_pip) {
  SINGLE_GUARD(h);
  if (max_pip != h->n) return set_err(h, DEM_ERR_ARG, "max_pip mismatch");
  const size_t n = h->n;
  if (acc_old) cudaMemcpyAsync(h->acc_old, acc_old, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream);
  if (rot_acc_old) cudaMemcpyAsync(h->rot_acc_old, rot_acc_old, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream);
  h->first_pass = first_pass != 0;
  return check_cuda(h, cudaStreamSynchronize(h->stream), "ab2 history");
}

int dem_get_ab2_history(dem_handle* h, double* acc_old, double* rot_acc_old, int32_t max_pip) {
  API_GUARD(h);
  if (max_pip != h->n) return set_err(h, DEM_ERR_ARG, "max_pip mismatch");
  const size_t n = h->n;
  if (acc_old) cudaMemcpyAsync(acc_old, h->acc_old, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream);
  if (rot_acc_old) cudaMemcpyAsync(rot_acc_old, h->rot_acc_old, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "ab2 history");
}

int dem_pair_count(dem_handle* h, int64_t* np) {
  API_GUARD(h);
  if (!np) return DEM_ERR_ARG;
  *np = host_pairs(h);
  return 0;
}

int dem_download_pairs(dem_handle* h, int32_t* ni, int32_t* nb, double* pf, int64_t cap, int32_t max_pip) {
  SINGLE_GUARD(h);
  if (max_pip != h->n) return set_err(h, DEM_ERR_ARG, "max_pip mismatch");
  const long long P = host_pairs(h);
  if ((nb || pf) && cap < P) return set_err(h, DEM_ERR_CAPACITY, "pair capacity too small");
  if (ni) cudaMemcpyAsync(ni, h->row_end[h->rb], sizeof(int) * h->n, cudaMemcpyDeviceToHost, h->stream);
  if (nb && P) cudaMemcpyAsync(nb, h->nbrs[h->rb], sizeof(int) * P, cudaMemcpyDeviceToHost, h->stream);
  if (pf && P) cudaMemcpyAsync(pf, h->pft[h->pcur], sizeof(double) * 3 * P, cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "download pairs")) return rc;
  if (ni) for (int i = 0; i < h->n; ++i) ni[i] += 1;
  if (nb) for (long long c = 0; c < P; ++c) nb[c] += 1;
  return 0;
}

__global__ void k_owner_from_rows(int n, const int* __restrict__ row_end, int* __restrict__ owner) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int s = i ? row_end[i - 1] : 0, e = row_end[i];
  for (int c = s; c < e; ++c) owner[c] = i;
}
int dem_upload_pairs(dem_handle* h, const int32_t* ni, const int32_t* nb, const double* pf, int64_t np, int32_t max_pip) {
  SINGLE_GUARD(h);
  if (max_pip != h->n || np < 0 || !ni || (np > 0 && (!nb || !pf))) return set_err(h, DEM_ERR_ARG, "bad pair arrays");
  // validate the CSR on the host: monotone end pointers, indices in range
  long long prev = 0;
  std::vector<int> re(h->n), nbr((size_t)np);
  for (int i = 0; i < h->n; ++i) {
    long long e = (long long)ni[i] - 1;
    if (e < prev || e > np) return set_err(h, DEM_ERR_ARG, "NEIGHBOR_INDEX is not a valid CSR");
    re[i] = (int)e;
    prev = e;
  }
  if (prev != np) return set_err(h, DEM_ERR_ARG, "NEIGHBOR_INDEX(MAX_PIP) does not match the pair count");
  for (long long c = 0; c < np; ++c) {
    if (nb[c] < 1 || nb[c] > h->n) return set_err(h, DEM_ERR_ARG, "NEIGHBORS index out of range");
    nbr[c] = nb[c] - 1;
  }
  if (int rc = ensure_pair_capacity(h, np + 1)) return rc;
  cudaMemcpyAsync(h->row_end[h->rb], re.data(), sizeof(int) * h->n, cudaMemcpyHostToDevice, h->stream);
  if (np) {
    cudaMemcpyAsync(h->nbrs[h->rb], nbr.data(), sizeof(int) * np, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->pft[h->pcur], pf, sizeof(double) * 3 * np, cudaMemcpyHostToDevice, h->stream);
  }
  h->n_pairs = np;
  h->np_stale = false;
  {
    int v = (int)np;
    cudaMemcpyAsync(h->d_np, &v, sizeof(int), cudaMemcpyHostToDevice, h->stream);
    cudaStreamSynchronize(h->stream);
  }
  const int T = 256, B = (h->n + T - 1) / T;
  k_owner_from_rows<<<B, T, 0, h->stream>>>(h->n, h->row_end[h->rb], h->pair_owner);
  h->launches++;
  set_hist_flags(h);
  skin_unknown(h);  // no gaps for an uploaded list: no pair is skipped until the next build
  if (int rc = build_transpose(h, h->rb)) return rc;
  h->have_pairs = true;
  return check_cuda(h, cudaStreamSynchronize(h->stream), "upload pairs");
}

int dem_download_wall_history(dem_handle* h, int32_t* fid, double* pf, int32_t max_pip) {
  SINGLE_GUARD(h);
  if (max_pip != h->n) return set_err(h, DEM_ERR_ARG, "max_pip mismatch");
  const size_t cnt = (size_t)h->n * h->dp.cmax;
  if (fid) cudaMemcpyAsync(fid, h->wall_fid, sizeof(int) * cnt, cudaMemcpyDeviceToHost, h->stream);
  if (pf) cudaMemcpyAsync(pf, h->wall_pft, sizeof(double) * 3 * cnt, cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "download wall history")) return rc;
  if (fid) for (size_t s = 0; s < cnt; ++s) fid[s] = fid[s] < 0 ? -1 : fid[s] + 1;
  return 0;
}

int dem_upload_wall_history(dem_handle* h, const int32_t* fid, const double* pf, int32_t max_pip) {
  SINGLE_GUARD(h);
  if (max_pip != h->n || !fid || !pf) return set_err(h, DEM_ERR_ARG, "bad wall history arrays");
  const size_t cnt = (size_t)h->n * h->dp.cmax;
  std::vector<int> ids(cnt);
  for (size_t s = 0; s < cnt; ++s) {
    if (fid[s] != -1 && (fid[s] < 1 || fid[s] > h->nf)) return set_err(h, DEM_ERR_ARG, "facet id out of range");
    ids[s] = fid[s] < 0 ? -1 : fid[s] - 1;
  }
  cudaMemcpyAsync(h->wall_fid, ids.data(), sizeof(int) * cnt, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(h->wall_pft, pf, sizeof(double) * 3 * cnt, cudaMemcpyHostToDevice, h->stream);
  // every particle may hold history now; the wall kernel clears the mark
  // where no slot is in use
  cudaMemsetAsync(h->wall_live, 1, h->n, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "upload wall history");
}

int dem_download_cells(dem_handle* h, int32_t* cells, int32_t max_pip) {
  SINGLE_GUARD(h);
  if (max_pip != h->n || !cells) return set_err(h, DEM_ERR_ARG, "bad arguments");
  cudaMemcpyAsync(cells, h->dg_pijk, sizeof(int) * h->n, cudaMemcpyDeviceToHost, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "download cells");
}

int dem_desgrid_pic(dem_handle* h) {
  SINGLE_GUARD(h);
  if (!h->have_state) return set_err(h, DEM_ERR_STATE, "no particle state uploaded");
  if (int rc = run_desgrid_pic(h, true)) return rc;
  return fetch_errors(h);
}

int dem_neighbour(dem_handle* h) {
  SINGLE_GUARD(h);
  if (!h->have_state) return set_err(h, DEM_ERR_STATE, "no particle state uploaded");
  if (int rc = run_neighbour(h, true)) return rc;
  return fetch_errors(h);
}

int dem_init_neighbors(dem_handle* h) {
  SINGLE_GUARD(h);
  if (!h->have_state) return set_err(h, DEM_ERR_STATE, "no particle state uploaded");
  h->have_pairs = false;
  if (int rc = run_desgrid_pic(h, true)) return rc;
  if (int rc = run_neighbour(h, false)) return rc;
  return fetch_errors(h);
}

int dem_calc_force(dem_handle* h) {
  SINGLE_GUARD(h);
  if (!h->have_state || !h->have_pairs) return set_err(h, DEM_ERR_STATE, "state or pair list missing");
  cudaMemsetAsync(&h->derr->n_contacts, 0, 2 * sizeof(unsigned long long), h->stream);
  if (int rc = run_force(h, false)) return rc;
  return fetch_errors(h);
}

int dem_cfnewvalues(dem_handle* h) {
  SINGLE_GUARD(h);
  if (!h->have_state) return set_err(h, DEM_ERR_STATE, "no particle state uploaded");
  if (int rc = run_cfnewvalues(h)) return rc;
  return check_cuda(h, cudaStreamSynchronize(h->stream), "cfnewvalues");
}

// One DES_TIME_STEP(NN) of a pure DEM run: force + integration, then the
// cell binning (every step with periodic axes) and the neighbour rebuild
// when NN == 1 or mod(NN, NEIGHBOR_SEARCH_N) == 0 (des_time_march.f:398-414).
static int step_once(dem_handle* h, int nn) {
  const DevParams& p = h->dp;
  const bool anyper = p.per[0] || p.per[1] || (p.per[2] && !p.no_k);
  cudaMemsetAsync(&h->derr->n_contacts, 0, 2 * sizeof(unsigned long long), h->stream);
  bool force = false;
  if (h->obc.empty()) {
    if (int rc = run_force(h, true)) return rc;
    if (int rc = run_mass_inflow(h)) return rc;  // MASS_INFLOW_DEM
  } else {
    // outflow boundaries: forces, then exit velocities + CFNEWVALUES +
    // MASS_OUTFLOW_DEM, whose deletions force the neighbour search
    if (int rc = run_force(h, false)) return rc;
    if (int rc = run_cfnewvalues_outflow(h, &force)) return rc;
  }
  const bool do_nsearch = (nn == 1) || (nn % h->prm.neighbor_search_n == 0) || force;
  // the integrating gather of a periodic system already placed the particles
  const bool placed = cells_in_gather(h);
  if (do_nsearch || (anyper && !placed)) {
    if (int rc = run_desgrid_pic(h, do_nsearch)) return rc;
  }
  if (do_nsearch) {
    if (int rc = run_neighbour(h, true)) return rc;
  }
  h->s_time = h->s_time + h->prm.dtsolid;
  h->steps_done++;
  return 0;
}

// The NEIGHBOR_SEARCH_N steps NN = m*N+1 .. (m+1)*N (m >= 1) end with the one
// rebuild of the period and are otherwise identical, so they are captured
// once as a CUDA graph per combination of buffer parities and replayed.  A
// replay cannot grow the pair arrays: the capacity is kept at twice the
// last known pair count before every replay, and a build that still
// overflows is reported as DEM_ERR_PAIR_OVERFLOW.
static int replay_period(dem_handle* h, int nn0) {
  const int nsn = h->prm.neighbor_search_n;
  const long long P = host_pairs(h);
  if (2 * P + 1024 > h->pair_cap) {
    if (int rc = ensure_pair_capacity(h, 2 * P + 1024)) return rc;
    invalidate_graphs(h);
  }
  const int key = (h->cur << 2) | (h->pcur << 1) | h->rb;
  if (!h->graphs[key]) {
    cudaGraph_t graph;
    h->capturing = true;
    if (int rc = check_cuda(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "begin capture")) {
      h->capturing = false;
      return rc;
    }
    int rc = 0;
    const int cur0 = h->cur, pcur0 = h->pcur, rb0 = h->rb;
    const long long sd0 = h->steps_done;
    const double st0 = h->s_time;
    const long long l0 = h->launches;
    for (int j = 0; j < nsn && !rc; ++j) rc = step_once(h, nn0 + j);
    cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
    h->capturing = false;
    // capture only recorded the work: restore the bookkeeping, then launch
    h->cur = cur0; h->pcur = pcur0; h->rb = rb0; h->steps_done = sd0; h->s_time = st0;
    h->graph_launches += h->launches - l0;
    h->launches = l0;
    if (rc) return rc;
    if (int r2 = check_cuda(h, ce, "end capture")) return r2;
    cudaGraphExec_t exec;
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (int r2 = check_cuda(h, ce, "graph instantiate")) return r2;
    h->graphs[key] = exec;
    h->graph_kernels[key] = h->graph_launches;
    h->graph_launches = 0;
  }
  if (int rc = check_cuda(h, cudaGraphLaunch(h->graphs[key], h->stream), "graph launch")) return rc;
  h->launches += h->graph_kernels[key];
  // buffer parities and bookkeeping after the period: N force passes flip
  // the state buffers, the rebuild flips the list and history buffers
  for (int j = 0; j < nsn; ++j) {
    h->cur = 1 - h->cur;
    h->s_time = h->s_time + h->prm.dtsolid;
    h->steps_done++;
  }
  h->pcur = 1 - h->pcur;
  h->rb = 1 - h->rb;
  h->first_pass = false;
  h->np_stale = true;
  return 0;
}

int dem_step(dem_handle* h, int32_t nn_first, int32_t nsteps) {
  SINGLE_GUARD(h);
  if (!h->have_state || !h->have_pairs) return set_err(h, DEM_ERR_STATE, "state or pair list missing");
  if (nsteps < 0 || nn_first < 1) return set_err(h, DEM_ERR_ARG, "bad step range");
  const int nsn = h->prm.neighbor_search_n;
  const bool graphs_ok = h->stream != nullptr && !h->prof && !h->no_graphs && h->obc.empty() && h->ibc.empty();
  int k = 0;
  while (k < nsteps) {
    const int nn = nn_first + k;
    if (graphs_ok && !h->first_pass && nn > 1 && (nn - 1) % nsn == 0 && nsteps - k >= nsn) {
      if (int rc = replay_period(h, nn)) return rc;
      k += nsn;
    } else {
      if (int rc = step_once(h, nn)) return rc;
      ++k;
    }
  }
  return fetch_errors(h);
}

int dem_set_graphs(dem_handle* h, int32_t on) {
  API_GUARD(h);
  h->no_graphs = on == 0;
  if (h->no_graphs) invalidate_graphs(h);
  return 0;
}

int dem_get_stats(dem_handle* h, dem_stats* s) {
  API_GUARD(h);
  if (!s) return DEM_ERR_ARG;
  memset(s, 0, sizeof *s);
  if (int rc = stats_range(h, 0, h->n, s)) return rc;
  cudaMemcpyAsync(h->herr, h->derr, sizeof(DevErr), cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "stats")) return rc;
  s->n_pairs = host_pairs(h);
  s->n_contacts = (int64_t)h->herr->n_contacts;
  s->n_wall_contacts = (int64_t)h->herr->n_wall_contacts;
  s->n_rogue_removed = (int64_t)h->herr->rogue_removed;
  s->n_outflow_removed = (int64_t)h->herr->outflow_removed;
  s->n_inflow_added = (int64_t)h->inflow_added;
  s->n_candidate_lists = (int64_t)h->herr->cand_lists;
  s->n_builds_filtered = (int64_t)h->herr->cand_filtered;
  s->steps_done = h->steps_done;
  s->s_time = h->s_time;
  return 0;
}

// The same statistics as dem_get_stats from the same two kernels and the
// same block-ordered sums, with every intermediate kept in g_stats_scratch:
// no device or host allocation on any call.
int dem_get_stats_noalloc(dem_handle* h, dem_stats* s) {
  API_GUARD(h);
  if (!s) return DEM_ERR_ARG;
  if (h->n > DEM_STATS_NOALLOC_MAX_PARTICLES) {
    char b[200];
    snprintf(b, sizeof b, "dem_get_stats_noalloc: %d particles exceed its limit of %d (DEM_STATS_NOALLOC_MAX_PARTICLES)",
             h->n, (int)DEM_STATS_NOALLOC_MAX_PARTICLES);
    return set_err(h, DEM_ERR_CAPACITY, b);
  }
  double* scr = nullptr;
  if (int rc = stats_scratch(h, &scr)) return rc;
  memset(s, 0, sizeof *s);
  const int T = STAT_T, B = (h->n + T - 1) / T;
  double* tot = scr + STATS_TOTAL_OFF;
  double sum[8];
  if (B > 0) {
    k_stats1<<<B, T, 0, h->stream>>>(h->n, h->pos4[h->cur], h->vel4[h->cur], h->state, scr);
    h->launches++;
  }
  k_stats_total<<<1, 32, 0, h->stream>>>(B, 8, scr, tot);
  h->launches++;
  if (int rc = check_cuda(h, cudaGetLastError(), "stats launch")) return rc;
  cudaMemcpyAsync(sum, tot, sizeof sum, cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "stats")) return rc;
  const double nn = sum[0];
  double mv[3] = {0, 0, 0};
  if (nn > 0) for (int c = 0; c < 3; ++c) mv[c] = sum[1 + c] / nn;
  if (B > 0) {
    k_stats2<<<B, T, 0, h->stream>>>(h->n, h->vel4[h->cur], h->state, mv[0], mv[1], mv[2], scr);
    h->launches++;
  }
  k_stats_total<<<1, 32, 0, h->stream>>>(B, 3, scr, tot);
  h->launches++;
  if (int rc = check_cuda(h, cudaGetLastError(), "stats launch")) return rc;
  double gt[3];
  cudaMemcpyAsync(gt, tot, sizeof gt, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(h->herr, h->derr, sizeof(DevErr), cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "stats")) return rc;
  s->n_normal = (int64_t)nn;
  for (int c = 0; c < 3; ++c) { s->mean_vel[c] = mv[c]; s->gran_temp[c] = nn > 0 ? gt[c] / nn : 0.0; }
  s->n_pairs = host_pairs(h);
  s->n_contacts = (int64_t)h->herr->n_contacts;
  s->n_wall_contacts = (int64_t)h->herr->n_wall_contacts;
  s->n_rogue_removed = (int64_t)h->herr->rogue_removed;
  s->n_outflow_removed = (int64_t)h->herr->outflow_removed;
  s->n_inflow_added = (int64_t)h->inflow_added;
  s->n_candidate_lists = (int64_t)h->herr->cand_lists;
  s->n_builds_filtered = (int64_t)h->herr->cand_filtered;
  s->steps_done = h->steps_done;
  s->kinetic_energy = sum[6];
  s->bed_height = sum[4] > 0 ? sum[5] / sum[4] : 0.0;
  s->s_time = h->s_time;
  return 0;
}

int dem_set_profiling(dem_handle* h, int32_t on) {
  API_GUARD(h);
  prof_collect(h);
  h->prof = on < 0 ? 0 : (on > 2 ? 2 : on);
  for (int k = 0; k < DEM_PROF_N; ++k) { h->prof_ms[k] = 0.0; h->prof_n[k] = 0; }
  return 0;
}

int dem_get_profile(dem_handle* h, double* ms, int64_t* launches) {
  API_GUARD(h);
  prof_collect(h);
  for (int k = 0; k < DEM_PROF_N; ++k) {
    if (ms) ms[k] = h->prof_ms[k];
    if (launches) launches[k] = h->prof_n[k];
  }
  return 0;
}

int dem_force_error(dem_handle* h, double* rel_err) {
  SINGLE_GUARD(h);
  if (!rel_err) return DEM_ERR_ARG;
  return run_split_force_error(h, rel_err);
}

}  // extern "C"
