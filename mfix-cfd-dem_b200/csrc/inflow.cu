// inflow.cu -- DEM mass-inflow boundaries: MASS_INFLOW_DEM
// (model/des/mass_inflow_dem.f:44-293) with SEED_NEW_PARTICLE (306-408) and
// SET_NEW_PARTICLE_PROPS (419-642, plain spheres).
//
// The entering test is per particle: an ENTERING particle whose DES cell of
// the last DESGRID_PIC lies in a boundary's box (the DG_PIC lists of
// DEM_BCMI_IJK) and that is clear of the boundary's plane by more than its
// radius becomes NORMAL.  A particle seeded since the last DESGRID_PIC is
// in no DG_PIC list yet, so it is not tested (pic_fresh).
//
// Seeding is sequential bookkeeping on a handful of particles: the host
// walks the boundaries in order, draws RAND(3), checks the injection time,
// cycles the layout's windows and builds the new particles' records; one
// block then puts the records into the first NONEXISTENT slots in index
// order, the slots the reference's search from LS = 1 finds.
#include "dem_internal.cuh"

#include <cmath>

using namespace demb;

namespace {

// A new particle as SET_NEW_PARTICLE_PROPS leaves it.
struct SeedRec {
  double x[3], r;
  double v[3], m;
  double omoi;
  int32_t phase0;  // 0-based solids phase
  int32_t cell;    // DG_PIJK
};

__device__ __forceinline__ bool in_box(const DevParams& p, const dem_inflow_bc& b, int c) {
  if (c < 1) return false;
  const int ijk[3] = {dg_iof(p, c), dg_jof(p, c), dg_kof(p, c)};
  for (int a = 0; a < 3; ++a)
    if (ijk[a] < b.dg_lo[a] || ijk[a] > b.dg_hi[a]) return false;
  return true;
}

__host__ __device__ __forceinline__ int normal_axis(int plane) {
  return (plane == 'N' || plane == 'S') ? 1 : ((plane == 'E' || plane == 'W') ? 0 : 2);
}

// The entering test of MASS_INFLOW_DEM (mass_inflow_dem.f:82-140): DIST is
// the distance into the domain from the boundary's plane.
__global__ void k_entering(DevParams p, const dem_inflow_bc* __restrict__ bcs, int nbc,
                           const int* __restrict__ dg_pijk, const double4* __restrict__ pos4,
                           int8_t* __restrict__ state, const uint8_t* __restrict__ fresh) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= p.n) return;
  if (state[me] != DEM_STATE_ENTERING || fresh[me]) return;
  const int cell = dg_pijk[me];
  const double4 X = pos4[me];
  for (int b = 0; b < nbc; ++b) {
    const dem_inflow_bc& B = bcs[b];
    if (!in_box(p, B, cell)) continue;
    const int idx = normal_axis(B.plane);
    const double xi = idx == 0 ? X.x : (idx == 1 ? X.y : X.z);
    const double dist = (B.plane == 'N' || B.plane == 'E' || B.plane == 'T') ? xi - B.face : B.face - xi;
    if (dist > X.w) {
      state[me] = DEM_STATE_NORMAL;
      return;
    }
  }
}

// The new particles into the first k NONEXISTENT slots, in index order: one
// block walks the state array a tile of SEED_T slots at a time (bounded by
// n), ranking the free slots of each tile with a block-wide scan.
constexpr int SEED_T = 1024;
static_assert(SEED_T == 32 * 32, "one warp scans the warp counts");
__global__ void __launch_bounds__(SEED_T)
k_seed(int n, int k, const SeedRec* __restrict__ rec, int8_t* __restrict__ state, double4* __restrict__ pos4,
       double4* __restrict__ vel4, double4* __restrict__ omg4, uint8_t* __restrict__ phase,
       int* __restrict__ dg_pijk, uint8_t* __restrict__ wall_cand, const int* __restrict__ fbin_start,
       int cell_off, uint8_t* __restrict__ wall_live, float* __restrict__ wgap, uint8_t* __restrict__ touched,
       uint8_t* __restrict__ wall_hit, uint8_t* __restrict__ fresh, DevErr* __restrict__ err) {
  __shared__ int warp_n[SEED_T / 32];
  __shared__ int tile_total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int found = 0;
  for (int base = 0; base < n && found < k; base += SEED_T) {
    const int j = base + threadIdx.x;
    const bool freeslot = j < n && state[j] == DEM_STATE_NONEXISTENT;
    const unsigned m = __ballot_sync(0xffffffffu, freeslot);
    if (lane == 0) warp_n[warp] = __popc(m);
    __syncthreads();
    if (warp == 0) {
      const int c = warp_n[lane];
      int incl = c;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      warp_n[lane] = incl - c;
      if (lane == 31) tile_total = incl;
    }
    __syncthreads();
    const int rank = found + warp_n[warp] + __popc(m & ((1u << lane) - 1u));
    if (freeslot && rank < k) {
      const SeedRec& r = rec[rank];
      pos4[j] = make_double4(r.x[0], r.x[1], r.x[2], r.r);
      vel4[j] = make_double4(r.v[0], r.v[1], r.v[2], r.m);
      omg4[j] = make_double4(0.0, 0.0, 0.0, r.omoi);
      phase[j] = (uint8_t)r.phase0;
      dg_pijk[j] = r.cell;
      const int fc = cell_off + r.cell - 1;
      wall_cand[j] = fbin_start[fc + 1] > fbin_start[fc] ? 1 : 0;
      wall_live[j] = 0;
      wgap[j] = -1.0f;  // clearance unknown until the next build: walls are checked
      touched[j] = 0;
      wall_hit[j] = 0;
      fresh[j] = 1;
      state[j] = DEM_STATE_ENTERING;
    }
    found += tile_total;
    __syncthreads();  // warp_n and tile_total are rewritten by the next tile
  }
  if (threadIdx.x == 0 && found < k) atomicOr(&err->flags, EF_INFLOW_CAP);
}

// splitmix64, mapped to [0,1) with 53 bits
double next_uniform(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * 0x1.0p-53;
}

// IofPOS/JofPOS/KofPOS (desgrid_mod.f:391-419)
int host_ofpos(const DevParams& p, int ax, double x, int start1) {
  return (int)std::floor((x - p.dg_start[ax]) * p.dg_inv[ax]) + start1;
}

}  // namespace

namespace demb {

int run_mass_inflow(dem_handle* h) {
  if (h->ibc.empty()) return 0;
  const DevParams& p = h->dp;
  const int nbc = (int)h->ibc.size();
  const int T = 256, G = (h->n + T - 1) / T, c = h->cur;
  k_entering<<<G, T, 0, h->stream>>>(p, h->d_ibc, nbc, h->dg_pijk, h->pos4[c], h->state, h->pic_fresh);
  DEM_LAUNCH(h);
  std::vector<SeedRec> add;
  const double s_time = h->s_time, dt = h->prm.dtsolid;
  for (dem_handle::Inflow& I : h->ibc) {
    dem_inflow_bc& b = I.bc;
    double rnd[3];
    for (double& r : rnd) {
      if (!h->irand.empty()) { r = h->irand.front(); h->irand.pop_front(); }
      else r = next_uniform(h->irng);
    }
    if (b.mi_time > s_time) continue;
    if (s_time < b.start_time || s_time > b.end_time) continue;
    for (int ip = 0; ip < b.pi_count; ++ip) {
      // SEED_NEW_PARTICLE
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
      double pos[3];
      const double pv = I.p[vac - 1] + rand1, qv = I.q[vac - 1] + rand2;
      switch (b.plane) {
        case 'N': case 'S': pos[0] = pv; pos[2] = qv; pos[1] = b.offset; break;
        case 'E': case 'W': pos[1] = pv; pos[2] = qv; pos[0] = b.offset; break;
        default: pos[0] = pv; pos[1] = qv; pos[2] = b.offset; break;  // 'T', 'B'
      }
      if (p.no_k) pos[2] = 0.0;
      const int li = host_ofpos(p, 0, pos[0], p.istart1), lj = host_ofpos(p, 1, pos[1], p.jstart1),
                lk = host_ofpos(p, 2, pos[2], p.kstart1);
      // one rank owns the whole DES grid, its ghost layers included
      // (DG_ISTART = DG_IMIN2 .. DG_IEND = DG_IMAX2, desgrid_mod.f:756-761)
      bool owns = p.istart2 <= li && li <= p.iend2 && p.jstart2 <= lj && lj <= p.jend2;
      if (!p.no_k) owns = owns && p.kstart2 <= lk && lk <= p.kend2;
      if (!owns) continue;
      // SET_NEW_PARTICLE_PROPS for a plain sphere
      SeedRec r;
      for (int a = 0; a < 3; ++a) { r.x[a] = pos[a]; r.v[a] = b.vel[m][a]; }
      r.r = d * 0.5;
      const double pvol = (4.0 / 3.0) * M_PI * (r.r * r.r * r.r);
      r.m = pvol * b.ro_s0[m];
      r.omoi = 2.5 / (r.m * (r.r * r.r));
      r.phase0 = m;
      const int ci = std::min(p.iend2, std::max(p.istart2, li));
      const int cj = std::min(p.jend2, std::max(p.jstart2, lj));
      const int ck = p.no_k ? 1 : std::min(p.kend2, std::max(p.kstart2, lk));
      r.cell = cj + ci * p.c1 + ck * p.c2 + p.c3;
      add.push_back(r);
    }
    b.mi_time = b.mi_time + b.pi_factor * dt;
  }
  if (add.empty()) return check_cuda(h, cudaGetLastError(), "inflow");
  const int k = (int)add.size();
  if (k > h->seed_cap) {
    cudaStreamSynchronize(h->stream);
    if (h->d_seed) cudaFree(h->d_seed);
    h->d_seed = nullptr;
    h->seed_cap = 0;
    if (int rc = check_cuda(h, cudaMalloc(&h->d_seed, sizeof(SeedRec) * (size_t)k), "cudaMalloc seeds")) return rc;
    h->seed_cap = k;
  }
  // pageable source: the copy has read it when the call returns
  cudaMemcpyAsync(h->d_seed, add.data(), sizeof(SeedRec) * (size_t)k, cudaMemcpyHostToDevice, h->stream);
  k_seed<<<1, SEED_T, 0, h->stream>>>(h->n, k, (const SeedRec*)h->d_seed, h->state, h->pos4[c], h->vel4[c],
                                      h->omg4[c], h->phase, h->dg_pijk, h->wall_cand, h->fbin_start, p.cell_off,
                                      h->wall_live, h->wgap, h->touched, h->wall_hit, h->pic_fresh, h->derr);
  DEM_LAUNCH(h);
  h->inflow_added += k;
  return check_cuda(h, cudaGetLastError(), "inflow seeding");
}

}  // namespace demb

extern "C" {

int dem_set_inflow_bcs(dem_handle* h, const dem_inflow_bc* bcs, int32_t n, uint64_t seed) {
  if (!h) return DEM_ERR_ARG;
  cudaSetDevice(h->dev);
  if (h->batch()) return set_err(h, DEM_ERR_ARG, "inflow boundaries are per system; not available on a batch handle");
  if (n < 0 || (n > 0 && !bcs)) return set_err(h, DEM_ERR_ARG, "bad inflow boundaries");
  for (int32_t i = 0; i < n; ++i) {
    const dem_inflow_bc& b = bcs[i];
    const int pl = b.plane;
    if (pl != 'N' && pl != 'S' && pl != 'E' && pl != 'W' && pl != 'T' && pl != 'B')
      return set_err(h, DEM_ERR_ARG, "unknown BC_PLANE");
    if (b.pi_count < 0 || (b.pi_count > 0 && (b.occupants < 1 || !b.p || !b.q)))
      return set_err(h, DEM_ERR_ARG, "inflow layout missing");
    if (b.vacancy < 1 || (b.occupants > 0 && b.vacancy > b.occupants))
      return set_err(h, DEM_ERR_ARG, "inflow vacancy out of range");
    if (b.n_layout < 1 || !b.poly_layout) return set_err(h, DEM_ERR_ARG, "inflow phase layout missing");
    for (int32_t j = 0; j < b.n_layout; ++j)
      if (b.poly_layout[j] < 1 || b.poly_layout[j] > h->dp.nph)
        return set_err(h, DEM_ERR_ARG, "inflow phase out of range");
    for (int a = 0; a < 3; ++a)
      if (b.dg_lo[a] > b.dg_hi[a]) return set_err(h, DEM_ERR_ARG, "empty DES-cell box");
    if (!(b.pi_factor > 0.0) && b.pi_count > 0) return set_err(h, DEM_ERR_ARG, "PI_FACTOR must be positive");
  }
  cudaStreamSynchronize(h->stream);
  if (h->d_ibc) { cudaFree(h->d_ibc); h->d_ibc = nullptr; }
  h->ibc.clear();
  h->irand.clear();
  h->irng = seed;
  invalidate_graphs(h);
  if (n == 0) return 0;
  for (int32_t i = 0; i < n; ++i) {
    dem_handle::Inflow I;
    I.bc = bcs[i];
    const int occ = bcs[i].pi_count > 0 ? bcs[i].occupants : 0;
    I.p.assign(bcs[i].p, bcs[i].p + occ);
    I.q.assign(bcs[i].q, bcs[i].q + occ);
    I.layout.assign(bcs[i].poly_layout, bcs[i].poly_layout + bcs[i].n_layout);
    I.w.assign((size_t)occ, 0);
    I.hh.assign((size_t)occ, 0);
    if (bcs[i].w_cell) I.w.assign(bcs[i].w_cell, bcs[i].w_cell + occ);
    if (bcs[i].h_cell) I.hh.assign(bcs[i].h_cell, bcs[i].h_cell + occ);
    // the device copy holds no host pointers
    I.bc.p = nullptr; I.bc.q = nullptr; I.bc.poly_layout = nullptr; I.bc.w_cell = nullptr; I.bc.h_cell = nullptr;
    h->ibc.push_back(std::move(I));
  }
  if (!h->pic_fresh) {
    if (int rc = check_cuda(h, cudaMalloc(&h->pic_fresh, (size_t)h->n), "cudaMalloc pic_fresh")) return rc;
  }
  cudaMemsetAsync(h->pic_fresh, 0, (size_t)h->n, h->stream);
  if (int rc = check_cuda(h, cudaMalloc(&h->d_ibc, sizeof(dem_inflow_bc) * n), "cudaMalloc inflow")) return rc;
  std::vector<dem_inflow_bc> dev(n);
  for (int32_t i = 0; i < n; ++i) dev[i] = h->ibc[i].bc;
  cudaMemcpyAsync(h->d_ibc, dev.data(), sizeof(dem_inflow_bc) * n, cudaMemcpyHostToDevice, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "inflow boundaries");
}

int dem_push_inflow_random(dem_handle* h, const double* r, int64_t n) {
  if (!h) return DEM_ERR_ARG;
  if (n < 0 || (n > 0 && !r)) return set_err(h, DEM_ERR_ARG, "bad random numbers");
  for (int64_t i = 0; i < n; ++i) {
    if (!(r[i] >= 0.0 && r[i] <= 1.0)) return set_err(h, DEM_ERR_ARG, "random numbers must lie in [0,1]");
  }
  h->irand.insert(h->irand.end(), r, r + n);
  return 0;
}

int dem_get_inflow_state(dem_handle* h, int32_t bc, int32_t* vacancy, double* mi_time) {
  if (!h) return DEM_ERR_ARG;
  if (bc < 0 || bc >= (int32_t)h->ibc.size()) return set_err(h, DEM_ERR_ARG, "no such inflow boundary");
  if (vacancy) *vacancy = h->ibc[bc].bc.vacancy;
  if (mi_time) *mi_time = h->ibc[bc].bc.mi_time;
  return 0;
}

}  // extern "C"
