// outflow.cu -- DEM outflow boundaries: UPDATE_EXIT_DES_VEL, CFNEWVALUES and
// MASS_OUTFLOW_DEM (model/des/mass_outflow_dem.f, des_time_march.f:372-405).
//
// A particle belongs to a boundary when its DES cell of the last
// DESGRID_PIC lies in the boundary's box of DES cells (the DG_PIC lists of
// DEM_BCMO_IJK).  Every operation is per particle, so the reference's loop
// over boundaries, cells and particles is a particle-parallel loop over the
// boundaries in their order.  The step with outflow boundaries is taken
// unfused: CALC_FORCE_DEM into FC/TOW, then k_integrate_outflow, then
// k_mass_outflow, whose deletion count decides the neighbour search.
#include "dem_internal.cuh"

using namespace demb;

namespace {

__device__ __forceinline__ bool in_box(const DevParams& p, const dem_outflow_bc& b, int c) {
  if (c < 1) return false;
  const int ijk[3] = {dg_iof(p, c), dg_jof(p, c), dg_kof(p, c)};
  for (int a = 0; a < 3; ++a)
    if (ijk[a] < b.dg_lo[a] || ijk[a] > b.dg_hi[a]) return false;
  return true;
}

// FREEZE, IDX and SGN of a BC_PLANE (mass_outflow_dem.f:44-51)
__device__ __forceinline__ void plane_of(int plane, double fz[3], int& idx, double& sgn) {
  switch (plane) {
    case 'N': idx = 1; sgn = -1.0; break;
    case 'S': idx = 1; sgn = 1.0; break;
    case 'E': idx = 0; sgn = -1.0; break;
    case 'W': idx = 0; sgn = 1.0; break;
    case 'T': idx = 2; sgn = -1.0; break;
    default: idx = 2; sgn = 1.0; break;  // 'B'
  }
  fz[0] = fz[1] = fz[2] = 0.0;
  fz[idx] = 1.0;
}

// CFUPDATEOLD + UPDATE_EXIT_DES_VEL + CFNEWVALUES per particle.  An EXITING
// particle in the cells of a non-MASS_OUTFLOW boundary first integrates its
// force into a velocity frozen to the boundary-normal component
// (mass_outflow_dem.f:444-514, FC converted to an acceleration on the way
// for Adams-Bashforth); CFNEWVALUES then moves it with that velocity, as for
// every other particle it does not accelerate.
template <int MODE>
__global__ void k_integrate_outflow(DevParams p, const dem_outflow_bc* __restrict__ bcs, int nbc, int exit_first,
                                    const int* __restrict__ dg_pijk, double4* __restrict__ pos4,
                                    double4* __restrict__ vel4, double4* __restrict__ omg4,
                                    const int8_t* __restrict__ state, double* __restrict__ fc,
                                    double* __restrict__ tow, double* __restrict__ acc_old,
                                    double* __restrict__ rot_acc_old, unsigned* __restrict__ vslot) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= p.n) return;
  const size_t n = (size_t)p.n;
  const int8_t st = state[me];
  const double4 X = pos4[me], V = vel4[me], W = omg4[me];
  const double x[3] = {X.x, X.y, X.z}, v[3] = {V.x, V.y, V.z}, w[3] = {W.x, W.y, W.z};
  double f[3], t[3];
  for (int c = 0; c < 3; ++c) {
    f[c] = fc[c * n + me]; t[c] = tow[c * n + me];
    fc[c * n + me] = 0.0; tow[c * n + me] = 0.0;
  }
  bool exiting = false;
  double ve[3] = {v[0], v[1], v[2]};
  if (st == DEM_STATE_EXITING) {
    const int cell = dg_pijk[me];
    const double dt = p.dt;
    for (int b = 0; b < nbc; ++b) {
      if (bcs[b].mass_outflow || !in_box(p, bcs[b], cell)) continue;
      double fz[3]; int idx; double sgn;
      plane_of(bcs[b].plane, fz, idx, sgn);
      for (int c = 0; c < 3; ++c) {
        if (MODE == 1) {
          ve[c] = ve[c] + dt * (f[c] / V.w + p.grav[c]);
        } else {
          if (exit_first) acc_old[c * n + me] = f[c] / V.w + p.grav[c];
          f[c] = f[c] / V.w + p.grav[c];
          ve[c] = v[c] + 0.5 * (3.0 * f[c] - acc_old[c * n + me]) * dt;
          acc_old[c * n + me] = f[c];
        }
        ve[c] = ve[c] * fz[c];
      }
      exiting = true;
    }
  }
  if (!exiting) {
    finish_particle<MODE>(p, me, st, x, v, w, X.w, V.w, W.w, f, t, pos4, vel4, omg4, fc, tow, acc_old,
                          rot_acc_old, vslot);
    return;
  }
  // CFNEWVALUES of a particle it does not accelerate (cfnewvalues.f:672-812)
  const double dt = p.dt;
  double xn[3];
  for (int c = 0; c < 3; ++c) {
    if (MODE == 1) {
      xn[c] = x[c] + ve[c] * dt;
    } else {
      // DES_ACC_OLD = FC for every particle; ROT_ACC_OLD = TOW only on the
      // first pass
      acc_old[c * n + me] = f[c];
      if (p.first_pass) rot_acc_old[c * n + me] = t[c];
      xn[c] = x[c] + 0.5 * (v[c] + ve[c]) * dt;
    }
  }
  pos4[me] = make_double4(xn[0], xn[1], xn[2], X.w);
  vel4[me] = make_double4(ve[0], ve[1], ve[2], V.w);
  note_displacement(vslot, fmax(speed(v), speed(ve)) * dt);
}

// MASS_OUTFLOW_DEM (mass_outflow_dem.f:13-188) per particle, the boundaries
// in order; a deletion is DELETE_PARTICLE (mass_outflow_dem.f:201-303).
__global__ void k_mass_outflow(DevParams p, const dem_outflow_bc* __restrict__ bcs, int nbc,
                               const int* __restrict__ dg_pijk, double4* __restrict__ pos4,
                               double4* __restrict__ vel4, double4* __restrict__ omg4,
                               int8_t* __restrict__ state, const uint8_t* __restrict__ phase,
                               double* __restrict__ fc, double* __restrict__ tow, int* __restrict__ wall_fid,
                               DevErr* __restrict__ err) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= p.n) return;
  const int cell = dg_pijk[me];
  for (int b = 0; b < nbc; ++b) {
    const dem_outflow_bc& B = bcs[b];
    if (!in_box(p, B, cell)) continue;
    const int8_t st = state[me];
    if (st == DEM_STATE_NONEXISTENT || st >= DEM_STATE_NORMAL_GHOST || st == DEM_STATE_ENTERING) continue;
    double fz[3]; int idx; double sgn;
    plane_of(B.plane, fz, idx, sgn);
    const double4 X = pos4[me];
    const double xi = idx == 0 ? X.x : (idx == 1 ? X.y : X.z);
    const double dist = (B.plane == 'N' || B.plane == 'E' || B.plane == 'T') ? xi - B.face : B.face - xi;
    if (dist > X.w) {
      state[me] = DEM_STATE_NORMAL;
    } else if (dist > 0.0) {
      double4 V = vel4[me];
      if (!B.mass_outflow) {
        const double vi = idx == 0 ? V.x : (idx == 1 ? V.y : V.z);
        if (vi * sgn > 0.0) {
          V.x = V.x * fz[0]; V.y = V.y * fz[1]; V.z = V.z * fz[2];
          vel4[me] = V;
          state[me] = DEM_STATE_EXITING;
        }
      } else {
        const int m = phase[me];
        V.x = B.vel[m][0]; V.y = B.vel[m][1]; V.z = B.vel[m][2];
        vel4[me] = V;
        state[me] = DEM_STATE_EXITING;
      }
    } else {
      const size_t n = (size_t)p.n;
      pos4[me] = make_double4(0.0, 0.0, 0.0, 0.0);
      vel4[me] = make_double4(0.0, 0.0, 0.0, 3.4028234663852886e38);  // PMASS = HUGE(0.0)
      omg4[me] = make_double4(0.0, 0.0, 0.0, 0.0);
      for (int c = 0; c < 3; ++c) { fc[c * n + me] = 0.0; tow[c * n + me] = 0.0; }
      for (int s = 0; s < p.cmax; ++s) wall_fid[(size_t)me * p.cmax + s] = -1;
      state[me] = DEM_STATE_NONEXISTENT;
      atomicAdd(&err->outflow_removed, 1ull);
    }
  }
}

}  // namespace

namespace demb {

int run_cfnewvalues_outflow(dem_handle* h, bool* force_nsearch) {
  ProfScope ps(h, DEM_PROF_INTEGRATE);
  h->dp.first_pass = h->first_pass ? 1 : 0;
  const int nbc = (int)h->obc.size();
  const int T = 256, G = (h->n + T - 1) / T, c = h->cur;
  const int ef = h->exit_first_pass ? 1 : 0;
  if (h->dp.intg == DEM_INTG_AB2)
    k_integrate_outflow<2><<<G, T, 0, h->stream>>>(h->dp, h->d_obc, nbc, ef, h->dg_pijk, h->pos4[c], h->vel4[c],
                                                   h->omg4[c], h->state, h->fc, h->tow, h->acc_old, h->rot_acc_old,
                                                   h->vslot);
  else
    k_integrate_outflow<1><<<G, T, 0, h->stream>>>(h->dp, h->d_obc, nbc, ef, h->dg_pijk, h->pos4[c], h->vel4[c],
                                                   h->omg4[c], h->state, h->fc, h->tow, h->acc_old, h->rot_acc_old,
                                                   h->vslot);
  DEM_LAUNCH(h);
  launch_skin(h);
  h->first_pass = false;
  h->exit_first_pass = false;
  if (int rc = run_mass_inflow(h)) return rc;  // MASS_INFLOW_DEM comes before MASS_OUTFLOW_DEM
  unsigned long long before = 0, after = 0;
  cudaMemcpyAsync(&before, &h->derr->outflow_removed, sizeof before, cudaMemcpyDeviceToHost, h->stream);
  k_mass_outflow<<<G, T, 0, h->stream>>>(h->dp, h->d_obc, nbc, h->dg_pijk, h->pos4[c], h->vel4[c], h->omg4[c],
                                        h->state, h->phase, h->fc, h->tow, h->wall_fid, h->derr);
  DEM_LAUNCH(h);
  cudaMemcpyAsync(&after, &h->derr->outflow_removed, sizeof after, cudaMemcpyDeviceToHost, h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "mass outflow")) return rc;
  *force_nsearch = after != before;
  return 0;
}

}  // namespace demb

extern "C" {

int dem_set_outflow_bcs(dem_handle* h, const dem_outflow_bc* bcs, int32_t n) {
  if (!h) return DEM_ERR_ARG;
  cudaSetDevice(h->dev);
  if (h->batch()) return set_err(h, DEM_ERR_ARG, "outflow boundaries are per system; not available on a batch handle");
  if (n < 0 || (n > 0 && !bcs)) return set_err(h, DEM_ERR_ARG, "bad outflow boundaries");
  for (int32_t b = 0; b < n; ++b) {
    const int pl = bcs[b].plane;
    if (pl != 'N' && pl != 'S' && pl != 'E' && pl != 'W' && pl != 'T' && pl != 'B')
      return set_err(h, DEM_ERR_ARG, "unknown BC_PLANE");
    for (int a = 0; a < 3; ++a)
      if (bcs[b].dg_lo[a] > bcs[b].dg_hi[a]) return set_err(h, DEM_ERR_ARG, "empty DES-cell box");
    for (int c = 0; c < b; ++c) {
      bool overlap = true;
      for (int a = 0; a < 3; ++a)
        overlap = overlap && bcs[b].dg_lo[a] <= bcs[c].dg_hi[a] && bcs[c].dg_lo[a] <= bcs[b].dg_hi[a];
      if (overlap) return set_err(h, DEM_ERR_ARG, "outflow boundary boxes overlap");
    }
  }
  cudaStreamSynchronize(h->stream);
  if (h->d_obc) { cudaFree(h->d_obc); h->d_obc = nullptr; }
  h->obc.assign(bcs, bcs + n);
  h->exit_first_pass = true;
  invalidate_graphs(h);
  if (n > 0) {
    if (int rc = check_cuda(h, cudaMalloc(&h->d_obc, sizeof(dem_outflow_bc) * n), "cudaMalloc outflow")) return rc;
    cudaMemcpyAsync(h->d_obc, bcs, sizeof(dem_outflow_bc) * n, cudaMemcpyHostToDevice, h->stream);
  }
  return check_cuda(h, cudaStreamSynchronize(h->stream), "outflow boundaries");
}

}  // extern "C"
