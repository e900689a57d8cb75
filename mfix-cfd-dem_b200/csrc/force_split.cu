// force_split.cu -- split-precision contact forces (FP32 forces, FP64
// history and integration), one fused pass per step.
//
// Same contact law as the FP64 path (calc_force_dem.f:204-506 with
// CFRELVEL, cfrelvel.f:54-77) with this split of the arithmetic:
//   FP64  the displacement x_I - x_L and the velocity difference v_L - v_I
//         (differences of large, nearly equal numbers), the squared
//         distance and R_LM^2 - |x_I - x_L|^2 (the overlap is this over
//         R_LM + |x_I - x_L|, so no FP64 square root is needed), the
//         tangential-overlap history update PFT + DT*V_t and its Coulomb
//         rescaling, and the integration (CFNEWVALUES);
//   FP32  the unit normal, relative velocity at the contact point, spring and
//         damping coefficients, normal/tangential forces, torque arms and
//         rolling friction; per-particle sums use compensated (Neumaier)
//         FP32 accumulation.
//
// Structure: a group of lanes per particle walks every pair the particle is
// in -- the incoming entries of the transpose (pairs owned by other
// particles) and its own row -- and evaluates each contact itself, with the
// owner as L and the neighbour as I, through a single code path, so both
// particles of a pair compute bit-identical pair forces (equal and
// opposite).  No
// per-pair record goes through memory.  The history is double-buffered:
// both particles read PFT and the flags from buffer pcur, only the owner
// writes buffer 1 - pcur (flags of every row entry, PFT of pairs whose new
// history is nonzero), and the caller flips pcur after the pass.  The sum
// order differs from the serial reference (split results are compared with
// the FP64 path by the stated force tolerance, not bit for bit).  Wall terms
// come from the FP64 wall kernel (force.cu).
//
// This file is compiled with FMA contraction and fast single-precision
// square roots and divisions.
#include "dem_internal.cuh"

namespace demb {

struct Comp3 {  // Neumaier-compensated FP32 sum of a 3-vector
  float s[3], c[3];
  __device__ void zero() { for (int k = 0; k < 3; ++k) { s[k] = 0.f; c[k] = 0.f; } }
  __device__ __forceinline__ void add(int k, float x) {
    const float t = s[k] + x;
    if (fabsf(s[k]) >= fabsf(x)) c[k] += (s[k] - t) + x;
    else c[k] += (x - t) + s[k];
    s[k] = t;
  }
  __device__ __forceinline__ double value(int k) const { return (double)s[k] + (double)c[k]; }
};

// The pair force of one contact with L the owner and I the neighbour (the
// split arithmetic above): the force on L (fc; I receives -fc), the torque
// vector n x Ft with the two lever arms, KN and the overlap (rolling
// friction), and the new history ot.  dist = x_I - x_L, d2 = |dist|^2 and
// ovd = R_LM^2 - d2 come from the contact test in FP64.
struct PairTerms {
  float fc[3], tf[3], dcl2, dci2, kn, ov;
};

template <int COLL>
__device__ __forceinline__ void split_contact(const DevParams& p, const double4& xl, const double4& vl,
                                              const double4& wl, int phl, const double4& xi, const double4& vi,
                                              const double4& wi, int phi, const double dist[3], double d2,
                                              double ovd, const double pin[3], double ot[3], PairTerms& o) {
  const float rl = (float)xl.w, ri = (float)xi.w;
  const float dmag = sqrtf((float)d2);
  const float ov = (float)ovd / ((rl + ri) + dmag);
  const float inv = 1.f / dmag;
  const float nrm[3] = {(float)dist[0] * inv, (float)dist[1] * inv, (float)dist[2] * inv};
  float vrel[3] = {(float)(vl.x - vi.x), (float)(vl.y - vi.y), (float)(vl.z - vi.z)};
  const float dcl = 0.5f * dmag + (rl - ri) * (rl + ri) * (0.5f * inv);
  const float dci = dmag - dcl;
  const float osum[3] = {(float)wl.x * dcl + (float)wi.x * dci, (float)wl.y * dcl + (float)wi.y * dci,
                         (float)wl.z * dcl + (float)wi.z * dci};
  vrel[0] += osum[1] * nrm[2] - osum[2] * nrm[1];
  vrel[1] += osum[2] * nrm[0] - osum[0] * nrm[2];
  vrel[2] += osum[0] * nrm[1] - osum[1] * nrm[0];
  const float vrn = vrel[0] * nrm[0] + vrel[1] * nrm[1] + vrel[2] * nrm[2];
  const float vt[3] = {vrel[0] - vrn * nrm[0], vrel[1] - vrn * nrm[1], vrel[2] - vrn * nrm[2]};
  const int ix = phl * MAXP + phi;
  const float rad_eff = (rl * ri) / (rl + ri);
  const float ml = (float)vl.w, mi = (float)vi.w;
  const float m_eff = (ml * mi) / (ml + mi);
  float kn, kt, etan, etat;
  if (COLL == DEM_COLL_HERTZ) {
    float so = sqrtf(ov);
    const float sre = sqrtf(rad_eff);
    const float hkn = (float)p.hkn[ix], hkt = (float)p.hkt[ix];
    kn = hkn * so * sre;
    kt = hkt * so * sre;
    so = sqrtf(so);
    etan = (float)p.etan[ix] * so * sqrtf(hkn * sre * m_eff);
    etat = (float)p.etat[ix] * so * sqrtf(hkt * sre * m_eff);
  } else {
    kn = (float)p.kn; kt = (float)p.kt;
    const float sm = sqrtf(m_eff);
    etan = (float)p.etan[ix] * sm;
    etat = (float)p.etat[ix] * sm;
  }
  float fn[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) fn[c] = -(kn * ov + etan * vrn) * nrm[c];
  // tangential history in FP64: PFT + DT*V_t
#pragma unroll
  for (int c = 0; c < 3; ++c) ot[c] = p.dt * (double)vt[c] + pin[c];
  const float o32[3] = {(float)ot[0], (float)ot[1], (float)ot[2]};
  const float mag = sqrtf(o32[0] * o32[0] + o32[1] * o32[1] + o32[2] * o32[2]);
  float ft[3] = {0.f, 0.f, 0.f};
  if (mag > 0.f) {
#pragma unroll
    for (int c = 0; c < 3; ++c) ft[c] = -kt * o32[c] - etat * vt[c];
    const float ftmd = sqrtf(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
    const float fnmd = (float)p.mew * sqrtf(fn[0] * fn[0] + fn[1] * fn[1] + fn[2] * fn[2]);
    if (ftmd > fnmd) {
      // Coulomb slip: Ft = -|Fn|*mu t, history (|Fn|*mu/Kt) t with t = ot/|ot|
      const float im = 1.f / mag;
#pragma unroll
      for (int c = 0; c < 3; ++c) ft[c] = -fnmd * (o32[c] * im);
      const double sc = (double)(fnmd / kt * im);
#pragma unroll
      for (int c = 0; c < 3; ++c) ot[c] = sc * ot[c];
    }
  }
  o.dcl2 = dcl;
  o.dci2 = dci;
  o.tf[0] = nrm[1] * ft[2] - nrm[2] * ft[1];
  o.tf[1] = nrm[2] * ft[0] - nrm[0] * ft[2];
  o.tf[2] = nrm[0] * ft[1] - nrm[1] * ft[0];
#pragma unroll
  for (int c = 0; c < 3; ++c) o.fc[c] = fn[c] + ft[c];
  o.kn = kn;
  o.ov = ov;
}

// G lanes per particle (G = 1, 2, 4 or 8, consecutive lanes of a warp): lane
// j of the group takes entries j, j + G, ... of the particle's list -- k < nin:
// incoming entry in_pair[is + k] = (owner, pair); otherwise the particle's
// own row -- so the group has G entries' loads in flight at a time.  Each
// lane keeps compensated FP32 sums of its entries; the group adds the lanes'
// sums in FP64 in a fixed shuffle order, so results do not depend on timing.
// Lane 0 adds the wall terms (k_walls) and integrates (MODE 1 Euler, 2
// Adams-Bashforth) or stores the forces into FC/TOW (MODE 0).  Pairs that the
// build's gap and the displacement bound since prove apart (with no history)
// are skipped after reading their flag and gap, by both particles alike.
// The owner of a pair writes its output flag and keeps its output history
// slot exact: the new history where it is nonzero, zeros where the slot held
// history (its old output flag says so) and no longer does.
template <int COLL, int MODE, bool B, int G>
__global__ void __launch_bounds__(256)
k_force_split(DevParams p0, BatchView bv, const double4* __restrict__ pos_c, const double4* __restrict__ vel_c,
              const double4* __restrict__ omg_c, double4* __restrict__ pos_n, double4* __restrict__ vel_n,
              double4* __restrict__ omg_n, const int8_t* __restrict__ state, const uint8_t* __restrict__ phase,
              const double* __restrict__ wf, uint8_t* __restrict__ wall_hit, const int* __restrict__ row_end,
              const int* __restrict__ nbrs, const int* __restrict__ in_start, const int2* __restrict__ in_pair,
              const double* __restrict__ pft_in, double* __restrict__ pft_out, const uint8_t* __restrict__ flag_in,
              uint8_t* __restrict__ flag_out, const float* __restrict__ pgap, const double* __restrict__ skin,
              double* __restrict__ fc, double* __restrict__ tow, double* __restrict__ acc_old,
              double* __restrict__ rot_acc_old, unsigned* __restrict__ vslot, DevErr* __restrict__ err,
              CellOut cells) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int me = (int)(t / G);
  const int lane = (int)(t % G);
  unsigned long long ncont = 0;
  unsigned eflags = 0;
  if (me < p0.n) {
    const DevParams& p = sysp<B>(p0, bv, me);
    const int8_t st = state[me];
    const double4 X = pos_c[me], V = vel_c[me], W = omg_c[me];
    const int ph = phase[me];
    Comp3 F, T;
    F.zero(); T.zero();
    const float w32[3] = {(float)W.x, (float)W.y, (float)W.z};
    const float om = sqrtf(w32[0] * w32[0] + w32[1] * w32[1] + w32[2] * w32[2]);
    const bool roll = p.mew_r > 0.0 && om > 0.f;
    const float rf = (float)p.mew_r * (2.f * (float)X.w) / (om > 0.f ? om : 1.f);
    const double reach = 2.0 * skin[0];
    const int rs = me ? row_end[me - 1] : 0, re = row_end[me];
    // a NONEXISTENT particle adds no force, but it still carries its own
    // row's history and flags into the output buffers
    const int is = st != DEM_STATE_NONEXISTENT ? in_start[me] : 0;
    const int nin = st != DEM_STATE_NONEXISTENT ? in_start[me + 1] - is : 0;
    const int ntot = nin + (re - rs);
    for (int k = lane; k < ntot; k += G) {
      int other, cc;
      bool own;
      if (k < nin) {
        const int2 e = in_pair[is + k];
        other = e.x; cc = e.y; own = false;
      } else {
        cc = rs + (k - nin); other = nbrs[cc]; own = true;
      }
      const uint8_t f0b = flag_in[cc];
      uint8_t fnew = 0;
      bool carry = false;
      double ot[3] = {0.0, 0.0, 0.0};
      // provably apart, history zero (stays zero): nothing to add or carry
      if ((f0b & PF_HIST) || !((double)pgap[cc] > reach)) {
        const int8_t so = state[other];
        fnew = f0b & PF_HIST;  // NONEXISTENT partner or zero distance: history kept
        carry = true;
        if (st != DEM_STATE_NONEXISTENT && so != DEM_STATE_NONEXISTENT) {
          const double4 xo = pos_c[other];
          // L is the owner, I the neighbour, for both particles of the pair
          const double4& xl = own ? X : xo;
          const double4& xi = own ? xo : X;
          double dist[3];
          {
            const double a[3] = {xl.x, xl.y, xl.z}, b[3] = {xi.x, xi.y, xi.z};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              double pj = b[c];
              const double sh = periodic_shift(p, c, pj - a[c]);
              if (sh != 0.0) pj = pj + sh;
              dist[c] = pj - a[c];
            }
          }
          const double r_lm = xl.w + xi.w;
          const double d2 = dist[0] * dist[0] + dist[1] * dist[1] + dist[2] * dist[2];
          if (d2 > (r_lm - SMALL_NUMBER) * (r_lm - SMALL_NUMBER)) {
            fnew = 0;  // apart: history reset
            carry = false;
          } else if (d2 == 0.0) {
            if (own) {
              eflags |= EF_ZERO_DIST;
              err->zero_a = me; err->zero_b = other;
            }
          } else {
            const double4 vo = vel_c[other], wo = omg_c[other];
            const int pho = phase[other];
            double pin[3] = {0.0, 0.0, 0.0};
            if (f0b & PF_HIST) {
              const double* q = pft_in + 3 * (size_t)cc;
              pin[0] = q[0]; pin[1] = q[1]; pin[2] = q[2];
            }
            PairTerms o;
            if (own) split_contact<COLL>(p, X, V, W, ph, xo, vo, wo, pho, dist, d2, r_lm * r_lm - d2, pin, ot, o);
            else split_contact<COLL>(p, xo, vo, wo, pho, X, V, W, ph, dist, d2, r_lm * r_lm - d2, pin, ot, o);
            const float sg = own ? 1.f : -1.f;
            const float arm = own ? o.dcl2 : o.dci2;
#pragma unroll
            for (int c = 0; c < 3; ++c) { F.add(c, sg * o.fc[c]); T.add(c, arm * o.tf[c]); }
            if (roll) {
              const float sr = -(rf * o.kn * o.ov);
#pragma unroll
              for (int c = 0; c < 3; ++c) T.add(c, sr * w32[c]);
            }
            fnew = PF_CONTACT | ((ot[0] != 0.0 || ot[1] != 0.0 || ot[2] != 0.0) ? PF_HIST : 0);
            carry = false;
            if (own) ++ncont;
          }
        }
      }
      if (own) {
        const uint8_t fold = flag_out[cc];
        flag_out[cc] = fnew;
        double* q = pft_out + 3 * (size_t)cc;
        if (fnew & PF_HIST) {
          if (carry) {
            const double* a = pft_in + 3 * (size_t)cc;
            q[0] = a[0]; q[1] = a[1]; q[2] = a[2];
          } else {
            q[0] = ot[0]; q[1] = ot[1]; q[2] = ot[2];
          }
        } else if (fold & PF_HIST) {
          q[0] = 0.0; q[1] = 0.0; q[2] = 0.0;
        }
      }
    }
    // the group's sums in FP64, lanes added in a fixed order
    double f[3], tq[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) { f[c] = F.value(c); tq[c] = T.value(c); }
    if constexpr (G > 1) {
      const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << ((threadIdx.x & 31) & ~(G - 1));
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          f[c] += __shfl_down_sync(gmask, f[c], o, G);
          tq[c] += __shfl_down_sync(gmask, tq[c], o, G);
        }
      }
    }
    if (lane == 0) {
      double f0[3] = {0.0, 0.0, 0.0}, t0[3] = {0.0, 0.0, 0.0};
      if (wall_hit[me]) {
        wall_hit[me] = 0;
        if (st == DEM_STATE_NORMAL) {
          const double* o = wf + 6 * (size_t)me;
          f0[0] = o[0]; f0[1] = o[1]; f0[2] = o[2]; t0[0] = o[3]; t0[1] = o[4]; t0[2] = o[5];
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) { f[c] = f0[c] + f[c]; tq[c] = t0[c] + tq[c]; }
      const double x[3] = {X.x, X.y, X.z}, v[3] = {V.x, V.y, V.z}, w[3] = {W.x, W.y, W.z};
      finish_particle<MODE>(p, me, st, x, v, w, X.w, V.w, W.w, f, tq, pos_n, vel_n, omg_n, fc, tow, acc_old,
                            rot_acc_old, vslot, cells);
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

template <int COLL, int MODE, bool B, int L>
static void launch_force_split_t(dem_handle* h) {
  const int T = h->tune.gather_threads;
  const unsigned G = (unsigned)(((long long)h->n * L + T - 1) / T);
  const int c = h->cur, pc = h->pcur;
  k_force_split<COLL, MODE, B, L><<<G, T, 0, h->stream>>>(
      h->dp, h->bview(), h->pos4[c], h->vel4[c], h->omg4[c], h->pos4[1 - c], h->vel4[1 - c], h->omg4[1 - c],
      h->state, h->phase, h->wf, h->wall_hit, h->row_end[h->rb], h->nbrs[h->rb], h->in_start, h->in_pair,
      h->pft[pc], h->pft[1 - pc], h->pflagb[pc], h->pflagb[1 - pc], h->pgap, h->skin, h->fc, h->tow, h->acc_old,
      h->rot_acc_old, h->vslot, h->derr, gather_cells<MODE, B>(h));
  DEM_LAUNCH(h);
}

template <int MODE, int L>
static void launch_force_split_l(dem_handle* h) {
  const bool hz = h->dp.coll == DEM_COLL_HERTZ;
  if (h->batch()) hz ? launch_force_split_t<DEM_COLL_HERTZ, MODE, true, L>(h) : launch_force_split_t<DEM_COLL_LSD, MODE, true, L>(h);
  else hz ? launch_force_split_t<DEM_COLL_HERTZ, MODE, false, L>(h) : launch_force_split_t<DEM_COLL_LSD, MODE, false, L>(h);
}

template <int MODE>
static void launch_force_split_m(dem_handle* h) {
  switch (h->tune.split_lanes) {
    case 1: launch_force_split_l<MODE, 1>(h); break;
    case 2: launch_force_split_l<MODE, 2>(h); break;
    case 8: launch_force_split_l<MODE, 8>(h); break;
    default: launch_force_split_l<MODE, 4>(h); break;
  }
}

// The fused split pass: reads history buffer pcur, writes 1 - pcur (the
// caller flips pcur when the pass counts as a step).
void launch_force_split(dem_handle* h, int mode) {
  if (mode == 0) launch_force_split_m<0>(h);
  else if (mode == 1) launch_force_split_m<1>(h);
  else launch_force_split_m<2>(h);
}

}  // namespace demb
