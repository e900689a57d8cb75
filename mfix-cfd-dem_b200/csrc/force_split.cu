// force_split.cu -- split-precision contact forces (FP32 forces, FP64
// history and integration).
//
// Same structure as the FP64 path (walls -> pairs -> gather, see force.cu)
// and the same contact law (calc_force_dem.f:204-506, cfrelvel.f:54-77), with
// this split of the arithmetic:
//   FP64  the displacement x_I - x_L and the velocity difference v_L - v_I
//         (differences of large, nearly equal numbers), |x_I - x_L| and the
//         normal overlap R_LM - |x_I - x_L|; the tangential-overlap history
//         update (PFT + DT*V_t, its magnitude and the Coulomb rescaling) and
//         the integration (CFNEWVALUES);
//   FP32  the unit normal, relative velocity at the contact point, spring and
//         damping coefficients, normal/tangential forces, torque arms and
//         rolling friction; per-particle sums use compensated (Neumaier)
//         FP32 accumulation.
// Wall contacts use the FP64 wall kernel.  This file is compiled with FMA
// contraction and fast single-precision square roots and divisions.
#include "dem_internal.cuh"

namespace demb {

struct PairRec32 {  // 40 bytes, fits in a PairRec slot
  float fc[3], tf[3], dcl2, dci2, kn, ov;
};
static_assert(sizeof(PairRec32) <= sizeof(PairRec), "record size");

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

template <int COLL, bool B>
__global__ void __launch_bounds__(256, 4)
k_pairs_split(DevParams p0, BatchView bv, const int* __restrict__ d_np, long long cap, const int* __restrict__ owner, const int* __restrict__ nbrs,
              const double4* __restrict__ pos4, const double4* __restrict__ vel4,
              const double4* __restrict__ omg4, const int8_t* __restrict__ state,
              const uint8_t* __restrict__ phase, double* __restrict__ pft, uint8_t* __restrict__ pflag,
              uint8_t* __restrict__ touched, const float* __restrict__ pgap, const double* __restrict__ skin,
              PairRec32* __restrict__ prec, DevErr* __restrict__ err) {
  // persistent grid-stride loop over the device-side pair count (the grid
  // size does not depend on the list, so the launch can live in a graph)
  const long long np = min((long long)*d_np, cap);
  const long long stride = (long long)gridDim.x * blockDim.x;
  unsigned long long ncont = 0;
  unsigned eflags = 0;
  const double reach = 2.0 * skin[0];
  // four consecutive pairs per iteration (see k_pairs in force.cu)
  const long long ng = (np + 3) / 4;
  for (long long g4 = (long long)blockIdx.x * blockDim.x + threadIdx.x; g4 < ng; g4 += stride) {
    const long long c0 = 4 * g4;
    uint32_t fw = 0;  // the four flags, one per byte
    float4 gq = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c0 + 3 < np) {
      fw = *reinterpret_cast<const uint32_t*>(pflag + c0);
      gq = *reinterpret_cast<const float4*>(pgap + c0);
    } else {
      if (c0 < np) { fw |= pflag[c0]; gq.x = pgap[c0]; }
      if (c0 + 1 < np) { fw |= (uint32_t)pflag[c0 + 1] << 8; gq.y = pgap[c0 + 1]; }
      if (c0 + 2 < np) { fw |= (uint32_t)pflag[c0 + 2] << 16; gq.z = pgap[c0 + 2]; }
    }
    // bit j: pair c0+j is provably apart
    const unsigned apart = ((!(fw & PF_HIST) && (double)gq.x > reach) ? 1u : 0u) |
                           ((!((fw >> 8) & PF_HIST) && (double)gq.y > reach) ? 2u : 0u) |
                           ((!((fw >> 16) & PF_HIST) && (double)gq.z > reach) ? 4u : 0u) |
                           ((!((fw >> 24) & PF_HIST) && (double)gq.w > reach) ? 8u : 0u);
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
    const long long cc = c0 + j;
    if (cc >= np) break;
    const uint8_t f0 = (uint8_t)(fw >> (8 * j));
    // provably apart (see k_pairs in force.cu)
    if ((apart >> j) & 1u) {
      if (f0) pflag[cc] = 0;
      continue;
    }
    const int ll = owner[cc], i = nbrs[cc];
    const DevParams& p = sysp<B>(p0, bv, ll);
    uint8_t f = f0 & PF_HIST;  // NONEXISTENT partner or zero distance: history kept
    double* po = pft + 3 * cc;  // history updated in place (see k_pairs in force.cu)
    if (state[i] != DEM_STATE_NONEXISTENT && state[ll] != DEM_STATE_NONEXISTENT) {
      const double4 a = pos4[ll], b = pos4[i];
      const double xl[3] = {a.x, a.y, a.z}, xi[3] = {b.x, b.y, b.z};
      double dist[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double pj = xi[c];
        const double s = periodic_shift(p, c, pj - xl[c]);
        if (s != 0.0) pj = pj + s;
        dist[c] = pj - xl[c];
      }
      const double r_lm = a.w + b.w;
      const double d2 = dist[0] * dist[0] + dist[1] * dist[1] + dist[2] * dist[2];
      if (d2 > (r_lm - SMALL_NUMBER) * (r_lm - SMALL_NUMBER)) {
        if (f0 & PF_HIST) { po[0] = 0.0; po[1] = 0.0; po[2] = 0.0; }
        f = 0;
      } else if (d2 == 0.0) {
        eflags |= EF_ZERO_DIST;
        err->zero_a = ll; err->zero_b = i;
      } else {
        const double dmag64 = sqrt(d2);
        const float dmag = (float)dmag64;
        const float ov = (float)(r_lm - dmag64);
        const float rl = (float)a.w, ri = (float)b.w;
        const float nrm[3] = {(float)dist[0] / dmag, (float)dist[1] / dmag, (float)dist[2] / dmag};
        const double4 va = vel4[ll], vb = vel4[i], wa = omg4[ll], wb = omg4[i];
        float vrel[3] = {(float)(va.x - vb.x), (float)(va.y - vb.y), (float)(va.z - vb.z)};
        const float dcl = (dmag * dmag + rl * rl - ri * ri) / (2.f * dmag);
        const float dci = dmag - dcl;
        const float osum[3] = {(float)wa.x * dcl + (float)wb.x * dci, (float)wa.y * dcl + (float)wb.y * dci,
                               (float)wa.z * dcl + (float)wb.z * dci};
        vrel[0] += osum[1] * nrm[2] - osum[2] * nrm[1];
        vrel[1] += osum[2] * nrm[0] - osum[0] * nrm[2];
        vrel[2] += osum[0] * nrm[1] - osum[1] * nrm[0];
        const float vrn = vrel[0] * nrm[0] + vrel[1] * nrm[1] + vrel[2] * nrm[2];
        const float vt[3] = {vrel[0] - vrn * nrm[0], vrel[1] - vrn * nrm[1], vrel[2] - vrn * nrm[2]};
        const int ix = phase[ll] * MAXP + phase[i];
        const float rad_eff = (rl * ri) / (rl + ri);
        const float ml = (float)va.w, mi = (float)vb.w;
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
        // tangential history in FP64
        double pin[3] = {0.0, 0.0, 0.0};
        if (f0 & PF_HIST) { pin[0] = po[0]; pin[1] = po[1]; pin[2] = po[2]; }
        double ot[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) ot[c] = p.dt * (double)vt[c] + pin[c];
        const double mag = sqrt(ot[0] * ot[0] + ot[1] * ot[1] + ot[2] * ot[2]);
        float ft[3] = {0.f, 0.f, 0.f};
        if (mag > 0.0) {
#pragma unroll
          for (int c = 0; c < 3; ++c) ft[c] = -kt * (float)ot[c] - etat * vt[c];
          const float ftmd = sqrtf(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
          const float fnmd = (float)p.mew * sqrtf(fn[0] * fn[0] + fn[1] * fn[1] + fn[2] * fn[2]);
          if (ftmd > fnmd) {
            const double sc = (double)fnmd / (double)kt / mag;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const double tg = ot[c] / mag;
              ft[c] = -fnmd * (float)tg;
              ot[c] = sc * ot[c];
            }
          }
        }
        po[0] = ot[0]; po[1] = ot[1]; po[2] = ot[2];
        PairRec32 r;
        r.dcl2 = dmag * 0.5f + (rl * rl - ri * ri) / (2.f * dmag);
        r.dci2 = dmag - r.dcl2;
        r.tf[0] = nrm[1] * ft[2] - nrm[2] * ft[1];
        r.tf[1] = nrm[2] * ft[0] - nrm[0] * ft[2];
        r.tf[2] = nrm[0] * ft[1] - nrm[1] * ft[0];
#pragma unroll
        for (int c = 0; c < 3; ++c) r.fc[c] = fn[c] + ft[c];
        r.kn = kn;
        r.ov = ov;
        prec[cc] = r;
        touched[ll] = 1;
        touched[i] = 1;
        f = PF_CONTACT | ((ot[0] != 0.0 || ot[1] != 0.0 || ot[2] != 0.0) ? PF_HIST : 0);
        ++ncont;
      }
    }
    if (f != f0) pflag[cc] = f;
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

template <int MODE, bool B>
__global__ void __launch_bounds__(256)
k_gather_split(DevParams p0, BatchView bv, const double4* __restrict__ pos_c, const double4* __restrict__ vel_c,
               const double4* __restrict__ omg_c, double4* __restrict__ pos_n, double4* __restrict__ vel_n,
               double4* __restrict__ omg_n, const int8_t* __restrict__ state, const double* __restrict__ wf,
               const int* __restrict__ row_end, const int* __restrict__ in_start,
               const int2* __restrict__ in_pair, const uint8_t* __restrict__ pflag, uint8_t* __restrict__ touched,
               uint8_t* __restrict__ wall_hit,
               const PairRec32* __restrict__ prec, double* __restrict__ fc, double* __restrict__ tow,
               double* __restrict__ acc_old, double* __restrict__ rot_acc_old, unsigned* __restrict__ vslot,
         CellOut cells) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= p0.n) return;
  const DevParams& p = sysp<B>(p0, bv, me);
  const int8_t st = state[me];
  const double4 X = pos_c[me], V = vel_c[me], W = omg_c[me];
  const double x[3] = {X.x, X.y, X.z}, v[3] = {V.x, V.y, V.z}, w[3] = {W.x, W.y, W.z};
  const double r = X.w, m = V.w, omoi = W.w;
  double f0[3] = {0.0, 0.0, 0.0}, t0[3] = {0.0, 0.0, 0.0};
  // the contacts of this pass; a particle in none has no terms to add
  const bool wh = wall_hit[me] != 0, ph = touched[me] != 0;
  if (wh) wall_hit[me] = 0;
  if (ph) touched[me] = 0;
  if (wh && st == DEM_STATE_NORMAL) {
    const double* o = wf + 6 * (size_t)me;
    f0[0] = o[0]; f0[1] = o[1]; f0[2] = o[2]; t0[0] = o[3]; t0[1] = o[4]; t0[2] = o[5];
  }
  Comp3 F, T;
  F.zero(); T.zero();
  if (st != DEM_STATE_NONEXISTENT && ph) {
    const float wf32[3] = {(float)w[0], (float)w[1], (float)w[2]};
    const float om = sqrtf(wf32[0] * wf32[0] + wf32[1] * wf32[1] + wf32[2] * wf32[2]);
    const bool roll = p.mew_r > 0.0 && om > 0.f;
    const float rf = (float)p.mew_r * (2.f * (float)r);
    const int rs = me ? row_end[me - 1] : 0, re = row_end[me];
    const int is = in_start[me], ie = in_start[me + 1];
    auto add = [&](const PairRec32& o, bool nbr) {
#pragma unroll
      for (int c = 0; c < 3; ++c) { F.add(c, nbr ? -o.fc[c] : o.fc[c]); T.add(c, (nbr ? o.dci2 : o.dcl2) * o.tf[c]); }
      if (roll) {
        const float s = -(rf * o.kn * o.ov) / om;
#pragma unroll
        for (int c = 0; c < 3; ++c) T.add(c, s * wf32[c]);
      }
    };
    // 32 entries at a time: the window's contact flags first (independent
    // loads), then the flagged records, each load issued before the
    // previous record is added
    auto flagged = [&](unsigned mask, auto idx, bool nbr) {
      if (!mask) return;
      PairRec32 cur = prec[idx(__ffs(mask) - 1)];
      mask &= mask - 1u;
      while (true) {
        const bool more = mask != 0u;
        PairRec32 nxt;
        if (more) { nxt = prec[idx(__ffs(mask) - 1)]; mask &= mask - 1u; }
        add(cur, nbr);
        if (!more) break;
        cur = nxt;
      }
    };
    for (int base = is; base < ie; base += 32) {
      const int cnt = min(32, ie - base);
      unsigned mask = 0u;
#pragma unroll 8
      for (int k = 0; k < 32; ++k)
        if (k < cnt && (pflag[in_pair[base + k].y] & PF_CONTACT)) mask |= 1u << k;
      flagged(mask, [&](int k) { return in_pair[base + k].y; }, true);
    }
    for (int base = rs; base < re; base += 32) {
      const int cnt = min(32, re - base);
      unsigned mask = 0u;
#pragma unroll 8
      for (int k = 0; k < 32; ++k)
        if (k < cnt && (pflag[base + k] & PF_CONTACT)) mask |= 1u << k;
      flagged(mask, [&](int k) { return base + k; }, false);
    }
  }
  double f[3], t[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) { f[c] = f0[c] + F.value(c); t[c] = t0[c] + T.value(c); }
  finish_particle<MODE>(p, me, st, x, v, w, r, m, omoi, f, t, pos_n, vel_n, omg_n, fc, tow, acc_old,
                        rot_acc_old, vslot, cells);
}

template <int COLL, bool B>
static void launch_pairs_split_t(dem_handle* h) {
  const int c = h->cur;
  const int T = h->tune.pair_threads;
  k_pairs_split<COLL, B><<<(unsigned)(h->n_sm * h->tune.pair_bpsm), T, 0, h->stream>>>(
      h->dp, h->bview(), h->d_np, h->pair_cap, h->pair_owner, h->nbrs[h->rb], h->pos4[c], h->vel4[c], h->omg4[c],
      h->state, h->phase, h->pft[h->pcur], h->pflag, h->touched, h->pgap, h->skin, (PairRec32*)h->prec,
      h->derr);
  DEM_LAUNCH(h);
}

void launch_pairs_split(dem_handle* h) {
  const bool hz = h->dp.coll == DEM_COLL_HERTZ;
  if (h->batch()) hz ? launch_pairs_split_t<DEM_COLL_HERTZ, true>(h) : launch_pairs_split_t<DEM_COLL_LSD, true>(h);
  else hz ? launch_pairs_split_t<DEM_COLL_HERTZ, false>(h) : launch_pairs_split_t<DEM_COLL_LSD, false>(h);
}

template <int MODE, bool B>
static void launch_gather_split_t(dem_handle* h) {
  const int T = h->tune.gather_threads, G = (h->n + T - 1) / T;
  const int c = h->cur;
  k_gather_split<MODE, B><<<G, T, 0, h->stream>>>(
      h->dp, h->bview(), h->pos4[c], h->vel4[c], h->omg4[c], h->pos4[1 - c], h->vel4[1 - c], h->omg4[1 - c],
      h->state, h->wf, h->row_end[h->rb], h->in_start, h->in_pair, h->pflag,
      h->touched, h->wall_hit, (const PairRec32*)h->prec, h->fc, h->tow, h->acc_old, h->rot_acc_old, h->vslot,
      gather_cells<MODE, B>(h));
  DEM_LAUNCH(h);
}

void launch_gather_split(dem_handle* h, int mode) {
  const bool bt = h->batch();
  if (mode == 0) bt ? launch_gather_split_t<0, true>(h) : launch_gather_split_t<0, false>(h);
  else if (mode == 1) bt ? launch_gather_split_t<1, true>(h) : launch_gather_split_t<1, false>(h);
  else bt ? launch_gather_split_t<2, true>(h) : launch_gather_split_t<2, false>(h);
}

}  // namespace demb
