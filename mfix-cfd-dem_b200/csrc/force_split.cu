// force_split.cu -- split-precision contact forces (FP32 forces, FP64
// history and integration).
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
// Structure: the pair kernel evaluates every contact once (a thread per
// pair, consecutive pairs of the half list) and writes each particle's terms
// as a 32-byte FP32 record: the owner's at the pair index (rec_own, in row
// order) and the neighbour's at the pair's slot of the neighbour's incoming
// list (rec_in[in_pos[cc]], the transpose order).  The neighbour-side writes
// are scattered but never waited on; the per-particle kernel then reads its
// own row and its incoming list as two contiguous ranges, with no random
// load.  Contact flags: PF_CONTACT of pflag for the owner's records (row
// order), and in_flag (transpose order) for the neighbour's, written only
// when a pair's contact state changes.  Wall terms come from the FP64 wall
// kernel (force.cu).  The sum order differs from the serial reference;
// split results are compared with the FP64 path by the stated force
// tolerance, not bit for bit.
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
  bool near;  // the FP32 onset-of-slip test lies within 1e-4 of its threshold
};

// The onset-of-slip test of calc_force_dem.f:330-337 in FP64, evaluated as
// the FP64 kernels do (contact_force), for owner state (xl, vl, wl) and
// neighbour state (xi, vi, wi) with dist = x_I - x_L and history pin.  The
// friction law turns the tangential force at the onset of slip (below it
// -KT*OVERLAP_T - ETAT*VREL_T, above it MEW*|FN| along OVERLAP_T), so a
// contact whose FP32 test lies within the FP32 error of the threshold takes
// its branch from this test (k_slip_fix).
template <int COLL>
__device__ __forceinline__ bool slip_fp64(const DevParams& p, const double4& xl, const double4& vl,
                                          const double4& wl, const double4& xi, const double4& vi,
                                          const double4& wi, int ix, const double dist[3], double d2,
                                          const double pin[3]) {
  const double rl = xl.w, ri = xi.w;
  const double dmag = sqrt(d2);
  const double nrm[3] = {dist[0] / dmag, dist[1] / dmag, dist[2] / dmag};
  const double overlap_n = (rl + ri) - dmag;
  const double dcl = (dmag * dmag + rl * rl - ri * ri) / (2.0 * dmag);
  const double dci = dmag - dcl;
  const double osum[3] = {wl.x * dcl + wi.x * dci, wl.y * dcl + wi.y * dci, wl.z * dcl + wi.z * dci};
  const double vrel[3] = {vl.x - vi.x + (osum[1] * nrm[2] - osum[2] * nrm[1]),
                          vl.y - vi.y + (osum[2] * nrm[0] - osum[0] * nrm[2]),
                          vl.z - vi.z + (osum[0] * nrm[1] - osum[1] * nrm[0])};
  const double vrn = vrel[0] * nrm[0] + vrel[1] * nrm[1] + vrel[2] * nrm[2];
  const double vt[3] = {vrel[0] - vrn * nrm[0], vrel[1] - vrn * nrm[1], vrel[2] - vrn * nrm[2]};
  const double rad_eff = (rl * ri) / (rl + ri);
  const double m_eff = (vl.w * vi.w) / (vl.w + vi.w);
  double kn, kt, etan, etat;
  if (COLL == DEM_COLL_HERTZ) {
    double so = sqrt(overlap_n);
    kn = p.hkn[ix] * so * sqrt(rad_eff);
    kt = p.hkt[ix] * so * sqrt(rad_eff);
    so = sqrt(so);
    etan = p.etan[ix] * so * sqrt(p.hkn[ix] * sqrt(rad_eff) * m_eff);
    etat = p.etat[ix] * so * sqrt(p.hkt[ix] * sqrt(rad_eff) * m_eff);
  } else {
    kn = p.kn; kt = p.kt;
    etan = p.etan[ix] * sqrt(m_eff);
    etat = p.etat[ix] * sqrt(m_eff);
  }
  double fn2 = 0.0, ft2 = 0.0, ot2 = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double fn = -(kn * overlap_n * nrm[c] + etan * vrn * nrm[c]);
    const double ot = p.dt * vt[c] + pin[c];
    const double ft = -kt * ot - etat * vt[c];
    fn2 += fn * fn;
    ot2 += ot * ot;
    ft2 += ft * ft;
  }
  if (!(ot2 > 0.0)) return false;
  return sqrt(ft2) > p.mew * sqrt(fn2);
}

// FIX false: the pair kernel's evaluation, the onset of slip decided in
// FP32 and o.near set near its threshold; FIX true: the same evaluation
// with the onset of slip decided by slip_fp64 (k_slip_fix).
template <int COLL, bool FIX>
__device__ __forceinline__ void split_contact(const DevParams& p, const double4& xl, const double4& vl,
                                              const double4& wl, int phl, const double4& xi, const double4& vi,
                                              const double4& wi, int phi, const double dist[3], double d2,
                                              double ovd, const double pin[3], double ot[3], PairTerms& o) {
  const float rl = (float)xl.w, ri = (float)xi.w;
  const float d2f = (float)d2;
  const float inv = rsqrtf(d2f);
  const float dmag = d2f * inv;
  const float ov = (float)ovd / ((rl + ri) + dmag);
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
    // KN = HERT_KN*sqrt(ov)*sqrt(R_eff) = HERT_KN*q with q = sqrt(ov*R_eff);
    // ETA_N = DES_ETAN*ov^(1/4)*sqrt(HERT_KN*sqrt(R_eff)*M_eff)
    //       = DES_ETAN*sqrt(HERT_KN)*sqrt(q*M_eff), and the same for t
    const float q = sqrtf(ov * rad_eff);
    const float sqm = sqrtf(q * m_eff);
    kn = p.hkn32[ix] * q;
    kt = p.hkt32[ix] * q;
    etan = p.etan_sq32[ix] * sqm;
    etat = p.etat_sq32[ix] * sqm;
  } else {
    kn = p.kn32; kt = p.kt32;
    const float sm = sqrtf(m_eff);
    etan = p.etan32[ix] * sm;
    etat = p.etat32[ix] * sm;
  }
  float fn[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) fn[c] = -(kn * ov + etan * vrn) * nrm[c];
  // tangential history in FP64: PFT + DT*V_t
#pragma unroll
  for (int c = 0; c < 3; ++c) ot[c] = p.dt * (double)vt[c] + pin[c];
  const float o32[3] = {(float)ot[0], (float)ot[1], (float)ot[2]};
  const float mag2 = o32[0] * o32[0] + o32[1] * o32[1] + o32[2] * o32[2];
  float ft[3] = {0.f, 0.f, 0.f};
  o.near = false;
  if (mag2 > 0.f) {
#pragma unroll
    for (int c = 0; c < 3; ++c) ft[c] = -kt * o32[c] - etat * vt[c];
    const float ft2 = ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2];
    const float fn2 = fn[0] * fn[0] + fn[1] * fn[1] + fn[2] * fn[2];
    // |Ft| > MEW*|Fn|, compared squared
    const float thr = p.mew32 * p.mew32 * fn2;
    bool slip;
    if (FIX) {
      slip = slip_fp64<COLL>(p, xl, vl, wl, xi, vi, wi, ix, dist, d2, pin);
    } else {
      slip = ft2 > thr;
      o.near = fabsf(ft2 - thr) <= 1e-4f * thr;
    }
    if (slip) {
      // Coulomb slip: Ft = -MEW*|Fn| t, history (MEW*|Fn|/KT) t, t = ot/|ot|
      const float fnmd = p.mew32 * sqrtf(fn2);
      const float im = rsqrtf(mag2);
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

// One particle's terms of a contact: (force, KN*OVERLAP) and (torque, 0).
struct Rec32 {
  float4 a, b;
};

// The owner's record of a contact at its pair index, the neighbour's at its
// incoming slot.
__device__ __forceinline__ void put_records(const PairTerms& o, long long cc, const int* __restrict__ in_pos,
                                            Rec32* __restrict__ rec_own, Rec32* __restrict__ rec_in) {
  const float rol = o.kn * o.ov;
  Rec32 ro, ri;
  ro.a = make_float4(o.fc[0], o.fc[1], o.fc[2], rol);
  ro.b = make_float4(o.dcl2 * o.tf[0], o.dcl2 * o.tf[1], o.dcl2 * o.tf[2], 0.f);
  ri.a = make_float4(-o.fc[0], -o.fc[1], -o.fc[2], rol);
  ri.b = make_float4(o.dci2 * o.tf[0], o.dci2 * o.tf[1], o.dci2 * o.tf[2], 0.f);
  rec_own[cc] = ro;
  rec_in[in_pos[cc]] = ri;
}

// Kernel 1 (per pair): one CC iteration of CALC_FORCE_DEM, evaluated once.
// A pair that the build's gap and the displacement bound since prove apart
// (history zero) is skipped after reading its flag and gap.  Four
// consecutive pairs per thread-iteration: their flags and gaps arrive in one
// load each.
template <int COLL, bool B>
__global__ void __launch_bounds__(256, 4)
k_pairs_split(DevParams p0, BatchView bv, const int* __restrict__ d_np, long long cap, const int* __restrict__ owner,
              const int* __restrict__ nbrs, const int* __restrict__ in_pos, const double4* __restrict__ pos4,
              const double4* __restrict__ vel4, const double4* __restrict__ omg4, const int8_t* __restrict__ state,
              const uint8_t* __restrict__ phase, double* __restrict__ pft, uint8_t* __restrict__ pflag,
              uint8_t* __restrict__ in_flag, uint8_t* __restrict__ touched, const float* __restrict__ pgap,
              const double* __restrict__ skin, Rec32* __restrict__ rec_own, Rec32* __restrict__ rec_in,
              SlipFix* __restrict__ fix, DevErr* __restrict__ err) {
  const long long np = min((long long)*d_np, cap);
  const long long stride = (long long)gridDim.x * blockDim.x;
  // the bound in FP32, rounded up: a pair is skipped only when its gap
  // (rounded down at the build) exceeds it
  const float reach = __double2float_ru(2.0 * skin[0]);
  unsigned long long ncont = 0;
  unsigned eflags = 0;
  const long long ng = (np + 3) / 4;
  for (long long g4 = (long long)blockIdx.x * blockDim.x + threadIdx.x; g4 < ng; g4 += stride) {
    const long long c0 = 4 * g4;
    uint32_t fw = 0;
    float4 gq = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c0 + 3 < np) {
      fw = *reinterpret_cast<const uint32_t*>(pflag + c0);
      gq = *reinterpret_cast<const float4*>(pgap + c0);
    } else {
      if (c0 < np) { fw |= pflag[c0]; gq.x = pgap[c0]; }
      if (c0 + 1 < np) { fw |= (uint32_t)pflag[c0 + 1] << 8; gq.y = pgap[c0 + 1]; }
      if (c0 + 2 < np) { fw |= (uint32_t)pflag[c0 + 2] << 16; gq.z = pgap[c0 + 2]; }
    }
    const unsigned apart = ((!(fw & PF_HIST) && gq.x > reach) ? 1u : 0u) |
                           ((!((fw >> 8) & PF_HIST) && gq.y > reach) ? 2u : 0u) |
                           ((!((fw >> 16) & PF_HIST) && gq.z > reach) ? 4u : 0u) |
                           ((!((fw >> 24) & PF_HIST) && gq.w > reach) ? 8u : 0u);
    // the particles of the group's pairs in one load each, when any pair
    // needs them (a group past the list's end has fewer than four)
    int4 o4 = make_int4(0, 0, 0, 0), n4 = make_int4(0, 0, 0, 0);
    const unsigned live = c0 + 3 < np ? 15u : (1u << (unsigned)(np - c0)) - 1u;
    if (~apart & live) {
      if (c0 + 3 < np) {
        o4 = *reinterpret_cast<const int4*>(owner + c0);
        n4 = *reinterpret_cast<const int4*>(nbrs + c0);
      } else {
        o4.x = owner[c0]; n4.x = nbrs[c0];
        if (c0 + 1 < np) { o4.y = owner[c0 + 1]; n4.y = nbrs[c0 + 1]; }
        if (c0 + 2 < np) { o4.z = owner[c0 + 2]; n4.z = nbrs[c0 + 2]; }
      }
    }
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
      const long long cc = c0 + j;
      if (cc >= np) break;
      const uint8_t f0 = (uint8_t)(fw >> (8 * j));
      uint8_t f;
      if ((apart >> j) & 1u) {
        f = 0;
      } else {
        const int ll = j == 0 ? o4.x : (j == 1 ? o4.y : (j == 2 ? o4.z : o4.w));
        const int i = j == 0 ? n4.x : (j == 1 ? n4.y : (j == 2 ? n4.z : n4.w));
        f = f0 & PF_HIST;  // NONEXISTENT partner or zero distance: history kept
        double* po = pft + 3 * cc;
        // the states and the positions in one round of loads (any slot's
        // position can be read; it is used only for existing particles)
        const double4 a = pos4[ll], b = pos4[i];
        const int8_t sl = state[ll], si = state[i];
        if (si != DEM_STATE_NONEXISTENT && sl != DEM_STATE_NONEXISTENT) {
          const DevParams& p = sysp<B>(p0, bv, ll);
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
            const double4 va = vel4[ll], vb = vel4[i], wa = omg4[ll], wb = omg4[i];
            double pin[3] = {0.0, 0.0, 0.0};
            if (f0 & PF_HIST) { pin[0] = po[0]; pin[1] = po[1]; pin[2] = po[2]; }
            double ot[3];
            PairTerms o;
            // one solids phase: no phase to look up
            const int phl = p.nph > 1 ? phase[ll] : 0, phi = p.nph > 1 ? phase[i] : 0;
            split_contact<COLL, false>(p, a, va, wa, phl, b, vb, wb, phi, dist, d2, r_lm * r_lm - d2, pin, ot, o);
            // near the onset of slip k_slip_fix evaluates the contact again,
            // from the history as it was (left in place here)
            bool deferred = false;
            if (o.near) {
              const unsigned t = atomicAdd(&fix->count, 1u);
              if (t < (unsigned)SLIP_FIX_CAP) {
                fix->pair[t] = 2 * cc + ((f0 & PF_HIST) ? 1 : 0);
                deferred = true;
              }
            }
            if (!deferred) { po[0] = ot[0]; po[1] = ot[1]; po[2] = ot[2]; }
            put_records(o, cc, in_pos, rec_own, rec_in);
            touched[ll] = 1;
            touched[i] = 1;
            f = PF_CONTACT | ((ot[0] != 0.0 || ot[1] != 0.0 || ot[2] != 0.0) ? PF_HIST : 0);
            ++ncont;
          }
        }
      }
      if (f != f0) {
        pflag[cc] = f;
        // the neighbour's view of the contact, in transpose order
        if ((f ^ f0) & PF_CONTACT) in_flag[in_pos[cc]] = f & PF_CONTACT;
      }
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

// The contacts k_pairs_split left near the onset of slip, evaluated again
// with the onset decided in FP64 (slip_fp64): history, flag and both
// records rewritten.  Their history is still the one the pair kernel read.
// One block; it clears the count for the next pair pass when done.
template <int COLL, bool B>
__global__ void __launch_bounds__(128)
k_slip_fix(DevParams p0, BatchView bv, SlipFix* __restrict__ fix, const int* __restrict__ owner,
           const int* __restrict__ nbrs, const int* __restrict__ in_pos, const double4* __restrict__ pos4,
           const double4* __restrict__ vel4, const double4* __restrict__ omg4, const uint8_t* __restrict__ phase,
           double* __restrict__ pft, uint8_t* __restrict__ pflag, Rec32* __restrict__ rec_own,
           Rec32* __restrict__ rec_in) {
  const unsigned n = min(fix->count, (unsigned)SLIP_FIX_CAP);
  for (unsigned t = threadIdx.x; t < n; t += blockDim.x) {
    const long long code = fix->pair[t];
    const long long cc = code >> 1;
    const int ll = owner[cc], i = nbrs[cc];
    const DevParams& p = sysp<B>(p0, bv, ll);
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
    const double4 va = vel4[ll], vb = vel4[i], wa = omg4[ll], wb = omg4[i];
    double* po = pft + 3 * cc;
    double pin[3] = {0.0, 0.0, 0.0};
    if (code & 1) { pin[0] = po[0]; pin[1] = po[1]; pin[2] = po[2]; }
    const int phl = p.nph > 1 ? phase[ll] : 0, phi = p.nph > 1 ? phase[i] : 0;
    double ot[3];
    PairTerms o;
    split_contact<COLL, true>(p, a, va, wa, phl, b, vb, wb, phi, dist, d2, r_lm * r_lm - d2, pin, ot, o);
    po[0] = ot[0]; po[1] = ot[1]; po[2] = ot[2];
    put_records(o, cc, in_pos, rec_own, rec_in);
    pflag[cc] = PF_CONTACT | ((ot[0] != 0.0 || ot[1] != 0.0 || ot[2] != 0.0) ? PF_HIST : 0);
  }
  __syncthreads();  // every thread has read the count
  if (threadIdx.x == 0) fix->count = 0;
}

// Contact bits (PF_CONTACT, bit 0 of each flag byte) of flags[base,
// base + cnt), cnt <= 32, as a mask: the bytes are read as aligned 32-bit
// words (the flag arrays carry 16 bytes of padding past their capacity).
__device__ __forceinline__ unsigned contact_mask(const uint8_t* __restrict__ flags, int base, int cnt) {
  static_assert(PF_CONTACT == 1, "contact bit is bit 0");
  unsigned mask = 0u;
  const int w0 = base & ~3;
  for (int w = w0; w < base + cnt; w += 4) {
    const uint32_t v = *reinterpret_cast<const uint32_t*>(flags + w) & 0x01010101u;
    const unsigned b4 = (v | (v >> 7) | (v >> 14) | (v >> 21)) & 0xFu;  // byte k -> bit k
    const int sh = w - base;
    mask |= sh >= 0 ? (b4 << sh) : (b4 >> -sh);
  }
  return cnt >= 32 ? mask : (mask & ((1u << cnt) - 1u));
}

// The records of one contiguous range [a, e) whose flag bytes say contact,
// a window of up to 32 at a time: the window's flags first, then the flagged
// records, each issued before the previous one is added.
__device__ __forceinline__ void add_range(int a, int e, const uint8_t* __restrict__ flags,
                                          const Rec32* __restrict__ rec, Comp3& F, Comp3& T, float& rs,
                                          float& rc) {
  for (int base = a; base < e; base += 32) {
    const int cnt = min(32, e - base);
    unsigned mask = contact_mask(flags, base, cnt);
    if (!mask) continue;
    Rec32 cur = rec[base + __ffs(mask) - 1];
    mask &= mask - 1u;
    while (true) {
      const bool more = mask != 0u;
      Rec32 nxt;
      if (more) {
        nxt = rec[base + __ffs(mask) - 1];
        mask &= mask - 1u;
      }
      F.add(0, cur.a.x); F.add(1, cur.a.y); F.add(2, cur.a.z);
      T.add(0, cur.b.x); T.add(1, cur.b.y); T.add(2, cur.b.z);
      const float x = cur.a.w, t = rs + x;
      if (fabsf(rs) >= fabsf(x)) rc += (rs - t) + x;
      else rc += (x - t) + rs;
      rs = t;
      if (!more) break;
      cur = nxt;
    }
  }
}

// Kernel 2 (per particle): wall terms (k_walls), the particle's incoming
// records (transpose order) and its own row's -- only for particles the
// pair kernel marked as in some contact --, compensated FP32 sums, the
// rolling-friction torque -MEW_R*(2R)*sum(KN*OVERLAP_N)*OMEGA/|OMEGA|, and
// the integration (MODE 1 Euler, 2 Adams-Bashforth) or FC/TOW (MODE 0).
template <int MODE, bool B>
__global__ void __launch_bounds__(256)
k_gather_split(DevParams p0, BatchView bv, const double4* __restrict__ pos_c, const double4* __restrict__ vel_c,
               const double4* __restrict__ omg_c, double4* __restrict__ pos_n, double4* __restrict__ vel_n,
               double4* __restrict__ omg_n, const int8_t* __restrict__ state, const double* __restrict__ wf,
               uint8_t* __restrict__ wall_hit, uint8_t* __restrict__ touched, const int* __restrict__ row_end,
               const int* __restrict__ in_start, const uint8_t* __restrict__ pflag, const uint8_t* __restrict__ in_flag,
               const Rec32* __restrict__ rec_own, const Rec32* __restrict__ rec_in, double* __restrict__ fc,
               double* __restrict__ tow, double* __restrict__ acc_old, double* __restrict__ rot_acc_old,
               unsigned* __restrict__ vslot, CellOut cells) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= p0.n) return;
  const DevParams& p = sysp<B>(p0, bv, me);
  const int8_t st = state[me];
  // the sums first, the particle's own state and wall terms after them (few
  // registers live across the record loops)
  Comp3 F, T;
  F.zero(); T.zero();
  float rs = 0.f, rc = 0.f;
  // a particle in no contact of this pass has no record to add
  const bool ph = touched[me] != 0, wh = wall_hit[me] != 0;
  if (ph) touched[me] = 0;
  // no torque and Euler: the spin stays (OMEGA_NEW = OMEGA_NEW + 0), so it
  // is neither read nor written (the spin array is updated in place)
  const bool keep_w = MODE == 1 && !wh && !ph;
  if (st != DEM_STATE_NONEXISTENT && ph) {
    add_range(in_start[me], in_start[me + 1], in_flag, rec_in, F, T, rs, rc);
    add_range(me ? row_end[me - 1] : 0, row_end[me], pflag, rec_own, F, T, rs, rc);
  }
  const double4 X = pos_c[me], V = vel_c[me], W = keep_w ? make_double4(0.0, 0.0, 0.0, 0.0) : omg_c[me];
  double f0[3] = {0.0, 0.0, 0.0}, t0[3] = {0.0, 0.0, 0.0};
  if (wh) {
    wall_hit[me] = 0;
    if (st == DEM_STATE_NORMAL) {
      const double* o = wf + 6 * (size_t)me;
      f0[0] = o[0]; f0[1] = o[1]; f0[2] = o[2]; t0[0] = o[3]; t0[1] = o[4]; t0[2] = o[5];
    }
  }
  double f[3], t[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) { f[c] = f0[c] + F.value(c); t[c] = t0[c] + T.value(c); }
  if (p.mew_r > 0.0) {
    const float w32[3] = {(float)W.x, (float)W.y, (float)W.z};
    const float om = sqrtf(w32[0] * w32[0] + w32[1] * w32[1] + w32[2] * w32[2]);
    if (om > 0.f) {
      const double sc = -(p.mew_r * (2.0 * X.w) * ((double)rs + (double)rc)) / (double)om;
#pragma unroll
      for (int c = 0; c < 3; ++c) t[c] += sc * (double)w32[c];
    }
  }
  const double x[3] = {X.x, X.y, X.z}, v[3] = {V.x, V.y, V.z}, w[3] = {W.x, W.y, W.z};
  finish_particle<MODE>(p, me, st, x, v, w, X.w, V.w, W.w, f, t, pos_n, vel_n, omg_n, fc, tow, acc_old,
                        rot_acc_old, vslot, cells, keep_w);
}

// The split records live in the handle's record array: the owner records
// in its first 32*cap bytes, the neighbour records in the next 32*cap (the
// array holds 80*cap bytes, the FP64 record size).
static Rec32* rec_own_of(dem_handle* h) { return reinterpret_cast<Rec32*>(h->prec); }
static Rec32* rec_in_of(dem_handle* h) { return reinterpret_cast<Rec32*>(h->prec) + h->pair_cap; }
static_assert(2 * sizeof(Rec32) <= sizeof(PairRec), "split records fit the record array");

template <int COLL, bool B>
static void launch_pairs_split_t(dem_handle* h) {
  const int c = h->cur;
  const int T = h->tune.pair_threads;
  k_pairs_split<COLL, B><<<(unsigned)(h->n_sm * h->tune.pair_bpsm), T, 0, h->stream>>>(
      h->dp, h->bview(), h->d_np, h->pair_cap, h->pair_owner, h->nbrs[h->rb], h->in_pos, h->pos4[c], h->vel4[c],
      h->omg4[c], h->state, h->phase, h->pft[h->pcur], h->pflag(), h->in_flag, h->touched, h->pgap, h->skin,
      rec_own_of(h), rec_in_of(h), h->slipfix, h->derr);
  DEM_LAUNCH(h);
  k_slip_fix<COLL, B><<<1, 128, 0, h->stream>>>(h->dp, h->bview(), h->slipfix, h->pair_owner, h->nbrs[h->rb],
                                                h->in_pos, h->pos4[c], h->vel4[c], h->omg4[c], h->phase,
                                                h->pft[h->pcur], h->pflag(), rec_own_of(h), rec_in_of(h));
  DEM_LAUNCH(h);
}

void launch_pairs_split(dem_handle* h) {
  const bool hz = h->dp.coll == DEM_COLL_HERTZ;
  if (h->batch()) hz ? launch_pairs_split_t<DEM_COLL_HERTZ, true>(h) : launch_pairs_split_t<DEM_COLL_LSD, true>(h);
  else hz ? launch_pairs_split_t<DEM_COLL_HERTZ, false>(h) : launch_pairs_split_t<DEM_COLL_LSD, false>(h);
}

template <int MODE, bool B>
static void launch_gather_split_t(dem_handle* h) {
  const int T = h->tune.gather_threads, G = (h->nl() + T - 1) / T;
  const int c = h->cur;
  k_gather_split<MODE, B><<<G, T, 0, h->stream>>>(
      h->dp, h->bview(), h->pos4[c], h->vel4[c], h->omg4[c], h->pos4[1 - c], h->vel4[1 - c], h->omg4[1 - c],
      h->state, h->wf, h->wall_hit, h->touched, h->row_end[h->rb], h->in_start, h->pflag(), h->in_flag,
      rec_own_of(h), rec_in_of(h), h->fc, h->tow, h->acc_old, h->rot_acc_old, h->vslot, gather_cells<MODE, B>(h));
  DEM_LAUNCH(h);
}

void launch_gather_split(dem_handle* h, int mode) {
  const bool bt = h->batch();
  if (mode == 0) bt ? launch_gather_split_t<0, true>(h) : launch_gather_split_t<0, false>(h);
  else if (mode == 1) bt ? launch_gather_split_t<1, true>(h) : launch_gather_split_t<1, false>(h);
  else bt ? launch_gather_split_t<2, true>(h) : launch_gather_split_t<2, false>(h);
}

}  // namespace demb
