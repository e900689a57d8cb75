// tune.cu -- launch-shape autotuner of the hot kernels.
//
// No counterpart in the reference.  The pair kernel (threads per block and
// resident blocks per SM of its persistent grid), the gather kernel
// (threads per block) and the count pass of the pair build (threads per
// block) are timed with CUDA events on the handle's stream, on the handle's
// own current state, and the fastest shape of each is kept.  The pair
// history and its flags, which the pair kernel updates in place, are saved
// before and restored after the timing; everything else the timed launches
// write is scratch that the next step rewrites (contact records, FC/TOW, row
// counts), so tuning does not change any result.  The launch shape does not
// change the arithmetic, so results are also the same under every shape.
#include "dem_internal.cuh"

#include <cfloat>
#include <cstring>

using namespace demb;

namespace demb {

template <class F>
static float time_launches(dem_handle* h, int reps, F&& launch) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  launch();  // warm-up
  cudaEventRecord(a, h->stream);
  for (int r = 0; r < reps; ++r) launch();
  cudaEventRecord(b, h->stream);
  float ms = FLT_MAX;
  if (cudaEventSynchronize(b) == cudaSuccess) {
    cudaEventElapsedTime(&ms, a, b);
    ms /= (float)reps;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms;
}

static void fill_out(const dem_handle* h, dem_tuning* o, double pms, double gms, double nms) {
  memset(o, 0, sizeof *o);
  o->pair_threads = h->tune.pair_threads;
  o->pair_blocks_per_sm = h->tune.pair_bpsm;
  o->gather_threads = h->tune.gather_threads;
  o->neigh_threads = h->tune.neigh_threads;
  o->pair_ms = pms;
  o->gather_ms = gms;
  o->neigh_ms = nms;
}

}  // namespace demb

extern "C" {

int dem_autotune(dem_handle* h, int32_t reps, dem_tuning* out) {
  if (!h) return DEM_ERR_ARG;
  cudaSetDevice(h->dev);
  if (reps < 1) return set_err(h, DEM_ERR_ARG, "reps must be positive");
  if (!h->have_state || !h->have_pairs) return set_err(h, DEM_ERR_STATE, "state or pair list missing");
  invalidate_graphs(h);
  const size_t P = (size_t)host_pairs(h);
  char* snap = (char*)stage_buffer(h, sizeof(double) * 3 * P + 2 * P + 64);
  if (!snap) return set_err(h, DEM_ERR_CUDA, "cudaMalloc stage");
  if (P) {
    cudaMemcpyAsync(snap, h->pft[h->pcur], sizeof(double) * 3 * P, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(snap + sizeof(double) * 3 * P, h->pflag(), P, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(snap + sizeof(double) * 3 * P + P, h->in_flag, P, cudaMemcpyDeviceToDevice, h->stream);
  }
  const int threads[3] = {64, 128, 256};
  const int bpsm[4] = {2, 4, 8, 16};
  float best_p = FLT_MAX, best_g = FLT_MAX, best_n = FLT_MAX;
  dem_handle::Tune t = h->tune, best = h->tune;
  for (int T : threads)
    for (int b : bpsm) {
      h->tune.pair_threads = T;
      h->tune.pair_bpsm = b;
      const float ms = time_launches(h, reps, [&] { launch_pairs_only(h); });
      if (ms < best_p) { best_p = ms; best.pair_threads = T; best.pair_bpsm = b; }
    }
  // the gather reads the contact marks the pair kernel sets, so each timed
  // gather runs behind a pair launch (at the best pair shape)
  h->tune = t;
  h->tune.pair_threads = best.pair_threads;
  h->tune.pair_bpsm = best.pair_bpsm;
  for (int T : threads) {
    h->tune.gather_threads = T;
    const float ms = time_launches(h, reps, [&] { launch_pairs_only(h); launch_gather_only(h); });
    if (ms - best_p < best_g) { best_g = ms - best_p; best.gather_threads = T; }
  }
  h->tune = t;
  const int nthreads[3] = {32, 64, 128};
  for (int T : nthreads) {
    h->tune.neigh_threads = T;
    const float ms = time_launches(h, reps, [&] { launch_neigh_count(h); });
    if (ms < best_n) { best_n = ms; best.neigh_threads = T; }
  }
  h->tune = best;
  if (P) {
    cudaMemcpyAsync(h->pft[h->pcur], snap, sizeof(double) * 3 * P, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->pflag(), snap + sizeof(double) * 3 * P, P, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->in_flag, snap + sizeof(double) * 3 * P + P, P, cudaMemcpyDeviceToDevice, h->stream);
  }
  // the timed pair launches added to the contact counters
  cudaMemsetAsync(&h->derr->n_contacts, 0, 2 * sizeof(unsigned long long), h->stream);
  if (int rc = check_cuda(h, cudaStreamSynchronize(h->stream), "autotune")) return rc;
  if (out) fill_out(h, out, best_p, best_g, best_n);
  return 0;
}

int dem_get_tuning(dem_handle* h, dem_tuning* out) {
  if (!h || !out) return DEM_ERR_ARG;
  fill_out(h, out, 0.0, 0.0, 0.0);
  return 0;
}

int dem_set_tuning(dem_handle* h, const dem_tuning* in) {
  if (!h || !in) return DEM_ERR_ARG;
  cudaSetDevice(h->dev);
  auto ok = [](int v, int lo, int hi) { return v >= lo && v <= hi && (v % 32) == 0; };
  if (!ok(in->pair_threads, 32, 256) || !ok(in->gather_threads, 32, 256) || !ok(in->neigh_threads, 32, 128) ||
      in->pair_blocks_per_sm < 1 || in->pair_blocks_per_sm > 64)
    return set_err(h, DEM_ERR_ARG, "launch shape out of range");
  h->tune.pair_threads = in->pair_threads;
  h->tune.pair_bpsm = in->pair_blocks_per_sm;
  h->tune.gather_threads = in->gather_threads;
  h->tune.neigh_threads = in->neigh_threads;
  invalidate_graphs(h);
  return 0;
}

}  // extern "C"
