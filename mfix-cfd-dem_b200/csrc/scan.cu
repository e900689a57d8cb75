// scan.cu -- exclusive prefix sum over int32 (cell counts, row counts).
//
// Three-phase scan: each block of 512 threads scans 2048 items (4 per
// thread, warp shuffles + one shared-memory pass), block totals are scanned
// recursively, then added back.  Deterministic (integer arithmetic).
#include "dem_internal.cuh"

namespace demb {

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__global__ void k_scan_tile(const int* __restrict__ in, int* __restrict__ out, int n,
                            int* __restrict__ block_sums) {
  __shared__ int warp_tot[SCAN_THREADS / 32];
  const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  int s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int idx = base + k;
    v[k] = idx < n ? in[idx] : 0;
    s += v[k];
  }
  // inclusive warp scan of per-thread sums
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int w = lane < SCAN_THREADS / 32 ? warp_tot[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < SCAN_THREADS / 32) warp_tot[lane] = wi - w;  // exclusive
    if (lane == SCAN_THREADS / 32 - 1 && block_sums) block_sums[blockIdx.x] = wi;
  }
  __syncthreads();
  int run = warp_tot[wid] + incl - s;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int idx = base + k;
    if (idx < n) out[idx] = run;
    run += v[k];
  }
}

__global__ void k_scan_add(int* __restrict__ out, int n, const int* __restrict__ block_off) {
  const int b = blockIdx.x;
  const int add = block_off[b];
  const int base = b * SCAN_TILE;
  for (int k = threadIdx.x; k < SCAN_TILE; k += blockDim.x) {
    int idx = base + k;
    if (idx < n) out[idx] += add;
  }
}

__global__ void k_scan_total(const int* __restrict__ in, const int* __restrict__ out, int n,
                             int* __restrict__ total) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *total = n > 0 ? out[n - 1] + in[n - 1] : 0;
}

static size_t scratch_need(int n) {
  size_t need = 0;
  long long m = n;
  while (m > SCAN_TILE) {
    m = (m + SCAN_TILE - 1) / SCAN_TILE;
    need += (size_t)m + 1;
  }
  return need + 1;
}

static int scan_rec(dem_handle* h, const int* in, int* out, int n, int* tmp) {
  int nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (nb <= 1) {
    k_scan_tile<<<1, SCAN_THREADS, 0, h->stream>>>(in, out, n, nullptr);
    DEM_LAUNCH(h);
    return 0;
  }
  int* sums = tmp;
  int* rest = tmp + nb + 1;
  k_scan_tile<<<nb, SCAN_THREADS, 0, h->stream>>>(in, out, n, sums);
  DEM_LAUNCH(h);
  // scan the block sums in place (safe: k_scan_tile reads all before writing
  // within one block, and a single tile covers the whole array here when
  // nb <= SCAN_TILE; larger arrays recurse with their own scratch)
  int rc = scan_rec(h, sums, sums, nb, rest);
  if (rc) return rc;
  k_scan_add<<<nb, 256, 0, h->stream>>>(out, n, sums);
  DEM_LAUNCH(h);
  return 0;
}

int exclusive_scan(dem_handle* h, const int* in, int* out, int n, int* d_total) {
  if (n <= 0) {
    if (d_total) check_cuda(h, cudaMemsetAsync(d_total, 0, sizeof(int), h->stream), "memset");
    return 0;
  }
  size_t need = scratch_need(n);
  if (need > h->scan_tmp_elems) {
    if (h->scan_tmp) cudaFree(h->scan_tmp);
    h->scan_tmp = nullptr;
    h->scan_tmp_elems = 0;
    if (int rc = check_cuda(h, cudaMalloc(&h->scan_tmp, need * sizeof(int)), "cudaMalloc scan")) return rc;
    h->scan_tmp_elems = need;
  }
  // when in == out the total must be read before the scan overwrites in[n-1]
  if (d_total && in == out) {
    int* last = h->scan_tmp + h->scan_tmp_elems - 1;
    if (int rc = check_cuda(h, cudaMemcpyAsync(last, in + n - 1, sizeof(int), cudaMemcpyDeviceToDevice, h->stream), "copy")) return rc;
    if (int rc = scan_rec(h, in, out, n, h->scan_tmp)) return rc;
    k_scan_total<<<1, 32, 0, h->stream>>>(last, out + n - 1, 1, d_total);
    DEM_LAUNCH(h);
    return check_cuda(h, cudaGetLastError(), "scan");
  }
  if (int rc = scan_rec(h, in, out, n, h->scan_tmp)) return rc;
  if (d_total) {
    k_scan_total<<<1, 32, 0, h->stream>>>(in, out, n, d_total);
    DEM_LAUNCH(h);
  }
  return check_cuda(h, cudaGetLastError(), "scan");
}

}  // namespace demb
