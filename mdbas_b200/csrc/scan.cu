// scan.cu -- device-wide exclusive prefix sums (list offsets, cell starts).
//
// Three-phase tile scan: each 1024-thread block scans a tile of 4096 values
// in shared memory and writes the tile total; tile totals are scanned by the
// same kernel (recursively); a last pass adds each tile's base.  Used on
// arrays of cells, atoms or clusters (<= a few million entries), where it is
// launch-bound, so the simple form is enough.
#include "common.cuh"

namespace mdbas {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kTile = kScanThreads * kScanItems;

template <class TIn, class TOut>
__global__ void __launch_bounds__(kScanThreads)
k_scan_tiles(const TIn *__restrict__ in, TOut *__restrict__ out, long long *__restrict__ tile_sum,
             int n) {
  __shared__ long long warp_tot[kScanThreads / 32];
  const long long base = (long long)blockIdx.x * kTile;
  long long v[kScanItems];
  long long run = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    long long idx = base + (long long)threadIdx.x * kScanItems + k;
    v[k] = (idx < n) ? (long long)in[idx] : 0;
    run += v[k];
  }
  // inclusive scan of per-thread totals across the block
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  long long x = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    long long t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  long long excl = x - run + (warp > 0 ? warp_tot[warp - 1] : 0);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    long long idx = base + (long long)threadIdx.x * kScanItems + k;
    if (idx < n) out[idx] = (TOut)excl;
    excl += v[k];
  }
  if (threadIdx.x == kScanThreads - 1) tile_sum[blockIdx.x] = excl;
}

template <class TOut>
__global__ void k_scan_add(TOut *__restrict__ out, const long long *__restrict__ tile_base, int n) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < n) out[idx] = (TOut)((long long)out[idx] + tile_base[idx / kTile]);
}

template <class TOut>
__global__ void k_scan_total(TOut *out, const int *in, int n) {
  // out[n] = out[n-1] + in[n-1]
  if (n > 0) out[n] = (TOut)((long long)out[n - 1] + (long long)in[n - 1]);
  else out[0] = 0;
}

// Scan of the tile sums level by level; tmp layout: levels of long long.
int scan_ll(long long *data, int n, long long *tmp, cudaStream_t s) {
  // data (length n) -> exclusive scan in place
  int tiles = (n + kTile - 1) / kTile;
  long long *sums = tmp;
  MDB_LAUNCH((k_scan_tiles<long long, long long>), tiles, kScanThreads, 0, s, data, data, sums,
             n);
  if (tiles > 1) {
    MDB_TRY(scan_ll(sums, tiles, tmp + tiles, s));
    MDB_LAUNCH(k_scan_add<long long>, grid_for(n, 256), 256, 0, s, data, sums, n);
  }
  return MDBAS_NB_OK;
}

template <class TOut>
int scan_impl(const int *in, TOut *out, int n, void *tmpv, cudaStream_t s) {
  long long *tmp = static_cast<long long *>(tmpv);
  if (n <= 0) {
    MDB_LAUNCH(k_scan_total<TOut>, 1, 1, 0, s, out, in, 0);
    return MDBAS_NB_OK;
  }
  int tiles = (n + kTile - 1) / kTile;
  long long *sums = tmp;
  MDB_LAUNCH((k_scan_tiles<int, TOut>), tiles, kScanThreads, 0, s, in, out, sums, n);
  if (tiles > 1) {
    MDB_TRY(scan_ll(sums, tiles, tmp + tiles, s));
    MDB_LAUNCH(k_scan_add<TOut>, grid_for(n, 256), 256, 0, s, out, sums, n);
  }
  MDB_LAUNCH(k_scan_total<TOut>, 1, 1, 0, s, out, in, n);
  return MDBAS_NB_OK;
}

}  // namespace

size_t scan_tmp_bytes(int n) {
  size_t total = 0;
  long long m = n;
  do {
    m = (m + kTile - 1) / kTile;
    total += (size_t)m;
  } while (m > 1);
  return (total + 4) * sizeof(long long);
}

int exclusive_scan(const int *in, long long *out, int n, void *tmp, cudaStream_t s) {
  return scan_impl<long long>(in, out, n, tmp, s);
}

int exclusive_scan32(const int *in, int *out, int n, void *tmp, cudaStream_t s) {
  return scan_impl<int>(in, out, n, tmp, s);
}

}  // namespace mdbas
