// Exclusive prefix sum of 64-bit counts on the device (the row starts of a compaction and of the
// mosp combined graph's out-rows): three launches on the caller's stream.
//   1. k_scan_tiles: each block scans a tile of kScanTile values (kScanItems per thread, the
//      threads' sums scanned through warp shuffles and one shared-memory pass over the warps) and
//      writes the tile's total;
//   2. k_scan_totals: one block scans the tile totals in place, kScanTile at a time with a carry;
//   3. k_scan_add: every value gets its tile's offset.
// Scratch: scan_scratch(n) values.
#pragma once

#include "internal.hpp"

namespace dyngb200 {

constexpr int kScanBlock = 512;
constexpr int kScanItems = 8;
constexpr long long kScanTile = static_cast<long long>(kScanBlock) * kScanItems;

inline long long scan_scratch(long long n) { return (n + kScanTile - 1) / kScanTile + 1; }

// Exclusive scan of one value per thread across the block; *total receives the block's sum.
__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* total) {
  __shared__ long long s_warp[kScanBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  long long incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    long long w = lane < (kScanBlock / 32) ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < (kScanBlock / 32)) s_warp[lane] = w;  // inclusive totals of the warps
  }
  __syncthreads();
  const long long before = warp > 0 ? s_warp[warp - 1] : 0;
  *total = s_warp[kScanBlock / 32 - 1];
  __syncthreads();  // s_warp is reused by the next call
  return before + incl - v;
}

static __global__ void __launch_bounds__(kScanBlock) k_scan_tiles(const long long* in, long long* out,
                                                           long long n, long long* tile_sum) {
  const long long base = blockIdx.x * kScanTile + static_cast<long long>(threadIdx.x) * kScanItems;
  long long x[kScanItems];
  long long sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    x[i] = base + i < n ? in[base + i] : 0;
    sum += x[i];
  }
  long long total = 0;
  long long run = block_exclusive_scan(sum, &total);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = run;
    run += x[i];
  }
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

static __global__ void __launch_bounds__(kScanBlock) k_scan_totals(long long* tile_sum, long long tiles) {
  __shared__ long long s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (long long b = 0; b < tiles; b += kScanTile) {
    const long long base = b + static_cast<long long>(threadIdx.x) * kScanItems;
    long long x[kScanItems];
    long long sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      x[i] = base + i < tiles ? tile_sum[base + i] : 0;
      sum += x[i];
    }
    long long total = 0;
    long long run = s_carry + block_exclusive_scan(sum, &total);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      if (base + i < tiles) tile_sum[base + i] = run;
      run += x[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) s_carry += total;
    __syncthreads();
  }
}

static __global__ void __launch_bounds__(kScanBlock) k_scan_add(long long* out, long long n,
                                                         const long long* tile_offset) {
  const long long base = blockIdx.x * kScanTile + static_cast<long long>(threadIdx.x) * kScanItems;
  const long long off = tile_offset[blockIdx.x];
  if (off == 0) return;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) out[base + i] += off;
}

// out[i] = in[0] + ... + in[i - 1] for i < n (in and out distinct); scratch holds
// scan_scratch(n) values.  Returns the number of kernel launches queued.
inline int exclusive_scan(const long long* in, long long* out, long long n, long long* scratch,
                          cudaStream_t s) {
  if (n <= 0) return 0;
  const long long tiles = (n + kScanTile - 1) / kScanTile;
  k_scan_tiles<<<static_cast<unsigned>(tiles), kScanBlock, 0, s>>>(in, out, n, scratch);
  k_scan_totals<<<1, kScanBlock, 0, s>>>(scratch, tiles);
  k_scan_add<<<static_cast<unsigned>(tiles), kScanBlock, 0, s>>>(out, n, scratch);
  DYNGB200_CUDA(cudaGetLastError());
  return 3;
}

}  // namespace dyngb200
