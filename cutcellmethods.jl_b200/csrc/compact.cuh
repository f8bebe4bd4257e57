// compact.cuh -- in-order placement and block-sum scans for the surface extractors (mesh.cu,
// plic_mesh.cu).
//
// A surface pass visits every node or cell, but only a thin band (about one in a hundred at
// 512^3) contributes anything. The extractors test every item cheaply into a bitmap (one bit per
// item, 32 to a word), count the set bits per block, scan the block counts, and write the
// survivors in item order into flat lists; the long work (a clip, a tile, an edge walk) then runs
// over the lists one survivor per thread. This header holds the pieces those passes share: a
// block scan, round_prefix (the place of each word's set bits among a block's, in word order)
// and the block-sum scan.
#pragma once
#include <cstdint>

namespace cccompact {

// Exclusive scan of one value per thread over a block of MB threads; *total gets the sum.
template <int MB>
__device__ __forceinline__ unsigned long long block_scan(unsigned long long x, unsigned long long* total) {
  __shared__ unsigned long long warp_sum[MB / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned long long v = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) warp_sum[w] = v;
  __syncthreads();
  unsigned long long base = 0, all = 0;
  for (int q = 0; q < MB / 32; ++q) {
    if (q < w) base += warp_sum[q];
    all += warp_sum[q];
  }
  __syncthreads();
  *total = all;
  return base + v - x;
}

// ---- placing a block's set bits ----------------------------------------------------------------
// A block owns MB * IPT consecutive bitmap words, thread t taking word q*MB + t in round q, so
// block order is word order, and round_prefix places each word's set bits among the block's.

// Exclusive prefix, in block order (round, then thread), of one count per thread and round;
// pre[q] receives this thread's and the block total is returned. The counts are 64-bit so that
// several small counts packed in bit fields are placed by one call. Every thread of the block
// calls it; its shared slots are free again when it returns.
template <int MB, int IPT>
__device__ __forceinline__ unsigned long long round_prefix(const unsigned long long (&cnt)[IPT],
                                                           unsigned long long (&pre)[IPT]) {
  static_assert(IPT * (MB / 32) <= MB, "one (round, warp) slot per thread");
  constexpr int S = IPT * (MB / 32);
  __shared__ unsigned long long slot[S];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < IPT; ++q) {
    unsigned long long v = cnt[q];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    pre[q] = v - cnt[q];
    if (lane == 31) slot[q * (MB / 32) + w] = v;
  }
  __syncthreads();
  unsigned long long total;
  const unsigned long long first = block_scan<MB>(threadIdx.x < S ? slot[threadIdx.x] : 0ull, &total);
  if (threadIdx.x < S) slot[threadIdx.x] = first;  // block_scan's closing barrier ordered the reads
  __syncthreads();
#pragma unroll
  for (int q = 0; q < IPT; ++q) pre[q] += slot[q * (MB / 32) + w];
  __syncthreads();
  return total;
}

// In-place exclusive scan of `n` per-block counts (LANES interleaved series), one CTA of MB threads
// per series (launch LANES CTAs; series l = blockIdx.x), E * MB entries per pass taken round-major
// (entry base + e*MB + t in round e, so the loads coalesce and are all issued before the scan) and
// placed by round_prefix; totals[l] receives series l's sum.
template <int MB, int LANES, int E = 8>
__global__ void __launch_bounds__(MB) scan_series_kernel(unsigned long long* a, long long n, unsigned long long* totals) {
  const int l = blockIdx.x;
  unsigned long long carry = 0;  // the same in every thread
  for (long long base = 0; base < n; base += (long long)MB * E) {
    unsigned long long x[E], pre[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const long long q = base + (long long)e * MB + threadIdx.x;
      x[e] = q < n ? a[LANES * q + l] : 0ull;
    }
    const unsigned long long t = round_prefix<MB, E>(x, pre);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const long long q = base + (long long)e * MB + threadIdx.x;
      if (q < n) a[LANES * q + l] = carry + pre[e];
    }
    carry += t;
  }
  if (threadIdx.x == 0) totals[l] = carry;
}

}  // namespace cccompact
