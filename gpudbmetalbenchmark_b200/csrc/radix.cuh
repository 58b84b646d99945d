// Stable hash-radix partitioning of (key, payload) rows.
// Reference: sf100_radix_histogram / sf100_radix_prefix_sum / sf100_radix_scatter
// (kernels/microbenchmarks.metal:15-99): one 1024-way pass, threadgroup histograms,
// a single-threadgroup Blelloch scan, and an atomic-cursor scatter (unstable, one 4-byte
// write per row anywhere in memory).
//
// B200 design: partition p = key_hash32(key) & (2^bits - 1) (the reference's hash), in
// LSD passes of at most 8 bits, so the fan-out of a pass (256) fits the per-block counters
// and staging buffer in shared memory. Per pass:
//   radix_hist_kernel   per-tile bucket counts (shared atomics), bucket-major [b][tile];
//   exclusive_scan      over that array: global start of every (bucket, tile) piece;
//   radix_scatter_kernel ranks the tile's rows inside their bucket in input order
//                        (__match_any_sync per warp + per-bucket warp prefix in shared
//                        memory), stages the tile bucket-sorted in shared memory, then
//                        writes each bucket's run contiguously (coalesced stores).
// Passes are stable, so after the last pass rows are ordered by p with input order kept
// inside each partition. Row counts may live on the device (n_dev): grids are sized from
// a host upper bound and tiles past the device count do no work.
#pragma once
#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"
#include "scan.cuh"

namespace gpudb {

constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 16;
constexpr int kRadixTile = kRadixThreads * kRadixItems;   // 4096 rows per block
constexpr int kRadixPassBits = 8;                          // fan-out 256 per pass

__device__ __forceinline__ uint32_t radix_digit(int32_t key, int shift, uint32_t dmask) {
  return (key_hash32(key) >> shift) & dmask;
}

__device__ __forceinline__ uint64_t radix_rows(uint64_t n_max, const uint32_t* n_dev) {
  return n_dev ? (uint64_t)*n_dev : n_max;
}

static __global__ void __launch_bounds__(kRadixThreads) radix_hist_kernel(const int32_t* __restrict__ keys, uint64_t n_max,
                                                                          const uint32_t* n_dev, int shift, int dbits,
                                                                          uint32_t tiles, uint32_t* hist) {
  __shared__ uint32_t cnt[1 << kRadixPassBits];
  const uint32_t buckets = 1u << dbits, dmask = buckets - 1;
  for (uint32_t b = threadIdx.x; b < buckets; b += kRadixThreads) cnt[b] = 0;
  __syncthreads();
  const uint64_t n = radix_rows(n_max, n_dev);
  const uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
#pragma unroll 4
  for (int j = 0; j < kRadixItems; j++) {
    const uint64_t r = base + (uint64_t)j * kRadixThreads + threadIdx.x;
    if (r < n) atomicAdd(&cnt[radix_digit(keys[r], shift, dmask)], 1u);
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < buckets; b += kRadixThreads) hist[(size_t)b * tiles + blockIdx.x] = cnt[b];
}

// offsets: exclusive scan of hist (bucket-major) with the grand total at [buckets*tiles].
template <class P>
__global__ void __launch_bounds__(kRadixThreads) radix_scatter_kernel(const int32_t* __restrict__ keys_in,
                                                                      const P* __restrict__ pay_in, uint64_t n_max,
                                                                      const uint32_t* n_dev, int shift, int dbits,
                                                                      uint32_t tiles, const uint32_t* __restrict__ offsets,
                                                                      int32_t* __restrict__ keys_out, P* __restrict__ pay_out) {
  extern __shared__ unsigned long long radix_smem[];
  P* spay = reinterpret_cast<P*>(radix_smem);                          // kRadixTile
  int32_t* skey = reinterpret_cast<int32_t*>(spay + kRadixTile);       // kRadixTile
  __shared__ uint32_t tstart[1 << kRadixPassBits];
  __shared__ uint32_t run[1 << kRadixPassBits];
  __shared__ uint32_t wcnt[kRadixThreads / 32][1 << kRadixPassBits];
  __shared__ uint32_t wt[kRadixThreads / 32];
  const uint32_t buckets = 1u << dbits, dmask = buckets - 1;
  const uint64_t n = radix_rows(n_max, n_dev);
  const uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
  if (base >= n) return;   // uniform across the block
  const uint32_t tile_n = (uint32_t)((n - base) < (uint64_t)kRadixTile ? (n - base) : (uint64_t)kRadixTile);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // this tile's bucket counts -> exclusive prefix (one bucket per thread; buckets <= 256)
  {
    uint32_t c = 0;
    const uint32_t b = threadIdx.x;
    if (b < buckets) {
      const size_t i = (size_t)b * tiles + blockIdx.x;
      c = offsets[i + 1] - offsets[i];
    }
    const uint32_t inc = block_inclusive_scan<uint32_t>(c, wt);
    if (b < buckets) { tstart[b] = inc - c; run[b] = 0; }
  }
  __syncthreads();
  for (int j = 0; j < kRadixItems; j++) {
    for (int i = threadIdx.x; i < (kRadixThreads / 32) * (1 << kRadixPassBits); i += kRadixThreads)
      (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint32_t rr = (uint32_t)j * kRadixThreads + threadIdx.x;
    const bool valid = rr < tile_n;
    const uint64_t r = base + rr;
    const int32_t key = valid ? keys_in[r] : 0;
    const uint32_t d = valid ? radix_digit(key, shift, dmask) : (0x10000u + lane);
    const uint32_t peers = __match_any_sync(FULL_MASK, d);
    const uint32_t rank = __popc(peers & lanemask_lt());
    if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (threadIdx.x < buckets) {
      uint32_t s = run[threadIdx.x];
#pragma unroll
      for (int w = 0; w < kRadixThreads / 32; w++) {
        const uint32_t c = wcnt[w][threadIdx.x];
        wcnt[w][threadIdx.x] = s;
        s += c;
      }
      run[threadIdx.x] = s;
    }
    __syncthreads();
    if (valid) {
      const uint32_t lp = tstart[d] + wcnt[warp][d] + rank;
      skey[lp] = key;
      spay[lp] = pay_in ? pay_in[r] : (P)r;
    }
    __syncthreads();
  }
  for (uint32_t i = threadIdx.x; i < tile_n; i += kRadixThreads) {
    const int32_t k = skey[i];
    const uint32_t b = radix_digit(k, shift, dmask);
    const uint32_t o = offsets[(size_t)b * tiles + blockIdx.x] + (i - tstart[b]);
    keys_out[o] = k;
    pay_out[o] = spay[i];
  }
}

// Full-width partition histogram (2^bits counters): shared counters up to 4096 partitions,
// global atomics beyond.
static __global__ void __launch_bounds__(kRadixThreads) part_hist_kernel(const int32_t* __restrict__ keys, uint64_t n_max,
                                                                         const uint32_t* n_dev, int bits, uint32_t* hist) {
  __shared__ uint32_t cnt[4096];
  const uint32_t parts = 1u << bits, pmask = parts - 1;
  const bool local = parts <= 4096;
  if (local) {
    for (uint32_t i = threadIdx.x; i < parts; i += kRadixThreads) cnt[i] = 0;
    __syncthreads();
  }
  const uint64_t n = radix_rows(n_max, n_dev);
  const uint64_t stride = (uint64_t)gridDim.x * kRadixThreads;
  for (uint64_t r = (uint64_t)blockIdx.x * kRadixThreads + threadIdx.x; r < n; r += stride) {
    const uint32_t p = key_hash32(keys[r]) & pmask;
    if (local) atomicAdd(&cnt[p], 1u);
    else atomicAdd(&hist[p], 1u);
  }
  if (local) {
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < parts; i += kRadixThreads)
      if (cnt[i]) atomicAdd(&hist[i], cnt[i]);
  }
}

// Partitions rows [0, n) (n = *n_dev when given, else n_max) into 2^bits partitions.
// pay == nullptr partitions the row ids. keys_tmp/pay_tmp: n_max elements for the first
// of two passes. offsets: 2^bits + 1 entries (partition starts, total last).
template <class P>
int radix_partition_run(Call& call, const int32_t* keys, const P* pay, uint64_t n_max, const uint32_t* n_dev, int bits,
                        int32_t* keys_out, P* pay_out, uint32_t* offsets, int32_t* keys_tmp, P* pay_tmp) {
  gpudb_ctx* ctx = call.ctx();
  cudaStream_t s = call.stream();
  const uint64_t tiles = std::max<uint64_t>(1, (n_max + kRadixTile - 1) / kRadixTile);
  const int passes = bits <= kRadixPassBits ? 1 : 2;
  const int lo_bits = passes == 1 ? bits : bits - kRadixPassBits;
  const uint32_t parts = 1u << bits;
  // hist [256 x tiles] + total, its scan, scan scratch, full histogram
  const size_t hist_n = (size_t)(1u << kRadixPassBits) * tiles + 1;
  // the scan scratch serves both the per-pass histogram scan and the partition scan
  const size_t stmp_n = std::max<size_t>(scan_tiles_count(hist_n), scan_tiles_count(parts)) + 8;
  void* sc = nullptr;
  int rc = scratch(ctx, "radix.hist", (hist_n * 2 + stmp_n + parts + 1) * sizeof(uint32_t), &sc);
  if (rc) return rc;
  uint32_t* hist = static_cast<uint32_t*>(sc);
  uint32_t* offs = hist + hist_n;
  uint32_t* stmp = offs + hist_n;
  uint32_t* phist = stmp + stmp_n;
  const size_t smem = (size_t)kRadixTile * (sizeof(P) + sizeof(int32_t));
  GPUDB_CUDA(ctx, cudaFuncSetAttribute(radix_scatter_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int pass = 0; pass < passes; pass++) {
    const int shift = pass == 0 ? 0 : lo_bits;
    const int dbits = pass == 0 ? lo_bits : kRadixPassBits;
    const int32_t* kin = pass == 0 ? keys : keys_tmp;
    const P* pin = pass == 0 ? pay : pay_tmp;
    int32_t* kout = (pass == passes - 1) ? keys_out : keys_tmp;
    P* pout = (pass == passes - 1) ? pay_out : pay_tmp;
    const size_t hn = (size_t)(1u << dbits) * tiles;
    GPUDB_LAUNCH(call, radix_hist_kernel, (unsigned)tiles, kRadixThreads, 0, kin, n_max, n_dev, shift, dbits,
                 (uint32_t)tiles, hist);
    rc = exclusive_scan<uint32_t, uint32_t>(call, hist, hn, offs, stmp, offs + hn);
    if (rc) return rc;
    GPUDB_LAUNCH(call, radix_scatter_kernel<P>, (unsigned)tiles, kRadixThreads, smem, kin, pin, n_max, n_dev, shift, dbits,
                 (uint32_t)tiles, (const uint32_t*)offs, kout, pout);
  }
  GPUDB_CUDA(ctx, cudaMemsetAsync(phist, 0, (size_t)parts * 4, s));
  const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n_max + kRadixThreads - 1) / kRadixThreads,
                                                                       (uint64_t)ctx->sm_count * 8));
  GPUDB_LAUNCH(call, part_hist_kernel, g, kRadixThreads, 0, keys, n_max, n_dev, bits, phist);
  return exclusive_scan<uint32_t, uint32_t>(call, phist, parts, offsets, stmp, offsets + parts);
}

// Partition bits so that the average partition holds about `per_part` rows.
inline int radix_bits_for(uint64_t n, uint64_t per_part) {
  int b = 0;
  while (b < kRadixMaxBits && (n >> b) > per_part) b++;
  return b;
}

}  // namespace gpudb
