// Device-wide exclusive prefix sum (three launches: block totals, scan of the totals in
// one block, per-block scan plus offset). Used for run offsets of the generator,
// radix-partition offsets and order-preserving compaction.
#pragma once
#include "common.cuh"
#include "engine.h"

namespace gpudb {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;                          // per thread
constexpr int kScanTile = kScanThreads * kScanItems;    // per block

// Inclusive scan of one value per thread across a block of kScanThreads threads.
template <class T> __device__ __forceinline__ T block_inclusive_scan(T v, T* warp_tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T o = __shfl_up_sync(FULL_MASK, v, d);
    if (lane >= d) v += o;
  }
  if (lane == 31) warp_tot[warp] = v;
  __syncthreads();
  if (warp == 0) {
    T w = lane < (kScanThreads / 32) ? warp_tot[lane] : T(0);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      T o = __shfl_up_sync(FULL_MASK, w, d);
      if (lane >= d) w += o;
    }
    if (lane < (kScanThreads / 32)) warp_tot[lane] = w;
  }
  __syncthreads();
  if (warp > 0) v += warp_tot[warp - 1];
  __syncthreads();
  return v;
}

template <class TI, class TO>
__global__ void __launch_bounds__(kScanThreads) scan_tile_totals(const TI* in, uint64_t n, TO* totals) {
  __shared__ TO wt[kScanThreads / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  TO s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    uint64_t r = base + (uint64_t)i * kScanThreads + threadIdx.x;
    if (r < n) s += (TO)in[r];
  }
  s = block_inclusive_scan<TO>(s, wt);
  if (threadIdx.x == kScanThreads - 1) totals[blockIdx.x] = s;
}

// Exclusive scan of `m` tile totals in place, by one block looping over the totals.
template <class TO>
__global__ void __launch_bounds__(kScanThreads) scan_totals(TO* totals, uint64_t m, TO* grand_total) {
  __shared__ TO wt[kScanThreads / 32];
  __shared__ TO carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint64_t b = 0; b < m; b += kScanThreads) {
    uint64_t i = b + threadIdx.x;
    TO v = i < m ? totals[i] : TO(0);
    TO inc = block_inclusive_scan<TO>(v, wt);
    TO c = carry;
    if (i < m) totals[i] = c + inc - v;
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) carry = c + inc;
    __syncthreads();
  }
  if (threadIdx.x == 0 && grand_total) *grand_total = carry;
}

template <class TI, class TO>
__global__ void __launch_bounds__(kScanThreads) scan_tiles(const TI* in, uint64_t n, const TO* offsets, TO* out) {
  __shared__ TO wt[kScanThreads / 32];
  // each thread owns kScanItems consecutive elements of the tile
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  TO v[kScanItems];
  TO s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    v[i] = (base + i < n) ? (TO)in[base + i] : TO(0);
    s += v[i];
  }
  TO inc = block_inclusive_scan<TO>(s, wt);
  TO run = offsets[blockIdx.x] + inc - s;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
}

// out[i] = sum(in[0..i)), grand_total (device, nullable) = sum(in). `tmp` needs
// tiles(n) elements of TO.
inline uint64_t scan_tiles_count(uint64_t n) { return (n + kScanTile - 1) / kScanTile; }

template <class TI, class TO>
int exclusive_scan(Call& call, const TI* in, uint64_t n, TO* out, TO* tmp, TO* grand_total) {
  uint64_t tiles = scan_tiles_count(n);
  if (tiles == 0) {
    if (grand_total) {
      cudaError_t e = cudaMemsetAsync(grand_total, 0, sizeof(TO), call.stream());
      if (e != cudaSuccess) return cuda_fail(call.ctx(), e, "scan memset");
    }
    return GPUDB_OK;
  }
  GPUDB_LAUNCH(call, (scan_tile_totals<TI, TO>), (unsigned)tiles, kScanThreads, 0, in, n, tmp);
  GPUDB_LAUNCH(call, (scan_totals<TO>), 1, kScanThreads, 0, tmp, tiles, grand_total);
  GPUDB_LAUNCH(call, (scan_tiles<TI, TO>), (unsigned)tiles, kScanThreads, 0, in, n, (const TO*)tmp, out);
  return GPUDB_OK;
}

}  // namespace gpudb
