// Stable hash-radix partitioning of (key, payload) rows.
// Reference: sf100_radix_histogram / sf100_radix_prefix_sum / sf100_radix_scatter
// (kernels/microbenchmarks.metal:15-99): one 1024-way pass, threadgroup histograms,
// a single-threadgroup Blelloch scan, and an atomic-cursor scatter (unstable, one 4-byte
// write per row anywhere in memory).
//
// B200 design. Partition p = key_hash32(key) & (2^bits - 1) (the reference's hash), in LSD
// passes of at most kRxPassBits bits (one pass up to 1024 partitions). The input is cut into
// G super-tiles, as many as the scatter kernel's blocks that fit on the GPU at once, sized
// on the device from the row count; per pass:
//   rx_hist_kernel    counts each super-tile's rows per digit (shared-memory atomics; four
//                     blocks per super-tile, so every SM streams) into hist[digit][G], and
//                     in the first pass also the rows per final partition;
//   exclusive_scan    over hist (digit-major): where each (digit, super-tile) run starts;
//   rx_scatter_kernel one block per super-tile walks its sub-tiles (8192 rows by default) in
//                     order, the next two in flight as bulk copies (TMA) into a shared-memory
//                     ring. Each warp ranks its own contiguous rows by digit (__match_any_sync
//                     and per-warp counters, no atomics), one block-wide scan turns the
//                     (digit, warp) counts into staged positions, the sub-tile is staged
//                     digit-sorted in shared memory and written out run by run from
//                     per-digit cursors that carry across the super-tile's sub-tiles.
// The order inside a partition is the input order (stable), so later passes and the final
// result are deterministic. The row source is a template: plain columns (payload = row id
// when none is given) or a pipeline's filtered fact rows (Q3), so a filter and the first
// pass share one read of the columns.
#pragma once
#include <algorithm>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"
#include "scan.cuh"
#include "tma.cuh"

namespace gpudb {

constexpr int kRxThreads = 512;                         // histogram blocks
constexpr int kRxPassBits = 10;                         // fan-out of one pass <= 1024
constexpr uint32_t kRxMaxF = 1u << kRxPassBits;
constexpr int kRxFullSmemBits = 13;                     // final-partition counts in shared memory up to 8192
constexpr int kRxHistSplit = 4;                         // histogram blocks per super-tile

// Plain columns: keys, and a payload column or (null) the row number. Rows [0, n) with
// n = *n_dev when given (a count left on the device by an earlier kernel), capped at n_max.
// Whole sub-tiles can also come through the scatter's bulk-copy ring: stage_bytes() per
// sub-tile (keys, then payloads), issue() posts the copies, staged() reads one row back.
template <class P>
struct ColumnSource {
  const int32_t* keys;
  const P* pay;
  uint64_t n_max;
  const uint32_t* n_dev;
  __device__ __forceinline__ uint64_t rows() const {
    return n_dev ? min((uint64_t)*n_dev, n_max) : n_max;
  }
  __device__ __forceinline__ bool key(uint64_t r, int32_t& k) const {
    k = __ldg(keys + r);   // cached: the scatter pass reads the keys again
    return true;
  }
  __device__ __forceinline__ P payload(uint64_t r) const { return pay ? __ldcs(pay + r) : (P)r; }
  template <bool PAY>
  __host__ __device__ static constexpr uint32_t stage_bytes(uint32_t tile) { return tile * (4u + (PAY ? (uint32_t)sizeof(P) : 0u)); }
  // both columns start on 16 bytes, so every whole sub-tile does (sub-tiles start at
  // multiples of their row count, a multiple of 4)
  __device__ __forceinline__ bool bulk_ok() const {
    return ((uintptr_t)keys & 15u) == 0 && ((uintptr_t)pay & 15u) == 0;
  }
  template <bool PAY, uint32_t TILE>
  __device__ __forceinline__ void issue(uint64_t r0, unsigned char* st, uint64_t* bar) const {
    const bool pc = PAY && pay != nullptr;
    mbar_arrive_expect_tx(bar, TILE * 4u + (pc ? TILE * (uint32_t)sizeof(P) : 0u));
    bulk_copy_g2s(st, keys + r0, TILE * 4u, bar);
    if (pc) bulk_copy_g2s(st + TILE * 4u, pay + r0, TILE * (uint32_t)sizeof(P), bar);
  }
  template <bool PAY, uint32_t TILE>
  __device__ __forceinline__ bool staged(const unsigned char* st, uint32_t i, uint64_t r, int32_t& k, P& p) const {
    k = reinterpret_cast<const int32_t*>(st)[i];
    if (PAY) p = pay ? reinterpret_cast<const P*>(st + TILE * 4u)[i] : (P)r;
    return true;
  }
};

// Rows per super-tile for n rows over G super-tiles: whole sub-tiles of `tile` rows, at least
// one. Both kernels of a pass derive it from the same device row count, so a count that an
// earlier kernel left on the device (a filtered input) still spreads over all G blocks.
__host__ __device__ __forceinline__ uint64_t rx_super_rows_for(uint64_t n, uint32_t G, uint32_t tile) {
  const uint64_t per = (n + G - 1) / (G ? G : 1);
  const uint64_t s = (per + tile - 1) / tile * tile;
  return s < (uint64_t)tile ? (uint64_t)tile : s;
}

__device__ __forceinline__ uint32_t rx_digit(int32_t key, int shift, uint32_t mask) {
  return (key_hash32(key) >> shift) & mask;
}

// Inclusive scan of one value per thread across a block of NT threads.
template <int NT>
__device__ __forceinline__ uint32_t rx_block_scan(uint32_t v, uint32_t* warp_tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(FULL_MASK, v, d);
    if (lane >= d) v += o;
  }
  if (lane == 31) warp_tot[warp] = v;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < NT / 32 ? warp_tot[lane] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(FULL_MASK, w, d);
      if (lane >= d) w += o;
    }
    if (lane < NT / 32) warp_tot[lane] = w;
  }
  __syncthreads();
  if (warp > 0) v += warp_tot[warp - 1];
  __syncthreads();
  return v;
}

// Digit counts of super-tile blockIdx.x / kRxHistSplit (one quarter of it per block) into
// hist[digit * G + super-tile] (zeroed), and with `full` the rows per final partition
// (fbits bits; zeroed).
template <class Src>
__global__ void __launch_bounds__(kRxThreads) rx_hist_kernel(Src src, uint32_t G, uint32_t tile, int shift, int dbits,
                                                             int fbits, uint32_t* __restrict__ hist,
                                                             uint32_t* __restrict__ full) {
  __shared__ uint32_t cnt[kRxMaxF];
  __shared__ uint32_t fcnt[1u << kRxFullSmemBits];
  const uint32_t F = 1u << dbits, dmask = F - 1, fmask = (1u << fbits) - 1;
  const bool fs = full && fbits <= kRxFullSmemBits;
  for (uint32_t i = threadIdx.x; i < F; i += kRxThreads) cnt[i] = 0;
  if (fs)
    for (uint32_t i = threadIdx.x; i <= fmask; i += kRxThreads) fcnt[i] = 0;
  __syncthreads();
  const uint32_t g = blockIdx.x / kRxHistSplit, part = blockIdx.x % kRxHistSplit;
  const uint64_t n = src.rows();
  const uint64_t super_rows = rx_super_rows_for(n, G, tile);
  const uint64_t quarter = super_rows / kRxHistSplit;
  const uint64_t r0 = (uint64_t)g * super_rows + part * quarter;
  const uint64_t r1 = min(r0 + quarter, n);
  constexpr int U = 8;
  for (uint64_t r = r0 + threadIdx.x; r < r1; r += (uint64_t)U * kRxThreads) {
    int32_t k[U];
    bool v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint64_t rr = r + (uint64_t)u * kRxThreads;
      v[u] = rr < r1 && src.key(rr, k[u]);
    }
#pragma unroll
    for (int u = 0; u < U; u++)
      if (v[u]) {
        const uint32_t h = key_hash32(k[u]);
        atomicAdd(&cnt[(h >> shift) & dmask], 1u);
        if (fs) atomicAdd(&fcnt[h & fmask], 1u);
        else if (full) atomicAdd(&full[h & fmask], 1u);
      }
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < F; b += kRxThreads)
    if (cnt[b]) atomicAdd(&hist[(size_t)b * G + g], cnt[b]);
  if (fs)
    for (uint32_t i = threadIdx.x; i <= fmask; i += kRxThreads)
      if (fcnt[i]) atomicAdd(&full[i], fcnt[i]);
}

// Shared memory of one scatter block: STG staged input sub-tiles (the bulk-copy ring), the
// digit-sorted staging of one sub-tile, the digit counters (stable: per warp, u16; unstable:
// per block and the digit starts, u32) and the per-digit output cursors.
template <class Src, class P, bool PAY, int T, int I, int STG, bool STABLE>
__host__ __device__ constexpr size_t rx_scatter_smem(uint32_t F) {
  return (size_t)STG * Src::template stage_bytes<PAY>(T * I) + (PAY ? sizeof(P) * T * I : 0) +
         (sizeof(int32_t) + sizeof(uint32_t)) * T * I +
         (STABLE ? sizeof(uint16_t) * (T / 32) * F : 2 * sizeof(uint32_t) * F) + sizeof(uint32_t) * F;
}

// One block of T threads per super-tile (see the file comment), sub-tiles of T * I rows.
// offs: exclusive scan of hist. With STG > 0 and 16-byte aligned columns, thread 0 keeps the
// next STG whole sub-tiles in flight as bulk copies (TMA) into a shared-memory ring while the
// block ranks and writes the current one; the last, partial sub-tile is loaded directly. A
// ring wait is bounded: when it runs out the block sets ST_TIMEOUT in `status`, lets its
// copies land and leaves.
// STABLE ranks each warp's rows in row order (per-warp digit counters and a block scan over
// warps x digits). Otherwise a row's rank inside its sub-tile is the arrival order of one
// shared-memory atomic on its digit's counter, and only F counters are scanned: super-tiles
// and sub-tiles still go out in input order, the rows of one sub-tile and digit in any order.
template <class Src, class P, bool PAY, int T, int I, int STG, bool STABLE>
__global__ void __launch_bounds__(T) rx_scatter_kernel(Src src, uint32_t G, int shift, int dbits,
                                                       const uint32_t* __restrict__ offs, int32_t* __restrict__ kout,
                                                       P* __restrict__ pout, uint32_t* status) {
  constexpr int W = T / 32, TILE = T * I, WROWS = TILE / W;
  constexpr int NS = STG > 0 ? STG : 1;   // ring stages (1 when there is no ring)
  constexpr uint32_t SB = STG ? Src::template stage_bytes<PAY>(TILE) : 0u;
  extern __shared__ __align__(128) unsigned char rx_smem[];
  __shared__ __align__(8) uint64_t full[NS];
  const uint32_t F = 1u << dbits, dmask = F - 1;
  unsigned char* ring = rx_smem;
  P* spay = reinterpret_cast<P*>(rx_smem + STG * SB);
  // staged rows as (key, output row) pairs, one 8-byte access each way
  int2* sko = reinterpret_cast<int2*>(rx_smem + STG * SB + (PAY ? sizeof(P) * TILE : 0));
  uint16_t* wcnt = reinterpret_cast<uint16_t*>(sko + TILE);             // stable: [warp][digit]
  uint32_t* cur = reinterpret_cast<uint32_t*>(wcnt + W * F);            // stable: next output row per digit
  uint2* sc = reinterpret_cast<uint2*>(sko + TILE);                     // unstable: [digit] {staged start, next output row}
  uint32_t* cnt = reinterpret_cast<uint32_t*>(sc + F);                  // unstable: [digit] counts
  __shared__ uint32_t wt[W];
  __shared__ uint32_t s_total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t n = src.rows();
  const uint64_t super_rows = rx_super_rows_for(n, G, TILE);
  const uint64_t g0 = (uint64_t)blockIdx.x * super_rows;
  if (g0 >= n) return;   // uniform across the block
  const uint64_t g1 = min(g0 + super_rows, n);
  // whole sub-tiles that come through the ring
  const uint64_t nring = (STG > 0 && src.bulk_ok()) ? (g1 - g0) / TILE : 0;
  if (STG > 0 && threadIdx.x == 0 && nring) {
    for (int q = 0; q < NS; q++) mbar_init(&full[q], 1);
    mbar_fence_init();
  }
  if (STABLE) {
    for (uint32_t d = threadIdx.x; d < F; d += T) cur[d] = offs[(size_t)d * G + blockIdx.x];
    for (uint32_t i = threadIdx.x; i < W * F; i += T) wcnt[i] = 0;
  } else {
    for (uint32_t d = threadIdx.x; d < F; d += T) {
      sc[d] = make_uint2(0u, offs[(size_t)d * G + blockIdx.x]);
      cnt[d] = 0;
    }
  }
  __syncthreads();
  if (STG > 0 && threadIdx.x == 0)
    for (uint64_t q = 0; q < nring && q < (uint64_t)NS; q++)
      src.template issue<PAY, TILE>(g0 + q * TILE, ring + (q % NS) * SB, &full[q % NS]);
  uint16_t* mine = wcnt + warp * F;
  const uint32_t dpt = (F + T - 1) / T;   // digits per thread in the scan
  uint64_t k = 0;
  for (uint64_t t0 = g0; t0 < g1; t0 += TILE, k++) {
    int32_t key[I];
    P pay[I];
    uint32_t dr[I];   // digit << 16 | rank (stable: among the warp's rows of that digit); ~0u: no row
    const uint32_t wo = (uint32_t)warp * WROWS + lane;   // this thread's first row of the sub-tile
    if (STG > 0 && k < nring) {
      const int q = (int)(k % NS);
      const bool ok = mbar_wait(&full[q], (uint32_t)((k / NS) & 1), kMbarPollLimit);
      if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) {
          set_status(status, ST_TIMEOUT);
          for (uint64_t x = k; x < nring && x < k + NS; x++)
            mbar_wait(&full[x % NS], (uint32_t)((x / NS) & 1), kMbarPollLimit);
        }
        return;
      }
      const unsigned char* st = ring + q * SB;
#pragma unroll
      for (int j = 0; j < I; j++) {
        const uint32_t i = wo + (uint32_t)j * 32;
        const bool v = src.template staged<PAY, TILE>(st, i, t0 + i, key[j], pay[j]);
        dr[j] = v ? 0u : ~0u;
      }
    } else {
#pragma unroll
      for (int j = 0; j < I; j++) {
        const uint64_t r = t0 + wo + (uint64_t)j * 32;
        const bool v = r < g1 && src.key(r, key[j]);
        dr[j] = v ? 0u : ~0u;
        if (PAY && v) pay[j] = src.payload(r);
      }
    }
    if (STABLE) {
      // rank inside the warp, 32 rows at a time in row order: the first lane of each digit
      // reads and advances the warp's counter for it
#pragma unroll
      for (int j = 0; j < I; j++) {
        const bool v = dr[j] == 0u;
        const uint32_t d = v ? rx_digit(key[j], shift, dmask) : 0x10000u + lane;
        const uint32_t peers = __match_any_sync(FULL_MASK, d);
        const int leader = __ffs(peers) - 1;
        uint32_t base = (v && lane == leader) ? (uint32_t)mine[d] : 0u;
        base = __shfl_sync(FULL_MASK, base, leader);
        if (v) {
          if (lane == leader) mine[d] = (uint16_t)(base + __popc(peers));
          dr[j] = (d << 16) | (base + __popc(peers & lanemask_lt()));
        }
        __syncwarp();
      }
    } else {
#pragma unroll
      for (int j = 0; j < I; j++)
        if (dr[j] == 0u) {
          const uint32_t d = rx_digit(key[j], shift, dmask);
          dr[j] = (d << 16) | atomicAdd(&cnt[d], 1u);
        }
    }
    __syncthreads();
    // every thread has read its rows of the ring stage: refill it STG sub-tiles ahead
    if (STG > 0 && threadIdx.x == 0 && k + NS < nring)
      src.template issue<PAY, TILE>(g0 + (k + NS) * TILE, ring + (k % NS) * SB, &full[k % NS]);
    if (STABLE) {
      // (digit, warp) counts -> staged positions, digit-major: digit d's rows of warp 0, then
      // of warp 1, ... (row order); wcnt[0][d] becomes the start of digit d
      const uint32_t b0 = min(threadIdx.x * dpt, F), b1 = min(b0 + dpt, F);
      uint32_t sum = 0;
      for (uint32_t b = b0; b < b1; b++)
#pragma unroll
        for (int w = 0; w < W; w++) sum += wcnt[w * F + b];
      const uint32_t inc = rx_block_scan<T>(sum, wt);
      uint32_t run = inc - sum;
      for (uint32_t b = b0; b < b1; b++)
#pragma unroll
        for (int w = 0; w < W; w++) {
          const uint32_t c = wcnt[w * F + b];
          wcnt[w * F + b] = (uint16_t)run;
          run += c;
        }
      if (threadIdx.x == T - 1) s_total = inc;
    } else {
      // digit counts -> where each digit's rows start in the staging
      const uint32_t b0 = min(threadIdx.x * dpt, F), b1 = min(b0 + dpt, F);
      uint32_t sum = 0;
      for (uint32_t b = b0; b < b1; b++) sum += cnt[b];
      const uint32_t inc = rx_block_scan<T>(sum, wt);
      uint32_t run = inc - sum;
      for (uint32_t b = b0; b < b1; b++) {
        sc[b].x = run;
        run += cnt[b];
      }
      if (threadIdx.x == T - 1) s_total = inc;
    }
    __syncthreads();
    // stage digit-sorted, with each row's output row (its digit's cursor plus its rank
    // among the sub-tile's rows of that digit)
#pragma unroll
    for (int j = 0; j < I; j++)
      if (dr[j] != ~0u) {
        const uint32_t d = dr[j] >> 16, rank = dr[j] & 0xFFFFu;
        uint32_t pos, o;
        if (STABLE) {
          pos = (uint32_t)mine[d] + rank;
          o = cur[d] + pos - (uint32_t)wcnt[d];
        } else {
          const uint2 v = sc[d];
          pos = v.x + rank;
          o = v.y + rank;
        }
        sko[pos] = make_int2(key[j], (int32_t)o);
        if (PAY) spay[pos] = pay[j];
      }
    __syncthreads();
    // write out: consecutive threads take consecutive staged rows, i.e. consecutive output
    // rows inside each digit's run; the I rows of a thread are independent
    const uint32_t m = s_total;
#pragma unroll
    for (int j = 0; j < I; j++) {
      const uint32_t i = threadIdx.x + (uint32_t)j * T;
      if (i < m) {
        const int2 v = sko[i];
        kout[(uint32_t)v.y] = v.x;
        if (PAY) pout[(uint32_t)v.y] = spay[i];
      }
    }
    __syncthreads();
    if (STABLE) {
      for (uint32_t d = threadIdx.x; d < F; d += T) {
        const uint32_t end = d + 1 < F ? (uint32_t)wcnt[d + 1] : m;
        cur[d] += end - (uint32_t)wcnt[d];
      }
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < W * F; i += T) wcnt[i] = 0;
    } else {
      for (uint32_t d = threadIdx.x; d < F; d += T) {
        sc[d].y += cnt[d];
        cnt[d] = 0;
      }
    }
    __syncthreads();
  }
}

// offsets[b] = where digit b starts (the first super-tile's run), offsets[F] = total.
static __global__ void rx_starts_kernel(const uint32_t* __restrict__ offs, uint32_t F, uint32_t G,
                                        const uint32_t* __restrict__ total, uint32_t* __restrict__ offsets) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b <= F; b += gridDim.x * blockDim.x)
    offsets[b] = b < F ? offs[(size_t)b * G] : *total;
}

// Scratch words for one partitioning with `bits` bits over G super-tiles.
inline size_t rx_scratch_words(uint32_t G, int bits) {
  const size_t hn = (size_t)kRxMaxF * G + 1;
  const size_t parts = (size_t)1 << bits;
  return 2 * hn + std::max(scan_tiles_count(hn), scan_tiles_count(parts)) + 8 + parts + 8;
}

// Partitions the rows of `src` (at most n_max) into 2^bits partitions: keys (and payloads
// when PAY) to kout/pout, partition starts to offsets[0 .. 2^bits] (the total last). Two
// passes when bits > kRxPassBits, through ktmp/ptmp (n_max rows each). The scatter kernel
// runs with T threads, I rows per thread and an STG-stage bulk-copy ring (0: direct loads);
// there are as many super-tiles as its blocks fit on the GPU at once (fewer for a small
// input).
template <class Src, class P, bool PAY, int T, int I, int STG, bool STABLE>
int rx_partition_shaped(Call& call, const Src& src, uint64_t n_max, int bits, int32_t* kout, P* pout,
                        uint32_t* offsets, int32_t* ktmp, P* ptmp) {
  constexpr uint32_t TILE = T * I;
  gpudb_ctx* ctx = call.ctx();
  cudaStream_t s = call.stream();
  const int passes = bits <= kRxPassBits ? 1 : 2;
  const int d0 = passes == 1 ? bits : (bits + 1) / 2;
  auto k0 = rx_scatter_kernel<Src, P, PAY, T, I, STG, STABLE>;
  // the second pass is always stable: it must keep the first pass's order inside each of its
  // digits, or the rows of one final partition would not be contiguous
  auto k1 = rx_scatter_kernel<ColumnSource<P>, P, PAY, T, I, STG, true>;
  const size_t smem0 = rx_scatter_smem<Src, P, PAY, T, I, STG, STABLE>(1u << d0);
  GPUDB_CUDA(ctx, kernel_smem(ctx, (const void*)k0, smem0));
  if (passes > 1)
    GPUDB_CUDA(ctx, kernel_smem(ctx, (const void*)k1, rx_scatter_smem<ColumnSource<P>, P, PAY, T, I, STG, true>(1u << (bits - d0))));
  const int per_sm = kernel_occupancy(ctx, (const void*)k0, T, smem0);
  const uint64_t sub = (std::max<uint64_t>(n_max, 1) + TILE - 1) / TILE;
  const uint32_t G = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(sub, (uint64_t)ctx->sm_count * std::max(per_sm, 1)));
  const size_t hn = (size_t)kRxMaxF * G + 1;
  const size_t parts = (size_t)1 << bits;
  void* sc = nullptr;
  int rc = scratch(ctx, "radix.meta", rx_scratch_words(G, bits) * sizeof(uint32_t), &sc);
  if (rc) return rc;
  uint32_t* hist = static_cast<uint32_t*>(sc);
  uint32_t* offs = hist + hn;
  uint32_t* stmp = offs + hn;
  uint32_t* full = stmp + std::max(scan_tiles_count(hn), scan_tiles_count(parts)) + 8;
  for (int pass = 0; pass < passes; pass++) {
    const int shift = pass == 0 ? 0 : d0;
    const int dbits = pass == 0 ? d0 : bits - d0;
    const uint32_t F = 1u << dbits;
    const size_t hf = (size_t)F * G;
    int32_t* ko = pass == passes - 1 ? kout : ktmp;
    P* po = pass == passes - 1 ? pout : ptmp;
    const size_t sm0 = rx_scatter_smem<Src, P, PAY, T, I, STG, STABLE>(F);
    const size_t sm1 = rx_scatter_smem<ColumnSource<P>, P, PAY, T, I, STG, true>(F);
    GPUDB_CUDA(ctx, cudaMemsetAsync(hist, 0, hf * sizeof(uint32_t), s));
    if (pass == 0 && passes > 1) GPUDB_CUDA(ctx, cudaMemsetAsync(full, 0, parts * sizeof(uint32_t), s));
    uint32_t* fullp = (pass == 0 && passes > 1) ? full : nullptr;
    if (pass == 0) {
      GPUDB_LAUNCH(call, (rx_hist_kernel<Src>), G * kRxHistSplit, kRxThreads, 0, src, G, TILE, shift, dbits, bits,
                   hist, fullp);
      rc = exclusive_scan<uint32_t, uint32_t>(call, hist, hf, offs, stmp, offs + hf);
      if (rc) return rc;
      GPUDB_LAUNCH(call, k0, G, T, sm0, src, G, shift, dbits,
                   (const uint32_t*)offs, ko, po, call.status());
    } else {
      // rows of the first pass, in their pass-one order; their count is the first scan's total
      const uint32_t* total0 = full + parts;   // copied below
      const ColumnSource<P> s2{ktmp, PAY ? ptmp : nullptr, n_max, total0};
      GPUDB_LAUNCH(call, (rx_hist_kernel<ColumnSource<P>>), G * kRxHistSplit, kRxThreads, 0, s2, G, TILE, shift,
                   dbits, bits, hist, (uint32_t*)nullptr);
      rc = exclusive_scan<uint32_t, uint32_t>(call, hist, hf, offs, stmp, offs + hf);
      if (rc) return rc;
      GPUDB_LAUNCH(call, k1, G, T, sm1, s2, G, shift, dbits,
                   (const uint32_t*)offs, ko, po, call.status());
    }
    if (pass == 0 && passes > 1)
      GPUDB_CUDA(ctx, cudaMemcpyAsync(full + parts, offs + hf, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
  if (passes == 1) {
    const uint32_t F = 1u << bits;
    GPUDB_LAUNCH(call, rx_starts_kernel, (F + 256) / 256, 256, 0, (const uint32_t*)offs, F, G,
                 (const uint32_t*)(offs + (size_t)F * G), offsets);
    return GPUDB_OK;
  }
  return exclusive_scan<uint32_t, uint32_t>(call, full, parts, offsets, stmp, offsets + parts);
}

// Largest shared memory a scatter block may use (the B200 opt-in limit per block).
constexpr size_t kRxSmemLimit = 226 * 1024;

// Whether a scatter shape's blocks fit in shared memory for a partitioning of `bits` bits.
template <class Src, class P, bool PAY, int T, int I, int STG, bool STABLE>
constexpr bool rx_shape_fits(int bits) {
  const int d0 = bits <= kRxPassBits ? bits : (bits + 1) / 2;
  return rx_scatter_smem<Src, P, PAY, T, I, STG, STABLE>(1u << d0) <= kRxSmemLimit &&
         rx_scatter_smem<ColumnSource<P>, P, PAY, T, I, STG, true>(1u << (bits - d0 > 0 ? bits - d0 : 0)) <= kRxSmemLimit;
}

// The scatter block shape of the context (GPUDB_OPT_RADIX_SHAPE): 1 512 threads x 16 rows,
// 2 256 x 8 (both with direct loads), 3 512 x 8, 4 256 x 8, 5 512 x 16, 7 256 x 16 (each
// with a two-stage bulk-copy ring), 6 512 x 16 with a one-stage ring (more blocks per SM);
// 0 (default) picks 5. A shape whose shared memory does not fit falls back to 3, then 4,
// then 2. STABLE: rows keep their input order inside a partition.
template <class Src, class P, bool PAY, bool STABLE>
int rx_partition(Call& call, const Src& src, uint64_t n_max, int bits, int32_t* kout, P* pout, uint32_t* offsets,
                 int32_t* ktmp, P* ptmp) {
  int shape = call.ctx()->radix_shape ? call.ctx()->radix_shape : 5;
  if (shape == 6 && !rx_shape_fits<Src, P, PAY, 512, 16, 1, STABLE>(bits)) shape = 3;
  if (shape == 7 && !rx_shape_fits<Src, P, PAY, 256, 16, 2, STABLE>(bits)) shape = 4;
  if (shape == 5 && !rx_shape_fits<Src, P, PAY, 512, 16, 2, STABLE>(bits)) shape = 3;
  if (shape == 3 && !rx_shape_fits<Src, P, PAY, 512, 8, 2, STABLE>(bits)) shape = 4;
  if (shape == 4 && !rx_shape_fits<Src, P, PAY, 256, 8, 2, STABLE>(bits)) shape = 2;
  switch (shape) {
    case 1:
      return rx_partition_shaped<Src, P, PAY, 512, 16, 0, STABLE>(call, src, n_max, bits, kout, pout, offsets, ktmp, ptmp);
    case 3:
      return rx_partition_shaped<Src, P, PAY, 512, 8, 2, STABLE>(call, src, n_max, bits, kout, pout, offsets, ktmp, ptmp);
    case 4:
      return rx_partition_shaped<Src, P, PAY, 256, 8, 2, STABLE>(call, src, n_max, bits, kout, pout, offsets, ktmp, ptmp);
    case 5:
      return rx_partition_shaped<Src, P, PAY, 512, 16, 2, STABLE>(call, src, n_max, bits, kout, pout, offsets, ktmp, ptmp);
    case 6:
      return rx_partition_shaped<Src, P, PAY, 512, 16, 1, STABLE>(call, src, n_max, bits, kout, pout, offsets, ktmp, ptmp);
    case 7:
      return rx_partition_shaped<Src, P, PAY, 256, 16, 2, STABLE>(call, src, n_max, bits, kout, pout, offsets, ktmp, ptmp);
    default:
      return rx_partition_shaped<Src, P, PAY, 256, 8, 0, STABLE>(call, src, n_max, bits, kout, pout, offsets, ktmp, ptmp);
  }
}

// Plain columns (payload = row id when pay is null); the row count may be on the device.
// STABLE (the C ABI's partitioning) keeps the input order inside each partition; the joins,
// whose results do not depend on it, take the unstable form (for the first pass; a second
// pass is always stable).
template <class P, bool STABLE>
int radix_partition_run(Call& call, const int32_t* keys, const P* pay, uint64_t n_max, const uint32_t* n_dev, int bits,
                        int32_t* keys_out, P* pay_out, uint32_t* offsets, int32_t* keys_tmp, P* pay_tmp) {
  const ColumnSource<P> src{keys, pay, n_max, n_dev};
  return rx_partition<ColumnSource<P>, P, true, STABLE>(call, src, n_max, bits, keys_out, pay_out, offsets, keys_tmp,
                                                       pay_tmp);
}

// Keys only (no payload column is read or written), unstable.
inline int radix_partition_keys(Call& call, const int32_t* keys, uint64_t n, int bits, int32_t* keys_out,
                                uint32_t* offsets, int32_t* keys_tmp) {
  const ColumnSource<int32_t> src{keys, nullptr, n, nullptr};
  return rx_partition<ColumnSource<int32_t>, int32_t, false, false>(call, src, n, bits, keys_out, nullptr, offsets,
                                                                    keys_tmp, nullptr);
}

// Partition bits so that the average partition holds about `per_part` rows.
inline int radix_bits_for(uint64_t n, uint64_t per_part) {
  int b = 0;
  while (b < kRadixMaxBits && (n >> b) > per_part) b++;
  return b;
}

}  // namespace gpudb
