// Microbenchmark operators: selection, column sum and hash-join match count.
// Reference: runSelectionBenchmark / runAggregationBenchmark / runJoinBenchmark
// (src/microbenchmarks.cpp:8-251) and selection_kernel, sum_kernel_stage1/2,
// hash_join_build/probe (kernels/microbenchmarks.metal:160-294).
//
// B200 design:
//  - selection: 32-bit words of the row bitmask (the reference writes one 32-bit 0/1 word
//    per row). Bitmask and count alone: one kernel over SMs x occupancy blocks, 128-bit
//    loads a tile ahead, one atomic add per block. With row ids: per-tile counts, a device
//    scan, and a second pass that compacts the ids in input order (one ballot per 32 rows);
//  - sum: 128-bit loads, int64 per thread, warp shuffle + last-block fold (one launch);
//  - join count: build keys go into an open-addressing set (atomicCAS, power of two,
//    <= 50% load); probe rows count once per row at the first match (semi-join count,
//    as hash_join_probe does). Radix mode lives in radix.cu. Direct mode: the build keys'
//    [min, max] found on the device, one bit per key of that span (order keys of 15M
//    orders: 7.5 MB, L2-resident), and the probe streams its keys against the bits.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"
#include "micro.h"
#include "scan.cuh"

namespace gpudb {
namespace {

constexpr int kThreads = 256;
constexpr int kSelTile = kThreads * 16;     // rows per block in the selection kernels

// Bits and per-tile counts. Each warp step covers 128 rows: a lane loads 4 rows with one
// 128-bit load (scalar loads on a ragged or unaligned tail), forms a 4-bit nibble, and an
// OR-butterfly over 8 lanes assembles each 32-row word of the bitmask.
__global__ void __launch_bounds__(kThreads) select_count_kernel(const int32_t* __restrict__ col, uint64_t n,
                                                                int32_t value, uint32_t* bits, uint32_t* tile_counts) {
  __shared__ uint32_t wc[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * kSelTile;
  const bool vec = (reinterpret_cast<uintptr_t>(col) & 15u) == 0;
  uint32_t c = 0;
#pragma unroll 2
  for (int w = warp; w < kSelTile / 128; w += kThreads / 32) {
    const uint64_t r = base + (uint64_t)w * 128 + 4 * lane;
    uint32_t nib = 0;
    if (vec && r + 4 <= n) {
      const int4 v = ld_stream(reinterpret_cast<const int4*>(col + r));
      nib = (uint32_t)(v.x < value) | ((uint32_t)(v.y < value) << 1) | ((uint32_t)(v.z < value) << 2) |
            ((uint32_t)(v.w < value) << 3);
    } else {
      for (int i = 0; i < 4; i++)
        if (r + i < n && col[r + i] < value) nib |= 1u << i;
    }
    c += __popc(nib);
    uint32_t word = nib << (4 * (lane & 7));
    word |= __shfl_xor_sync(FULL_MASK, word, 1);
    word |= __shfl_xor_sync(FULL_MASK, word, 2);
    word |= __shfl_xor_sync(FULL_MASK, word, 4);
    const uint64_t wr = base + (uint64_t)w * 128 + 32 * (lane >> 3);   // first row of this word
    if (bits && (lane & 7) == 0 && wr < n) bits[wr >> 5] = word;
  }
  c = __reduce_add_sync(FULL_MASK, c);
  if (lane == 0) wc[warp] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kThreads / 32; w++) t += wc[w];
    tile_counts[blockIdx.x] = t;
  }
}

// Bitmask (when given) and count, no row ids, so no per-tile counts: a grid of SMs x occupancy
// blocks walks the tiles; a lane's four 128-row steps of a tile are loaded together, one
// tile ahead of the one being tested, the words are assembled as in select_count_kernel,
// and each block adds its count to *total once.
__global__ void __launch_bounds__(kThreads) select_bits_kernel(const int32_t* __restrict__ col, uint64_t n,
                                                               int32_t value, uint32_t* bits,
                                                               unsigned long long* total) {
  constexpr int kSteps = kSelTile / 128 / (kThreads / 32);   // 128-row steps of a warp per tile
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool vec = (reinterpret_cast<uintptr_t>(col) & 15u) == 0;
  const uint64_t tiles = (n + kSelTile - 1) / kSelTile;
  uint32_t c = 0;
  int4 nv[kSteps];   // the block's next tile, loading while this one is tested
  auto prefetch = [&](uint64_t tile) {
    if (vec && tile < tiles && (tile + 1) * kSelTile <= n) {
#pragma unroll
      for (int k = 0; k < kSteps; k++)
        nv[k] = ld_stream(reinterpret_cast<const int4*>(col + tile * kSelTile +
                                                        (uint64_t)(warp + k * (kThreads / 32)) * 128 + 4 * lane));
    }
  };
  prefetch(blockIdx.x);
  for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const uint64_t base = tile * kSelTile;
    const bool full = vec && base + kSelTile <= n;
    int4 v[kSteps];
#pragma unroll
    for (int k = 0; k < kSteps; k++) v[k] = nv[k];
    prefetch(tile + gridDim.x);
#pragma unroll
    for (int k = 0; k < kSteps; k++) {
      const uint64_t r = base + (uint64_t)(warp + k * (kThreads / 32)) * 128 + 4 * lane;
      uint32_t nib = 0;
      if (full) {
        nib = (uint32_t)(v[k].x < value) | ((uint32_t)(v[k].y < value) << 1) | ((uint32_t)(v[k].z < value) << 2) |
              ((uint32_t)(v[k].w < value) << 3);
      } else {
        for (int i = 0; i < 4; i++)
          if (r + i < n && col[r + i] < value) nib |= 1u << i;
      }
      c += __popc(nib);
      uint32_t word = nib << (4 * (lane & 7));
      word |= __shfl_xor_sync(FULL_MASK, word, 1);
      word |= __shfl_xor_sync(FULL_MASK, word, 2);
      word |= __shfl_xor_sync(FULL_MASK, word, 4);
      const uint64_t wr = r - 4 * (lane & 7);   // first row of this word
      if (bits && (lane & 7) == 0 && wr < n) bits[wr >> 5] = word;
    }
  }
  c = __reduce_add_sync(FULL_MASK, c);
  __shared__ uint32_t wc[kThreads / 32];
  if (lane == 0) wc[warp] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kThreads / 32; w++) t += wc[w];
    if (t) atomicAdd(total, (unsigned long long)t);
  }
}

// Row ids in input order: tile offset + rank inside the tile.
__global__ void __launch_bounds__(kThreads) select_rows_kernel(const int32_t* __restrict__ col, uint64_t n, int32_t value,
                                                               const uint64_t* __restrict__ tile_offsets, uint32_t* rows) {
  __shared__ uint32_t wc[kSelTile / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * kSelTile;
  uint32_t masks[kSelTile / 32 / (kThreads / 32)];
#pragma unroll
  for (int j = 0; j < kSelTile / kThreads; j++) {
    const int w = warp + j * (kThreads / 32);
    const uint64_t r = base + (uint64_t)w * 32 + lane;
    const bool hit = r < n && col[r] < value;
    masks[j] = __ballot_sync(FULL_MASK, hit);
    if (lane == 0) wc[w] = __popc(masks[j]);
  }
  __syncthreads();
  // exclusive scan of the 128 word counts (one warp)
  if (warp == 0) {
    uint32_t v[4], s = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) { v[i] = wc[lane * 4 + i]; s += v[i]; }
    uint32_t inc = s;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t o = __shfl_up_sync(FULL_MASK, inc, d);
      if (lane >= d) inc += o;
    }
    uint32_t run = inc - s;
#pragma unroll
    for (int i = 0; i < 4; i++) { wc[lane * 4 + i] = run; run += v[i]; }
  }
  __syncthreads();
  const uint64_t off = tile_offsets[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kSelTile / kThreads; j++) {
    const int w = warp + j * (kThreads / 32);
    const uint32_t m = masks[j];
    if ((m >> lane) & 1u) rows[off + wc[w] + __popc(m & lanemask_lt())] = (uint32_t)(base + (uint64_t)w * 32 + lane);
  }
}

__global__ void __launch_bounds__(kThreads) sum_i32_kernel(const int32_t* __restrict__ col, uint64_t n, bool vec,
                                                           int64_t* partials, unsigned* ticket, int64_t* out) {
  const uint64_t T = (uint64_t)gridDim.x * kThreads;
  const uint64_t tid = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  int64_t s = 0;
  if (vec) {
    const uint64_t nq = n >> 2;
    const int4* c4 = reinterpret_cast<const int4*>(col);
    for (uint64_t q = tid; q < nq; q += T) {
      const int4 v = ld_stream(c4 + q);
      s += (int64_t)v.x + v.y + (int64_t)v.z + v.w;
    }
    const uint64_t r = (nq << 2) + tid;
    if (r < n) s += col[r];
  } else {
    for (uint64_t r = tid; r < n; r += T) s += col[r];
  }
  __shared__ uint64_t sw[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t v = warp_sum_u64((uint64_t)s);
  if (lane == 0) sw[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t t = 0;
    for (int w = 0; w < kThreads / 32; w++) t += sw[w];
    partials[blockIdx.x] = (int64_t)t;
  }
  if (!grid_last_block(ticket)) return;
  uint64_t a = 0;
  for (unsigned i = threadIdx.x; i < gridDim.x; i += kThreads) a += (uint64_t)__ldcg(partials + i);
  a = warp_sum_u64(a);
  __syncthreads();
  if (lane == 0) sw[warp] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t t = 0;
    for (int w = 0; w < kThreads / 32; w++) t += sw[w];
    *out += (int64_t)t;
  }
}

__global__ void set_clear_kernel(int32_t* set, uint32_t cap) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += stride) set[i] = kEmptyKey;
}

__global__ void set_insert_kernel(const int32_t* __restrict__ keys, uint64_t n, int32_t* set, uint32_t cap,
                                  uint32_t* status) {
  const uint32_t mask = cap - 1;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t k = keys[i];
    if (k == kEmptyKey) { set_status(status, ST_KEY_RANGE); continue; }
    uint32_t s = key_slot(k, mask);
    bool done = false;
    for (uint32_t p = 0; p < cap && !done; p++, s = (s + 1) & mask) {
      const int32_t prev = atomicCAS(&set[s], kEmptyKey, k);
      done = (prev == kEmptyKey || prev == k);   // duplicates keep one entry (set semantics)
    }
    if (!done) set_status(status, ST_CAPACITY);
  }
}

__global__ void __launch_bounds__(kThreads) set_probe_count_kernel(const int32_t* __restrict__ keys, uint64_t n,
                                                                   const int32_t* __restrict__ set, uint32_t cap,
                                                                   unsigned long long* count) {
  const uint32_t mask = cap - 1;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint32_t c = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t k = ld_stream(keys + i);
    if (k == kEmptyKey) continue;
    uint32_t s = key_slot(k, mask);
    for (uint32_t p = 0; p < cap; p++, s = (s + 1) & mask) {
      const int32_t v = __ldg(set + s);
      if (v == k) { c++; break; }
      if (v == kEmptyKey) break;
    }
  }
  c = __reduce_add_sync(FULL_MASK, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// ---- direct mode: one bit per key of the build keys' span [lo, hi] -----------------------
constexpr uint64_t kDirectMaxSpan = 1ull << 30;   // keys the bitmap may span (128 MB of bits)

// span = {lo, hi} of the build keys. It starts as {0x7F7F7F7F, 0x80808080} (byte memsets),
// which can only widen the span of keys that lie beyond those values; no keys leave hi < lo.
__global__ void __launch_bounds__(kThreads) key_span_kernel(const int32_t* __restrict__ keys, uint64_t n,
                                                            int32_t* span) {
  int32_t lo = INT32_MAX, hi = INT32_MIN;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t k = __ldg(keys + i);   // cached: the bit-setting pass reads the keys again
    lo = min(lo, k);
    hi = max(hi, k);
  }
  lo = __reduce_min_sync(FULL_MASK, lo);
  hi = __reduce_max_sync(FULL_MASK, hi);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(span, lo);
    atomicMax(span + 1, hi);
  }
}

// Whether the span is usable: not empty and at most kDirectMaxSpan keys.
__device__ __forceinline__ bool span_usable(const int32_t* span, int64_t* lo, uint32_t* range) {
  const int64_t l = span[0], h = span[1];
  *lo = l;
  *range = (uint32_t)(h - l);
  return h >= l && (uint64_t)(h - l) < kDirectMaxSpan;
}

// Clears the span's bitmap words; a span over kDirectMaxSpan keys sets ST_KEY_RANGE instead.
__global__ void __launch_bounds__(kThreads) span_clear_kernel(const int32_t* span, uint32_t* bm, uint32_t* status) {
  int64_t lo;
  uint32_t range;
  if (!span_usable(span, &lo, &range)) {
    if (span[1] >= span[0] && blockIdx.x == 0 && threadIdx.x == 0) set_status(status, ST_KEY_RANGE);
    return;
  }
  const uint64_t words = ((uint64_t)range >> 5) + 1, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) bm[i] = 0u;
}

__global__ void __launch_bounds__(kThreads) span_set_kernel(const int32_t* __restrict__ keys, uint64_t n,
                                                            const int32_t* span, uint32_t* bm) {
  int64_t lo;
  uint32_t range;
  if (!span_usable(span, &lo, &range)) return;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t x = (uint32_t)((int64_t)__ldg(keys + i) - lo);   // in [0, range]: lo <= key <= hi
    atomicOr(bm + (x >> 5), 1u << (x & 31u));
  }
}

__device__ __forceinline__ uint32_t span_hit(const uint32_t* bm, int64_t lo, uint32_t range, int32_t k) {
  const int64_t d = (int64_t)k - lo;   // 64-bit: no key outside the span can alias into it
  return d >= 0 && d <= (int64_t)range ? (__ldg(bm + ((uint64_t)d >> 5)) >> ((uint32_t)d & 31u)) & 1u : 0u;
}

// Probe rows whose key's bit is set: 128-bit loads of the keys where the column allows.
__global__ void __launch_bounds__(kThreads) span_probe_kernel(const int32_t* __restrict__ keys, uint64_t n,
                                                              const int32_t* span, const uint32_t* __restrict__ bm,
                                                              unsigned long long* count) {
  int64_t lo;
  uint32_t range;
  if (!span_usable(span, &lo, &range)) return;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x, tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t c = 0;
  if ((reinterpret_cast<uintptr_t>(keys) & 15u) == 0) {
    const uint64_t nq = n >> 2;
    for (uint64_t q = tid; q < nq; q += stride) {
      const int4 v = ld_stream(reinterpret_cast<const int4*>(keys) + q);
      c += span_hit(bm, lo, range, v.x) + span_hit(bm, lo, range, v.y) + span_hit(bm, lo, range, v.z) +
           span_hit(bm, lo, range, v.w);
    }
    const uint64_t r = (nq << 2) + tid;
    if (r < n) c += span_hit(bm, lo, range, keys[r]);
  } else {
    for (uint64_t i = tid; i < n; i += stride) c += span_hit(bm, lo, range, ld_stream(keys + i));
  }
  c = __reduce_add_sync(FULL_MASK, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

unsigned grid_of(gpudb_ctx* ctx, uint64_t items, int per_sm) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + kThreads - 1) / kThreads, (uint64_t)ctx->sm_count * per_sm));
}

}  // namespace

// Open-addressing set of the build keys (capacity a power of two, <= 50% load).
int build_key_set(Call& call, const int32_t* keys, uint64_t n, int32_t** set_out, uint32_t* cap_out) {
  gpudb_ctx* ctx = call.ctx();
  uint32_t cap = 1024;
  while (cap < 2 * n && cap < (1u << 31)) cap <<= 1;
  void* set = nullptr;
  int rc = scratch(ctx, "join.set", (size_t)cap * 4, &set);
  if (rc) return rc;
  GPUDB_LAUNCH(call, set_clear_kernel, grid_of(ctx, cap, 16), kThreads, 0, (int32_t*)set, cap);
  if (n) GPUDB_LAUNCH(call, set_insert_kernel, grid_of(ctx, n, 16), kThreads, 0, keys, n, (int32_t*)set, cap, call.status());
  *set_out = (int32_t*)set;
  *cap_out = cap;
  return GPUDB_OK;
}

}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_select_lt(gpudb_ctx* ctx, const int32_t* col, uint64_t n, int32_t value, uint32_t* out_bits,
                               uint32_t* out_rows, uint64_t* count, gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!count || (n && !col)) return fail(ctx, GPUDB_E_INVALID, "select: col and count are required");
  if (n >= (1ull << 32)) return fail(ctx, GPUDB_E_INVALID, "select: at most 2^32-1 rows (32-bit row ids)");
  Call call(ctx, ex, t);
  int rc = call.begin(16);
  if (rc) return rc;
  const uint64_t tiles = (n + kSelTile - 1) / kSelTile;
  void* tmp = nullptr;
  rc = scratch(ctx, "select.tiles", (tiles + 1) * 4 + (tiles + 2) * 8 * 2 + 64, &tmp);
  if (rc) return rc;
  uint32_t* tile_counts = static_cast<uint32_t*>(tmp);
  uint64_t* tile_off = reinterpret_cast<uint64_t*>(static_cast<uint8_t*>(tmp) + ((tiles + 1) * 4 + 15) / 16 * 16);
  uint64_t* scan_tmp = tile_off + tiles + 2;
  uint64_t* total = call.result<uint64_t>();
  if (n && !out_rows) {
    // (the result slot is zero: Call::begin clears it)
    GPUDB_LAUNCH(call, select_bits_kernel, grid_of(ctx, tiles * kThreads, 8), kThreads, 0, col, n, value, out_bits,
                 reinterpret_cast<unsigned long long*>(total));
  } else if (n) {
    GPUDB_LAUNCH(call, select_count_kernel, (unsigned)tiles, kThreads, 0, col, n, value, out_bits, tile_counts);
    rc = exclusive_scan<uint32_t, uint64_t>(call, tile_counts, tiles, tile_off, scan_tmp, total);
    if (rc) return rc;
    if (out_rows)
      GPUDB_LAUNCH(call, select_rows_kernel, (unsigned)tiles, kThreads, 0, col, n, value, (const uint64_t*)tile_off,
                   out_rows);
  }
  return call.finish(16, [count](const uint8_t* h) {
    std::memcpy(count, h, 8);
    return GPUDB_OK;
  });
}

extern "C" int gpudb_sum_i32(gpudb_ctx* ctx, const int32_t* col, uint64_t n, int64_t* sum, gpudb_timing* t,
                             const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!sum || (n && !col)) return fail(ctx, GPUDB_E_INVALID, "sum: col and sum are required");
  Call call(ctx, ex, t);
  int rc = call.begin(16);
  if (rc) return rc;
  if (n) {
    const unsigned grid = grid_of(ctx, n / 4 + 1, 8);
    void* p = nullptr;   // new scratch is zeroed (the ticket); each launch's last block resets it
    rc = scratch(ctx, "sum.partials", (size_t)grid * 8 + 256, &p);
    if (rc) return rc;
    const bool vec = (reinterpret_cast<uintptr_t>(col) & 15u) == 0;
    GPUDB_LAUNCH(call, sum_i32_kernel, grid, kThreads, 0, col, n, vec, (int64_t*)((uint8_t*)p + 256), (unsigned*)p,
                 call.result<int64_t>());
  }
  return call.finish(16, [sum](const uint8_t* h) {
    std::memcpy(sum, h, 8);
    return GPUDB_OK;
  });
}

extern "C" int gpudb_hash_join_count(gpudb_ctx* ctx, const int32_t* build_keys, uint64_t n_build,
                                     const int32_t* probe_keys, uint64_t n_probe, int32_t mode, uint64_t* matches,
                                     gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!matches || (n_build && !build_keys) || (n_probe && !probe_keys))
    return fail(ctx, GPUDB_E_INVALID, "join: keys and matches are required");
  if (mode != GPUDB_JOIN_GLOBAL && mode != GPUDB_JOIN_RADIX && mode != GPUDB_JOIN_DIRECT)
    return fail(ctx, GPUDB_E_INVALID, "join: unknown mode");
  if (n_build > (1ull << 30)) return fail(ctx, GPUDB_E_INVALID, "join: build side larger than 2^30 rows");
  Call call(ctx, ex, t);
  int rc = call.begin(16);
  if (rc) return rc;
  unsigned long long* cnt = call.result<unsigned long long>();
  if (mode == GPUDB_JOIN_GLOBAL) {
    int32_t* set = nullptr;
    uint32_t cap = 0;
    rc = build_key_set(call, build_keys, n_build, &set, &cap);
    if (rc) return rc;
    if (n_probe)
      GPUDB_LAUNCH(call, set_probe_count_kernel, grid_of(ctx, n_probe, 8), kThreads, 0, probe_keys, n_probe,
                   (const int32_t*)set, cap, cnt);
  } else if (mode == GPUDB_JOIN_DIRECT) {
    // a bitmap over the build keys' span, found on the device (no host round trip)
    void* sp = nullptr;
    void* bm = nullptr;
    rc = scratch(ctx, "join.span", 256, &sp);
    if (!rc) rc = scratch(ctx, "join.bitmap", kDirectMaxSpan / 8, &bm);
    if (rc) return rc;
    int32_t* span = static_cast<int32_t*>(sp);
    GPUDB_CUDA(ctx, cudaMemsetAsync(span, 0x7F, 4, call.stream()));
    GPUDB_CUDA(ctx, cudaMemsetAsync(span + 1, 0x80, 4, call.stream()));
    if (n_build) GPUDB_LAUNCH(call, key_span_kernel, grid_of(ctx, n_build, 8), kThreads, 0, build_keys, n_build, span);
    GPUDB_LAUNCH(call, span_clear_kernel, grid_of(ctx, kDirectMaxSpan / 32, 8), kThreads, 0, (const int32_t*)span,
                 (uint32_t*)bm, call.status());
    if (n_build)
      GPUDB_LAUNCH(call, span_set_kernel, grid_of(ctx, n_build, 8), kThreads, 0, build_keys, n_build,
                   (const int32_t*)span, (uint32_t*)bm);
    if (n_probe)
      GPUDB_LAUNCH(call, span_probe_kernel, grid_of(ctx, n_probe / 4 + 1, 8), kThreads, 0, probe_keys, n_probe,
                   (const int32_t*)span, (const uint32_t*)bm, cnt);
  } else {
    rc = radix_join_count(call, build_keys, n_build, probe_keys, n_probe, cnt);
    if (rc) return rc;
  }
  return call.finish(16, [matches](const uint8_t* h) {
    std::memcpy(matches, h, 8);
    return GPUDB_OK;
  });
}
