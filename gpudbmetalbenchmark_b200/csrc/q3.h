// Q3-like pipeline entry points shared between the global-table (q3.cu) and the
// radix-partitioned (radix.cu) implementations.
#pragma once
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"

namespace gpudb {

// Orders hash-table slot; the table doubles as the per-order aggregation table.
struct Q3Slot {
  int32_t key;
  int32_t date;
  unsigned long long rev;
};

__device__ __forceinline__ int32_t ht_find(const Q3Slot* ht, uint32_t cap, int32_t key) {
  const uint32_t mask = cap - 1;
  uint32_t s = key_slot(key, mask);
  for (uint32_t p = 0; p < cap; p++, s = (s + 1) & mask) {
    const int32_t k = __ldg(&ht[s].key);
    if (k == key) return (int32_t)s;
    if (k == kEmptyKey) return -1;
  }
  return -1;
}

// Other blocks' top-k candidates, read past L1.
__device__ __forceinline__ u128 ld_cg_u128(const u128* p) {
  const ulonglong2 q = __ldcg(reinterpret_cast<const ulonglong2*>(p));
  return ((u128)q.y << 64) | q.x;
}

// ---- top-k of a Q3 table: select by a revenue histogram, then rank ------------------------
// Two streaming passes over the live table (hit counts, 16-byte loads per lane, four 128-slot
// chunks in flight per warp; slots read only where the hit count is nonzero):
//   1. q3_table_hist: counts the groups and builds a histogram of revenue over kRevBins
//      log-scale bins (rev_bin: the leading bit and the 5 bits after it);
//   2. q3_table_select: every block finds the highest bin b* whose count from the top
//      reaches k, appends the slots in bins >= b* (the k best and their near ties) to cand,
//      and the last block to finish ranks the appended composites among themselves.
// Both are exact: every top-k entry is in a bin >= b*, and ranking by the full composite
// settles the order inside b*. Should more than kTopkCandCap slots land in bins >= b* (data
// with very many near-equal revenues), the last block merges the whole table tile by tile
// with block_topk instead.
constexpr int kTopkWarps = kTopkThreads / 32;
constexpr int kRevBins = 2048;
constexpr uint32_t kTopkStateWords = kRevBins + 8;   // histogram, candidate count, ticket
constexpr uint32_t kTopkCandCap = 16384;             // appended candidates per table
constexpr uint32_t kTopkSlotsPerBlock = 4096;        // host-side grid sizing: at least this many slots per block

__device__ __forceinline__ uint32_t rev_bin(unsigned long long rev) {
  if (rev == 0) return 0;
  const int e = 63 - __clzll((long long)rev);
  const uint32_t m = e >= 5 ? (uint32_t)(rev >> (e - 5)) & 31u : (uint32_t)(rev << (5 - e)) & 31u;
  return (uint32_t)e * 32 + m;
}

// Grids of the two passes for a table of at most max_cap slots, fewer blocks for a small
// table; `share` requests split the SMs. The histogram pass (few registers) runs four
// blocks per SM, the select pass two.
inline unsigned q3_topk_grid(uint32_t max_cap, int sms, int share, int per_sm) {
  const uint64_t g = std::min<uint64_t>(max_cap / kTopkSlotsPerBlock, (uint64_t)sms * per_sm / share);
  return (unsigned)std::max<uint64_t>(1, g);
}

constexpr int kChunksInFlight = 4;   // 128-slot chunks a warp loads before using them

// Visits the slots of this warp's chunks, kChunksInFlight at a time: `f(base, valid)` gets
// the first slot of the lane's 4 slots in each chunk and which of the 4 * kChunksInFlight
// slots have hits.
template <class F>
__device__ __forceinline__ void q3_warp_chunks(const uint32_t* __restrict__ hits, uint32_t cap, F&& f) {
  constexpr int U = kChunksInFlight;
  const int lane = threadIdx.x & 31;
  const uint64_t W = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t chunks = cap / 128;
  for (uint64_t c0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c0 < chunks; c0 += U * W) {
    uint4 h[U];
    uint64_t base[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint64_t c = c0 + u * W;
      base[u] = c * 128 + lane * 4;
      h[u] = c < chunks ? __ldg(reinterpret_cast<const uint4*>(hits) + c * 32 + lane) : make_uint4(0, 0, 0, 0);
    }
    uint32_t valid = 0;
#pragma unroll
    for (int u = 0; u < U; u++)
      valid |= ((h[u].x != 0) | (h[u].y != 0) << 1 | (h[u].z != 0) << 2 | (h[u].w != 0) << 3) << (4 * u);
    f(base, valid);
  }
}

__device__ __forceinline__ ulonglong2 q3_slot_load(const Q3Slot* ht, uint64_t s) {
  return __ldg(reinterpret_cast<const ulonglong2*>(ht + s));
}
__device__ __forceinline__ u128 q3_slot_compose(ulonglong2 e) {
  return topk_compose((int64_t)e.y, (int32_t)(e.x >> 32), (int32_t)(uint32_t)e.x);
}

// Pass 1. `state` is the table's kTopkStateWords zeroed words, `sh` kRevBins shared words.
__device__ __forceinline__ void q3_table_hist(const Q3Slot* __restrict__ ht, const uint32_t* __restrict__ hits,
                                              uint32_t cap, uint32_t* state, unsigned long long* groups,
                                              uint32_t* sh) {
  for (int i = threadIdx.x; i < kRevBins; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  uint32_t cnt = 0;
  q3_warp_chunks(hits, cap, [&](const uint64_t (&base)[kChunksInFlight], uint32_t valid) {
    unsigned long long rev[4 * kChunksInFlight];
#pragma unroll
    for (int j = 0; j < 4 * kChunksInFlight; j++)
      rev[j] = (valid >> j & 1) ? __ldg(&ht[base[j >> 2] + (j & 3)].rev) : 0ull;
#pragma unroll
    for (int j = 0; j < 4 * kChunksInFlight; j++)
      if (valid >> j & 1) atomicAdd(&sh[rev_bin(rev[j])], 1u);
    cnt += __popc(valid);
  });
  cnt = __reduce_add_sync(FULL_MASK, cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(groups, (unsigned long long)cnt);
  __syncthreads();
  for (int i = threadIdx.x; i < kRevBins; i += blockDim.x)
    if (sh[i]) atomicAdd(&state[i], sh[i]);
}

// Top-k of n composites given by get(i), kTopkTile - k at a time, with the running top-k in
// `carry` (k entries); one block.
template <class G>
__device__ __forceinline__ void block_topk_stream(uint64_t n, int k, G&& get, u128* carry, u128* sm) {
  const uint64_t per = (uint64_t)kTopkTile - k;
  __syncthreads();
  for (int i = threadIdx.x; i < k; i += kTopkThreads) carry[i] = 0;
  __syncthreads();
  u128 v[kTopkPerThread];
  for (uint64_t c0 = 0; c0 < n; c0 += per) {
#pragma unroll
    for (int j = 0; j < kTopkPerThread; j++) {
      const uint64_t idx = (uint64_t)threadIdx.x * kTopkPerThread + j;
      if (idx < (uint64_t)k) v[j] = carry[idx];
      else v[j] = (c0 + idx - k < n) ? get(c0 + idx - k) : (u128)0;
    }
    __syncthreads();
    block_topk(v, k, carry, sm);
  }
}

// Pass 2 (blockDim.x == kTopkThreads). `sm` is kTopkScratch composites of shared scratch,
// `carry` GPUDB_Q3_MAX_K of them; `out` gets k composites, 0 past the number of groups.
__device__ __forceinline__ void q3_table_select(const Q3Slot* __restrict__ ht, const uint32_t* __restrict__ hits,
                                                uint32_t cap, int k, uint32_t* state, u128* cand, u128* out,
                                                u128* sm, u128* carry) {
  __shared__ uint32_t wsum[kTopkWarps];
  __shared__ uint32_t bstar;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  // thread t owns 8 bins counted down from the top: kRevBins - 1 - (8t + j)
  constexpr int kPer = kRevBins / kTopkThreads;
  uint32_t loc[kPer], sum = 0;
#pragma unroll
  for (int j = 0; j < kPer; j++) {
    loc[j] = __ldcg(state + kRevBins - 1 - (kPer * t + j));
    sum += loc[j];
  }
  uint32_t inc = sum;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(FULL_MASK, inc, d);
    if (lane >= d) inc += o;
  }
  if (lane == 31) wsum[warp] = inc;
  if (t == 0) bstar = 0;
  __syncthreads();
  uint32_t before = inc - sum;
  for (int w = 0; w < warp; w++) before += wsum[w];
  if (before < (uint32_t)k && before + sum >= (uint32_t)k) {
    uint32_t acc = before;
#pragma unroll
    for (int j = 0; j < kPer; j++) {
      acc += loc[j];
      if (acc >= (uint32_t)k) { bstar = kRevBins - 1 - (kPer * t + j); break; }
    }
  }
  __syncthreads();
  const uint32_t bs = bstar;
  uint32_t* ncand = state + kRevBins;
  q3_warp_chunks(hits, cap, [&](const uint64_t (&base)[kChunksInFlight], uint32_t valid) {
    ulonglong2 e[4 * kChunksInFlight];
#pragma unroll
    for (int j = 0; j < 4 * kChunksInFlight; j++)
      e[j] = (valid >> j & 1) ? q3_slot_load(ht, base[j >> 2] + (j & 3)) : make_ulonglong2(0, 0);
#pragma unroll
    for (int j = 0; j < 4 * kChunksInFlight; j++) {
      const bool take = (valid >> j & 1) && rev_bin(e[j].y) >= bs;
      if (__any_sync(FULL_MASK, take)) {
        const uint32_t pos = warp_append(take, ncand);
        if (take && pos < kTopkCandCap) cand[pos] = q3_slot_compose(e[j]);
      }
    }
  });
  if (!grid_last_block(state + kRevBins + 1)) return;
  const uint32_t C = __ldcg(ncand);
  if (C <= (uint32_t)kTopkScratch) {
    for (uint32_t i = t; i < C; i += kTopkThreads) sm[i] = ld_cg_u128(cand + i);
    __syncthreads();
    for (uint32_t i = t; i < C; i += kTopkThreads) {
      const u128 x = sm[i];
      uint32_t r = 0;
      for (uint32_t j = 0; j < C; j++) r += sm[j] > x;
      if (r < (uint32_t)k) out[r] = x;
    }
    for (uint32_t i = C + t; i < (uint32_t)k; i += kTopkThreads) out[i] = 0;
    return;
  }
  if (C <= kTopkCandCap) {
    block_topk_stream(C, k, [&](uint64_t i) { return ld_cg_u128(cand + i); }, carry, sm);
  } else {
    block_topk_stream(cap, k, [&](uint64_t i) {
      return __ldg(&hits[i]) ? q3_slot_compose(q3_slot_load(ht, i)) : (u128)0;
    }, carry, sm);
  }
  for (int i = t; i < k; i += kTopkThreads) out[i] = carry[i];
}

// Result conversion shared by the single and the batched Q3: payload {u64 groups, u64 pad,
// u128 rows[k]} -> gpudb_q3_result.
void q3_result_from(const uint8_t* h, int k, gpudb_q3_result* out, int join_mode);

// Q3 requests (global-table mode, device-resident lineitem, identical tables) evaluated
// together: every stage is one launch for all of them and the fact table is probed once.
// Returns GPUDB_OK if enqueued; each request's outcome arrives in its status.
constexpr int kQ3Batch = 8;
bool q3_batchable(const gpudb_request& q);
int q3_batch_run(gpudb_ctx* ctx, gpudb_request* reqs, const std::vector<uint32_t>& ids, const gpudb_exec* ex);

// Result payload of every mode: {u64 groups, u64 pad, u128 rows[k]} (rows as top-k
// composites, see topk_compose).
int q3_global(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_lineitem* li,
              const gpudb_q3_params& p, uint8_t* result);
int q3_radix(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_lineitem* li,
             const gpudb_q3_params& p, uint8_t* result);

}  // namespace gpudb
