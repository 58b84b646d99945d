// Building blocks shared by the join pipelines: bitmap semi-join filters, warp-ballot
// compaction, open-addressing hash tables keyed by int32 with atomicCAS insertion, and
// block top-k selection over 128-bit sortable composites.
#pragma once
#include "common.cuh"

namespace gpudb {

constexpr int32_t kEmptyKey = INT32_MIN;   // empty slot marker; INT32_MIN is not a valid key

__device__ __forceinline__ uint32_t lanemask_lt() { uint32_t m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m; }
__device__ __forceinline__ uint32_t lanemask_le() { uint32_t m; asm("mov.u32 %0, %%lanemask_le;" : "=r"(m)); return m; }
__device__ __forceinline__ uint32_t lanemask_gt() { uint32_t m; asm("mov.u32 %0, %%lanemask_gt;" : "=r"(m)); return m; }

// Sets bit `key` for rows whose predicate column equals `value` (value < 0: is nonzero;
// all rows if pred is null). Lanes that hit the same 32-bit word are combined first, so a
// dense key run costs one atomicOr per word instead of one per row. Rows first, first +
// stride, ... (whole warps).
__device__ __forceinline__ void bitmap_build_rows(const int32_t* __restrict__ keys, const uint8_t* __restrict__ pred,
                                                  int32_t value, uint64_t n, int32_t key_max, uint32_t* bitmap,
                                                  uint32_t* status, uint64_t first, uint64_t stride) {
  const uint64_t end = (n + 31) & ~31ull;   // whole warps stay in the loop
  for (uint64_t i = first; i < end; i += stride) {
    bool on = false;
    int32_t key = 0;
    if (i < n) {
      key = keys[i];
      on = pred ? (value >= 0 ? pred[i] == (uint8_t)value : pred[i] != 0) : true;
      if (on && (key < 0 || key > key_max)) { set_status(status, ST_KEY_RANGE); on = false; }
    }
    const uint32_t word = (uint32_t)key >> 5, bit = 1u << ((uint32_t)key & 31u);
    uint32_t pending = __ballot_sync(FULL_MASK, on);
    while (pending) {
      const int leader = __ffs(pending) - 1;
      const uint32_t lw = __shfl_sync(FULL_MASK, word, leader);
      const bool mine = on && word == lw;
      const uint32_t bits = __reduce_or_sync(FULL_MASK, mine ? bit : 0u);
      const uint32_t same = __ballot_sync(FULL_MASK, mine);
      if ((int)(threadIdx.x & 31) == leader) atomicOr(bitmap + lw, bits);
      pending &= ~same;
    }
  }
}

static __global__ void bitmap_build_kernel(const int32_t* __restrict__ keys, const uint8_t* __restrict__ pred, int32_t value,
                                           uint64_t n, int32_t key_max, uint32_t* bitmap, uint32_t* status) {
  bitmap_build_rows(keys, pred, value, n, key_max, bitmap, status, (uint64_t)blockIdx.x * blockDim.x + threadIdx.x,
                    (uint64_t)gridDim.x * blockDim.x);
}

// ---- key filter held in shared memory ------------------------------------------------------
// A fact scan that tests every row's key against a dimension bitmap makes one scattered
// 4-byte load per row; from global memory those are bound by L1/L2 transaction rates (one
// sector each), from shared memory by bank conflicts (a few cycles per warp). The filter is
// the exact bitmap when keys 0..key_max fit kSmemFilterBits bits, else a blocked Bloom filter
// of kSmemFilterWords words: a key maps to one word and three bit positions in it and passes
// when all three are set (one shared-memory load per test; with ~110K keys, the Q9 parts
// that pass at 2M parts, about 1% of the other keys pass too). Its hits are either confirmed
// by the caller with the exact bitmap in global memory, or, where a later step drops a false
// positive by itself, left unconfirmed.
constexpr uint32_t kSmemFilterWords = 51200;   // 200 KB of shared memory
constexpr uint32_t kSmemFilterBits = kSmemFilterWords * 32;

__host__ __device__ inline bool smem_filter_exact(int32_t key_max) {
  return key_max >= 0 && (uint32_t)key_max < kSmemFilterBits;
}
// Words of the filter: the exact bitmap's words, or all kSmemFilterWords.
__host__ __device__ inline uint32_t smem_filter_words(int32_t key_max) {
  return smem_filter_exact(key_max) ? ((uint32_t)key_max >> 5) + 1 : kSmemFilterWords;
}
// The Bloom form's hash of a key: Fibonacci hashing (the key times 2^32 / golden ratio, one
// multiply). Its high bits pick the word (multiplied onto [0, kSmemFilterWords)), the 5-bit
// fields at bits 1, 6 and 11 the three bit positions (each mask bit a funnel shift, whose
// shift count wraps at 32). About 1.3% of keys outside a random 5.5% of 2M keys pass.
__device__ __forceinline__ uint32_t smem_filter_mix(int32_t key) { return (uint32_t)key * 0x9E3779B1u; }
__device__ __forceinline__ uint32_t smem_filter_word(uint32_t h) { return __umulhi(h, kSmemFilterWords); }
__device__ __forceinline__ uint32_t smem_filter_bits(uint32_t h) {
  return __funnelshift_l(0u, 1u, h >> 1) | __funnelshift_l(0u, 1u, h >> 6) | __funnelshift_l(0u, 1u, h >> 11);
}

// Bloom filter of an exact bitmap of `words` words: every set key sets its three bits.
// `filt` holds kSmemFilterWords zeroed words.
static __global__ void hashed_filter_kernel(const uint32_t* __restrict__ bits, uint32_t words, uint32_t* filt) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
    uint32_t x = bits[w];
    while (x) {
      const uint32_t b = __ffs(x) - 1;
      x &= x - 1;
      const uint32_t h = smem_filter_mix((int32_t)(w * 32 + b));
      atomicOr(filt + smem_filter_word(h), smem_filter_bits(h));
    }
  }
}

// Copies `words` filter words into shared memory (whole block; 16-byte copies where the
// source allows) and waits for the block.
__device__ __forceinline__ void smem_filter_load(const uint32_t* __restrict__ src, uint32_t words, uint32_t* dst) {
  if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
    const uint32_t quads = words >> 2;
    for (uint32_t i = threadIdx.x; i < quads; i += blockDim.x)
      reinterpret_cast<uint4*>(dst)[i] = __ldg(reinterpret_cast<const uint4*>(src) + i);
    for (uint32_t i = (quads << 2) + threadIdx.x; i < words; i += blockDim.x) dst[i] = __ldg(src + i);
  } else {
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = __ldg(src + i);
  }
  __syncthreads();
}

// Filter of N keys (ok[j]: key j is in [0, key_max]) -> bit j set where key j passes: the
// shared-memory tests first, then (Bloom form) every confirming load of `bits` issued before
// any is used, so a thread waits for one memory latency, not N.
template <int N>
__device__ __forceinline__ uint32_t smem_filter_mask(const uint32_t* sfilt, bool exact, const uint32_t* bits,
                                                     const int32_t (&key)[N], uint32_t ok) {
  uint32_t hit = 0;
  if (exact) {
#pragma unroll
    for (int j = 0; j < N; j++) {
      // a key outside [0, key_max] reads bit 0 and is masked off (its index would be out of range)
      const uint32_t b = ((ok >> j) & 1u) ? (uint32_t)key[j] : 0u;
      hit |= ((ok >> j) & (sfilt[b >> 5] >> (b & 31u)) & 1u) << j;
    }
    return hit;
  }
#pragma unroll
  for (int j = 0; j < N; j++) {
    const uint32_t h = smem_filter_mix(key[j]), m = smem_filter_bits(h);
    hit |= (uint32_t)(((ok >> j) & 1u) && (sfilt[smem_filter_word(h)] & m) == m) << j;
  }
  if (!hit) return hit;
  uint32_t w[N];
#pragma unroll
  for (int j = 0; j < N; j++) w[j] = ((hit >> j) & 1u) ? __ldg(bits + ((uint32_t)key[j] >> 5)) : 0u;
  uint32_t pass = 0;
#pragma unroll
  for (int j = 0; j < N; j++) pass |= ((w[j] >> ((uint32_t)key[j] & 31u)) & 1u) << j;
  return pass & hit;
}

// Sets bit `key` of `bitmap` for the lanes with `on` (keys already range-checked): one
// atomicOr per distinct word of the warp (lanes of a word found with __match_any_sync, their
// bits merged with a masked OR-reduce). Every lane of the warp calls it.
__device__ __forceinline__ void warp_bitmap_or(bool on, int32_t key, uint32_t* bitmap) {
  const uint32_t onmask = __ballot_sync(FULL_MASK, on);
  if (!on) return;
  const uint32_t word = (uint32_t)key >> 5;
  const uint32_t peers = __match_any_sync(onmask, word);
  const uint32_t bits = __reduce_or_sync(peers, 1u << ((uint32_t)key & 31u));
  if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicOr(bitmap + word, bits);
}

// key -> nation byte for the rows whose nation (0..24) is in `mask`; the map starts at 0xFF
// (the caller clears it). A key outside 0..key_max sets ST_KEY_RANGE. (Q5, Q7, Q8.)
static __global__ void nation_map_kernel(const int32_t* __restrict__ key, const uint8_t* __restrict__ nation,
                                         uint64_t n, int32_t key_max, uint32_t mask, uint8_t* map, uint32_t* status) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const int32_t k = ld_stream(key + i);
    const uint32_t nt = ld_stream(nation + i);
    if (k < 0 || k > key_max) { set_status(status, ST_KEY_RANGE); continue; }
    if (nt < 25u && ((mask >> nt) & 1u)) map[k] = (uint8_t)nt;
  }
}

// Warp-aggregated append: returns this lane's output position (valid where `take`).
__device__ __forceinline__ uint32_t warp_append(bool take, uint32_t* counter) {
  const uint32_t m = __ballot_sync(FULL_MASK, take);
  uint32_t base = 0;
  const int lane = threadIdx.x & 31;
  if (lane == 0 && m) base = atomicAdd(counter, (uint32_t)__popc(m));
  base = __shfl_sync(FULL_MASK, base, 0);
  return base + __popc(m & lanemask_lt());
}

// Block-aggregated reservation: each thread asks for `mine` output positions and gets the
// first of them; the block takes one atomicAdd on `counter`. Every thread of the block must
// call it the same number of times. `sh` needs 33 words of shared memory.
template <int T>
__device__ __forceinline__ uint32_t block_reserve(uint32_t mine, uint32_t* counter, uint32_t* sh) {
  static_assert(T % 32 == 0 && T <= 1024, "block_reserve: whole warps, at most 1024 threads");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = mine;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(FULL_MASK, inc, d);
    if (lane >= d) inc += o;
  }
  if (lane == 31) sh[warp] = inc;
  __syncthreads();
  if (warp == 0) {   // scan of the warp totals, one atomicAdd for the block
    const uint32_t c = lane < T / 32 ? sh[lane] : 0u;
    uint32_t x = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(FULL_MASK, x, d);
      if (lane >= d) x += o;
    }
    const uint32_t total = __shfl_sync(FULL_MASK, x, 31);
    uint32_t base = 0;
    if (lane == 0 && total) base = atomicAdd(counter, total);
    base = __shfl_sync(FULL_MASK, base, 0);
    if (lane < T / 32) sh[lane] = base + x - c;
  }
  __syncthreads();
  const uint32_t pos = sh[warp] + inc - mine;
  __syncthreads();
  return pos;
}

// Open-addressing table capacity from a device-side count: the smallest power of two
// >= count << shift (load at most 1/2^shift), at least `min_cap`, at most `max_cap`.
__device__ __forceinline__ uint32_t table_capacity(uint32_t count, uint32_t min_cap, uint32_t max_cap, int shift = 1) {
  uint64_t want = (uint64_t)count << shift;
  uint32_t cap = min_cap;
  while (cap < want && cap < max_cap) cap <<= 1;
  return cap;
}

__device__ __forceinline__ uint32_t key_slot(int32_t key, uint32_t mask) {
  return slot_hash64((uint32_t)key) & mask;
}

// ---- 128-bit sortable composites for top-k: larger composite = earlier in the output --
// hi = revenue with the sign bit flipped (signed order as unsigned order), lo = (~date, ~key)
// with flipped signs, so larger lo = smaller date, then smaller key.
__host__ __device__ __forceinline__ u128 topk_compose(int64_t rev, int32_t date, int32_t key) {
  const uint64_t hi = (uint64_t)rev ^ 0x8000000000000000ull;
  const uint64_t lo = ((uint64_t)(~((uint32_t)date ^ 0x80000000u)) << 32) | (uint64_t)(~((uint32_t)key ^ 0x80000000u));
  return ((u128)hi << 64) | lo;
}
__host__ __device__ __forceinline__ void topk_decompose(u128 c, int64_t* rev, int32_t* date, int32_t* key) {
  const uint64_t hi = (uint64_t)(c >> 64), lo = (uint64_t)c;
  *rev = (int64_t)(hi ^ 0x8000000000000000ull);
  *date = (int32_t)((~(uint32_t)(lo >> 32)) ^ 0x80000000u);
  *key = (int32_t)((~(uint32_t)lo) ^ 0x80000000u);
}

__device__ __forceinline__ u128 shfl_u128(u128 v, int src) {
  uint64_t lo = __shfl_sync(FULL_MASK, (uint64_t)v, src);
  uint64_t hi = __shfl_sync(FULL_MASK, (uint64_t)(v >> 64), src);
  return ((u128)hi << 64) | lo;
}

constexpr int kTopkThreads = 256;
constexpr int kTopkPerThread = 16;
constexpr int kTopkTile = kTopkThreads * kTopkPerThread;   // 4096 candidates per block

// Block top-k over a tile held as kTopkPerThread composites per thread (0 = no candidate),
// k <= GPUDB_Q3_MAX_K. Writes the k largest composites in descending order (0-padded) to
// out. Method: rank the 256 per-thread maxima; only the k threads whose maxima rank below
// k can hold a top-k element, and only their values >= T (the maximum of rank k-1) can, so
// at most kTopkPerThread*k candidates remain; each candidate's rank among them is its
// output position. Composites of one tile are distinct apart from 0; ties are broken by
// position all the same, so every rank is unique. `sm` is shared scratch of kTopkScratch
// composites.
constexpr int kTopkScratch = kTopkThreads + kTopkPerThread * 64;
__device__ __forceinline__ void block_topk(const u128 (&v)[kTopkPerThread], int k, u128* out, u128* sm) {
  __shared__ uint32_t ncand;
  __shared__ u128 thr;
  u128* mx = sm;
  u128* cand = sm + kTopkThreads;
  const int t = threadIdx.x;
  u128 m = v[0];
#pragma unroll
  for (int j = 1; j < kTopkPerThread; j++) m = v[j] > m ? v[j] : m;
  mx[t] = m;
  if (t == 0) ncand = 0;
  __syncthreads();
  int rank = 0;
#pragma unroll 8
  for (int u = 0; u < kTopkThreads; u++) {
    const u128 o = mx[u];
    rank += (o > m) | ((o == m) & (u < t));
  }
  if (rank == k - 1) thr = m;
  __syncthreads();
  if (rank < k) {
    const u128 T = thr;
#pragma unroll
    for (int j = 0; j < kTopkPerThread; j++)
      if (v[j] != 0 && v[j] >= T) cand[atomicAdd(&ncand, 1u)] = v[j];
  }
  __syncthreads();
  const int C = (int)ncand;
  for (int i = t; i < C; i += kTopkThreads) {
    const u128 c = cand[i];
    int r = 0;
    for (int j = 0; j < C; j++) {
      const u128 o = cand[j];
      r += (o > c) | ((o == c) & (j < i));
    }
    if (r < k) out[r] = c;
  }
  for (int i = C + t; i < k; i += kTopkThreads) out[i] = 0;
  __syncthreads();
}

// Top-k of `n` composites (tiles of kTopkTile per block) -> k per block.
static __global__ void __launch_bounds__(kTopkThreads) topk_merge_kernel(const u128* __restrict__ in, uint64_t n, int k,
                                                                  u128* __restrict__ out) {
  __shared__ u128 wtop[kTopkScratch];
  u128 v[kTopkPerThread];
  const uint64_t base = (uint64_t)blockIdx.x * kTopkTile + (uint64_t)threadIdx.x * kTopkPerThread;
#pragma unroll
  for (int j = 0; j < kTopkPerThread; j++) v[j] = (base + j < n) ? in[base + j] : (u128)0;
  block_topk(v, k, out + (size_t)blockIdx.x * k, wtop);
}

}  // namespace gpudb
