// Q3-like pipeline: bitmap semi-join filter on the dimension table, filtered hash build
// on orders, probe + per-order aggregation of the fact table, and device top-k.
// Reference: kernels/q3.metal:43-340 (bitmap, direct map / hash table build, fused probe
// + CAS aggregation, compaction), src/q3.cpp:8-538 (driver), src/infra.h:538-564 (CPU
// top-10).
//
// B200 design (global-table mode):
//  1. bitmap_build_kernel: customers with segment == S -> bitmap (warp-combined atomicOr).
//  2. orders_filter_kernel: orders with order_date < D and cust in the bitmap (a shared-memory
//     copy of it when it is at most 48 KB, else tested in place) are compacted (block prefix
//     sum + one atomicAdd per block step) into a staging list; the qualifying
//     count stays on the device.
//  3. table_clear_kernel: sizes the hash table from that count on the device (power of two,
//     <= 50% load) and clears only those slots, so no host round trip is needed.
//  4. orders_insert_kernel: atomicCAS insertion; each slot is {key, date, revenue} and a
//     parallel hit counter, so the orders table doubles as the per-order aggregation table
//     (the group key equals the join key).
//  5. q3_probe_kernel: one lane per fact row; runs of equal order keys (adjacent rows of one
//     order) are found with a warp ballot, only the run head probes the table (after a test
//     of the order-key bitmap that step 4 sets, which turns away most misses), and each row
//     that joins adds its revenue and a count with one atomic each (a few percent of rows).
//     ext_price and discount are loaded only for rows that passed the date filter and found
//     their order (late materialisation); the next step's keys and dates load meanwhile.
//  6. q3_hist_kernel: groups and a log-scale revenue histogram of the live table.
//  7. q3_select_kernel: the slots in the histogram bins that can hold the top-k are
//     appended, and the last block to finish ranks them.
// Radix mode partitions both sides by key hash (radix.cuh) and joins each partition in
// shared memory. The kept orders also set a hashed key set (16 bits per orders row, no key
// range needed), and the fact filter drops the rows whose order key misses it before they
// are compacted and partitioned: a semi-join reduction, so only rows that may join (plus
// about 2% of the others, false positives that the partition join drops) are partitioned.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"
#include "q3.h"
#include "radix.cuh"

namespace gpudb {

namespace {

constexpr int kFilterRows = 4;                 // rows per thread per block step of orders_filter_kernel
constexpr uint32_t kSmemCustWords = 12288;     // customer filters up to 48 KB are copied to shared memory

// Orders with order_date < date_lt whose customer passes the customer filter, compacted into
// (key, date) with a block prefix sum and one atomicAdd per T * 4 rows. SMEM: the filter
// (the exact bitmap, or a hashed one confirmed in `bitmap`) is copied into shared memory, for
// small filters (1024 threads, two blocks per SM); otherwise the exact bitmap is tested in
// place (256 threads, several blocks per SM). The three columns load together and the next
// step's load while this one is tested.
// Where the orders that pass go: (key, date) staging lists (global and radix modes), or in
// direct mode a dense slot per order ({key, date, revenue 0}, hit count 0) whose number the
// direct map omap[key] receives, and the order's bit in the order-key bitmap okbm.
struct FilterOut {
  int32_t* key;
  int32_t* date;
  Q3Slot* slots;
  uint32_t* hits;
  int32_t* omap;
  uint32_t* okbm;
  int32_t key_max;
  uint32_t* kset;       // radix mode: hashed set of the kept order keys (kset_mask + 1 words), or null
  uint32_t kset_mask;
};

// The hashed key set of the radix mode: a power-of-two array of words sized from the orders
// row count (16 bits per row), so it needs no key range. Keys come in blocks of 32: the block
// (key >> 5) is hashed to a word and the key's low 5 bits pick the bit, so the keys of one
// order-clustered run of fact rows share a word (a warp's 128 rows read a few words, not 128
// scattered ones). A fact row whose order key misses the set cannot join; a hit may be a
// false positive (another block hashed to the same word), which the partition join drops.
__device__ __forceinline__ uint32_t kset_word(int32_t key, uint32_t mask) {
  return slot_hash64((uint64_t)((uint32_t)key >> 5)) & mask;
}
__device__ __forceinline__ bool kset_test(const uint32_t* set, uint32_t mask, int32_t key) {
  return (__ldg(set + kset_word(key, mask)) >> ((uint32_t)key & 31u)) & 1u;
}

template <int T, bool SMEM, bool DIRECT>
__global__ void __launch_bounds__(T, SMEM ? 2 : 1) orders_filter_kernel(
    const int32_t* __restrict__ okey, const int32_t* __restrict__ ocust, const int32_t* __restrict__ odate, uint64_t n,
    int32_t date_lt, const uint32_t* __restrict__ bitmap, int32_t cust_max, const uint32_t* __restrict__ filt,
    uint32_t filt_words, bool exact, FilterOut out, uint32_t* count, uint32_t* status) {
  extern __shared__ uint32_t sfilt[];
  __shared__ uint32_t sh[33];
  const uint32_t* f = bitmap;
  if (SMEM) {
    smem_filter_load(filt, filt_words, sfilt);
    f = sfilt;
  }
  const bool ex = SMEM ? exact : true;
  const uint64_t step = (uint64_t)gridDim.x * T * kFilterRows;
  int32_t nkey[kFilterRows], ndate[kFilterRows], ncust[kFilterRows];
  auto fetch = [&](uint64_t b) {
#pragma unroll
    for (int j = 0; j < kFilterRows; j++) {
      const uint64_t i = b + (uint64_t)j * T + threadIdx.x;
      const bool in = i < n;
      ndate[j] = in ? ld_stream(odate + i) : date_lt;
      ncust[j] = in ? ld_stream(ocust + i) : -1;
      nkey[j] = in ? ld_stream(okey + i) : 0;
    }
  };
  uint64_t b = (uint64_t)blockIdx.x * T * kFilterRows;
  fetch(b);
  // whole blocks stay in the loop: block_reserve needs every thread of the block
  for (; b < n; b += step) {
    int32_t key[kFilterRows], date[kFilterRows], cust[kFilterRows];
#pragma unroll
    for (int j = 0; j < kFilterRows; j++) { key[j] = nkey[j]; date[j] = ndate[j]; cust[j] = ncust[j]; }
    fetch(b + step);
    uint32_t ok = 0;
#pragma unroll
    for (int j = 0; j < kFilterRows; j++) ok |= (uint32_t)(date[j] < date_lt && cust[j] >= 0 && cust[j] <= cust_max) << j;
    uint32_t take = smem_filter_mask(f, ex, bitmap, cust, ok);
#pragma unroll
    for (int j = 0; j < kFilterRows; j++)
      if (((take >> j) & 1u) && (key[j] == kEmptyKey || (DIRECT && (key[j] < 0 || key[j] > out.key_max)))) {
        set_status(status, ST_KEY_RANGE);
        take &= ~(1u << j);
      }
    uint32_t pos = block_reserve<T>(__popc(take), count, sh);
#pragma unroll
    for (int j = 0; j < kFilterRows; j++)
      if (take & (1u << j)) {
        if (DIRECT) {
          *reinterpret_cast<ulonglong2*>(out.slots + pos) =
              make_ulonglong2((unsigned long long)(uint32_t)key[j] | ((unsigned long long)(uint32_t)date[j] << 32), 0ull);
          out.hits[pos] = 0;
          out.omap[key[j]] = (int32_t)pos;
        } else {
          out.key[pos] = key[j];
          out.date[pos] = date[j];
        }
        // the order-key bit (direct) or key-set bit (radix), one atomicOr per kept order: about
        // one order in ten is kept, so few lanes of a warp share a word (merging the lanes of
        // a word with __match_any_sync first was slower)
        const uint32_t bit = 1u << ((uint32_t)key[j] & 31u);
        if (DIRECT) {
          if (atomicOr(out.okbm + ((uint32_t)key[j] >> 5), bit) & bit) set_status(status, ST_DUPLICATE);
        } else if (out.kset) {
          atomicOr(out.kset + kset_word(key[j], out.kset_mask), bit);
        }
        pos++;
      }
  }
}

template <int T, bool SMEM, bool DIRECT>
int launch_orders_filter_as(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_q3_params& p,
                            const uint32_t* bitmap, const uint32_t* filt, uint32_t fwords, bool exact,
                            const FilterOut& out, uint32_t* cnt) {
  gpudb_ctx* ctx = call.ctx();
  auto kern = orders_filter_kernel<T, SMEM, DIRECT>;
  const size_t smem = SMEM ? (size_t)fwords * 4 : 0;
  if (SMEM) GPUDB_CUDA(ctx, kernel_smem(ctx, (const void*)kern, smem));
  const int per_sm = kernel_occupancy(ctx, (const void*)kern, T, smem);
  const uint64_t per_block = (uint64_t)T * kFilterRows;
  const unsigned g = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((od.n_rows + per_block - 1) / per_block, (uint64_t)ctx->sm_count * std::max(1, per_sm)));
  GPUDB_LAUNCH(call, kern, g, T, smem, od.order_key, od.cust_key, od.order_date, od.n_rows, p.order_date_lt, bitmap,
               cu.key_max, filt, fwords, exact, out, cnt, call.status());
  return GPUDB_OK;
}

// The orders filter of every join mode, after the customer bitmap: the shared-memory form
// when the customer filter is at most 48 KB (two 1024-thread blocks per SM), else the
// in-place form on the exact bitmap. (With one block per SM, as a larger filter allows, each
// step's block barriers leave the SM idle: the 188 KB filter of 1.5M customers took 213 us
// in shared memory against 115 us in place for 15M orders.)
template <bool DIRECT>
int launch_orders_filter(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_q3_params& p,
                         const uint32_t* bitmap, const FilterOut& out, uint32_t* cnt) {
  if (od.n_rows == 0) return GPUDB_OK;
  if (smem_filter_exact(cu.key_max) && smem_filter_words(cu.key_max) <= kSmemCustWords)
    return launch_orders_filter_as<1024, true, DIRECT>(call, cu, od, p, bitmap, bitmap, smem_filter_words(cu.key_max),
                                                       true, out, cnt);
  return launch_orders_filter_as<256, false, DIRECT>(call, cu, od, p, bitmap, bitmap, 0, true, out, cnt);
}

FilterOut staging_out(int32_t* key, int32_t* date, uint32_t* kset = nullptr, uint32_t kset_mask = 0) {
  return FilterOut{key, date, nullptr, nullptr, nullptr, nullptr, 0, kset, kset_mask};
}

__global__ void table_clear_kernel(const uint32_t* count, uint32_t min_cap, uint32_t max_cap, int shift, uint32_t* cap_out,
                                   Q3Slot* ht, uint32_t* hits) {
  const uint32_t cap = table_capacity(*count, min_cap, max_cap, shift);
  if (blockIdx.x == 0 && threadIdx.x == 0) *cap_out = cap;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += stride) {
    ht[i].key = kEmptyKey;
    ht[i].date = 0;
    ht[i].rev = 0;
    hits[i] = 0;
  }
}

// Also sets bit `key` of the order-key bitmap `okbm` (keys in [0, key_max]); a key outside
// that range turns the bitmap off for this query (okbm_off), so the probe then walks the
// table for every run.
__global__ void orders_insert_kernel(const int32_t* __restrict__ key, const int32_t* __restrict__ date,
                                     const uint32_t* count, const uint32_t* cap_p, Q3Slot* ht, uint32_t* okbm,
                                     int32_t key_max, uint32_t* okbm_off, uint32_t* status) {
  const uint32_t n = *count, cap = *cap_p, mask = cap - 1;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t k = key[i];
    if (okbm) {
      if (k >= 0 && k <= key_max) atomicOr(okbm + ((uint32_t)k >> 5), 1u << ((uint32_t)k & 31u));
      else *okbm_off = 1u;
    }
    uint32_t s = key_slot(k, mask);
    bool done = false;
    for (uint32_t p = 0; p < cap && !done; p++, s = (s + 1) & mask) {
      const int32_t prev = atomicCAS(&ht[s].key, kEmptyKey, k);
      if (prev == kEmptyKey) { ht[s].date = date[i]; done = true; }
      else if (prev == k) { set_status(status, ST_DUPLICATE); done = true; }
    }
    if (!done) set_status(status, ST_CAPACITY);
  }
}


constexpr int kProbeBatches = 4;   // independent 32-row batches per warp step (memory-level parallelism)

__global__ void __launch_bounds__(256) q3_probe_kernel(const int32_t* __restrict__ lkey, const int32_t* __restrict__ lship,
                                                       const int64_t* __restrict__ lext, const int32_t* __restrict__ ldisc,
                                                       uint64_t n, int32_t ship_gt, Q3Slot* ht, uint32_t* hits,
                                                       const uint32_t* cap_p, const uint32_t* __restrict__ okbm,
                                                       int32_t key_max, const uint32_t* okbm_off) {
  const uint32_t cap = *cap_p;
  // order-key bitmap: a run whose key is not in it cannot join (skips the table walk)
  const uint32_t* bm = (okbm && *okbm_off == 0u) ? okbm : nullptr;
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  constexpr int U = kProbeBatches;
  const uint64_t step = warps * 32 * U;
  uint64_t base = ((uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32 * U;
  // the next step's keys and ship dates are loaded while this step is processed
  int32_t nkey[U], nship[U];
#pragma unroll
  for (int u = 0; u < U; u++) {
    const uint64_t row = base + u * 32 + lane;
    nkey[u] = row < n ? ld_stream(lkey + row) : kEmptyKey;
    nship[u] = row < n ? ld_stream(lship + row) : ship_gt;
  }
  for (; base < n; base += step) {
    int32_t key[U];
    bool pass[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      key[u] = nkey[u];
      pass[u] = nship[u] > ship_gt;
      const uint64_t row = base + step + u * 32 + lane;
      nkey[u] = row < n ? ld_stream(lkey + row) : kEmptyKey;
      nship[u] = row < n ? ld_stream(lship + row) : ship_gt;
    }
    int32_t slot[U];
    int my_head[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int32_t prev = __shfl_up_sync(FULL_MASK, key[u], 1);
      const bool head = (lane == 0) || (key[u] != prev);
      const uint32_t heads = __ballot_sync(FULL_MASK, head);
      const uint32_t passm = __ballot_sync(FULL_MASK, pass[u]);
      // run = [head lane, next head); probe once per run that has a passing row
      my_head[u] = 31 - __clz(heads & lanemask_le());
      const uint32_t later = heads & lanemask_gt();
      const uint32_t upto = later ? (1u << (__ffs(later) - 1)) - 1u : 0xFFFFFFFFu;
      slot[u] = -1;
      if (head && (passm & upto & ~((1u << lane) - 1u)) && key[u] != kEmptyKey) {
        const bool maybe = !bm || (key[u] >= 0 && key[u] <= key_max && bitmap_test(bm, key[u]));
        if (maybe) slot[u] = ht_find(ht, cap, key[u]);
      }
    }
    // rows that join add their revenue and count (integer sums: the order does not matter)
#pragma unroll
    for (int u = 0; u < U; u++) {
      slot[u] = __shfl_sync(FULL_MASK, slot[u], my_head[u]);
      if (pass[u] && slot[u] >= 0) {
        const uint64_t row = base + u * 32 + lane;
        const int64_t v = ld_stream(lext + row) * (int64_t)(100 - ld_stream(ldisc + row));
        atomicAdd(&ht[slot[u]].rev, (unsigned long long)v);
        atomicAdd(&hits[slot[u]], 1u);
      }
    }
  }
}

// Hit counts of the dense slots between `count` and the next multiple of 128 (at least 128)
// are zeroed and that capacity is published: the top-k passes read whole 128-slot chunks.
__device__ __forceinline__ void seal_dense_slots(const uint32_t* count, uint32_t* hits, uint32_t* cap_out) {
  const uint32_t c = *count, cap = max(128u, (c + 127u) & ~127u);
  for (uint32_t i = c + threadIdx.x; i < cap; i += blockDim.x) hits[i] = 0;
  if (threadIdx.x == 0) *cap_out = cap;
}

__global__ void q3_seal_kernel(const uint32_t* count, uint32_t* hits, uint32_t* cap_out) {
  seal_dense_slots(count, hits, cap_out);
}

// ---- direct mode ---------------------------------------------------------------------
// The orders filter gave every qualifying order a dense slot and set its bit in the order-key
// bitmap; the direct map omap (order key -> slot) is read only where that bit is set, so it is
// never cleared. Per warp step, kDirectBatches independent 32-row batches go through three
// phases whose loads are all in flight together: run heads (adjacent rows of one order) with
// a passing row read their bitmap word, heads whose bit is set read their slot, and rows that
// join load ext_price/discount and add revenue and a count with one atomic each. The next
// step's keys and ship dates load meanwhile. Block 0 also zeroes the hit counts of the slots
// between the order count and the next multiple of 128 (the top-k passes read whole 128-slot
// chunks) and publishes that capacity.
constexpr int kDirectBatches = 8;

__global__ void __launch_bounds__(256) q3_direct_probe_kernel(
    const int32_t* __restrict__ lkey, const int32_t* __restrict__ lship, const int64_t* __restrict__ lext,
    const int32_t* __restrict__ ldisc, uint64_t n, int32_t ship_gt, const uint32_t* __restrict__ okbm,
    const int32_t* __restrict__ omap, int32_t key_max, Q3Slot* ht, uint32_t* hits, const uint32_t* count,
    uint32_t* cap_out) {
  if (blockIdx.x == 0) seal_dense_slots(count, hits, cap_out);
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  constexpr int U = kDirectBatches;
  const uint64_t step = warps * 32 * U;
  uint64_t base = ((uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32 * U;
  int32_t nkey[U], nship[U];
#pragma unroll
  for (int u = 0; u < U; u++) {
    const uint64_t row = base + u * 32 + lane;
    nkey[u] = row < n ? ld_stream(lkey + row) : kEmptyKey;
    nship[u] = row < n ? ld_stream(lship + row) : ship_gt;
  }
  for (; base < n; base += step) {
    int32_t key[U];
    uint32_t pass = 0, want = 0;
    int head_lane[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      key[u] = nkey[u];
      pass |= (uint32_t)(nship[u] > ship_gt) << u;
      const uint64_t row = base + step + u * 32 + lane;
      nkey[u] = row < n ? ld_stream(lkey + row) : kEmptyKey;
      nship[u] = row < n ? ld_stream(lship + row) : ship_gt;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int32_t prev = __shfl_up_sync(FULL_MASK, key[u], 1);
      const bool head = (lane == 0) || (key[u] != prev);
      const uint32_t heads = __ballot_sync(FULL_MASK, head);
      const uint32_t passm = __ballot_sync(FULL_MASK, (pass >> u) & 1u);
      head_lane[u] = 31 - __clz(heads & lanemask_le());
      const uint32_t later = heads & lanemask_gt();
      const uint32_t upto = later ? (1u << (__ffs(later) - 1)) - 1u : 0xFFFFFFFFu;
      // the run [head, next head) has a passing row and a key the map covers
      if (head && (passm & upto & ~((1u << lane) - 1u)) && key[u] >= 0 && key[u] <= key_max) want |= 1u << u;
    }
    uint32_t word[U];
#pragma unroll
    for (int u = 0; u < U; u++) word[u] = (want >> u & 1u) ? __ldg(okbm + ((uint32_t)key[u] >> 5)) : 0u;
    int32_t slot[U];
#pragma unroll
    for (int u = 0; u < U; u++)
      slot[u] = ((want >> u & 1u) && (word[u] >> ((uint32_t)key[u] & 31u) & 1u)) ? __ldg(omap + key[u]) : -1;
    int64_t ext[U];
    int32_t disc[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      slot[u] = __shfl_sync(FULL_MASK, slot[u], head_lane[u]);
      const uint64_t row = base + u * 32 + lane;
      const bool join = (pass >> u & 1u) && slot[u] >= 0;
      ext[u] = join ? ld_stream(lext + row) : 0;
      disc[u] = join ? ld_stream(ldisc + row) : 0;
    }
#pragma unroll
    for (int u = 0; u < U; u++)
      if ((pass >> u & 1u) && slot[u] >= 0) {
        atomicAdd(&ht[slot[u]].rev, (unsigned long long)(ext[u] * (int64_t)(100 - disc[u])));
        atomicAdd(&hits[slot[u]], 1u);
      }
  }
}

// Quad form of the direct probe, for 16-byte aligned columns: a lane takes kDirectQuads quads
// (4 consecutive rows each: one 16-byte load of keys and one of ship dates per quad). Inside a
// quad, rows of one order are adjacent, so the lane looks up each distinct key among its
// passing rows once (bitmap word, then slot), and rows of equal slot are summed before one
// atomic pair. ext_price / discount of a quad load only when one of its rows joins. The
// kDirectQuads quads' loads are issued phase by phase, all in flight together. Tail rows past
// the last whole quad go one per thread.
constexpr int kDirectQuads = 2;

__global__ void __launch_bounds__(256) q3_direct_quad_kernel(
    const int4* __restrict__ lkey4, const int4* __restrict__ lship4, const longlong2* __restrict__ lext2,
    const int4* __restrict__ ldisc4, uint64_t n, int32_t ship_gt, const uint32_t* __restrict__ okbm,
    const int32_t* __restrict__ omap, int32_t key_max, Q3Slot* ht, uint32_t* hits, const uint32_t* count,
    uint32_t* cap_out) {
  if (blockIdx.x == 0) seal_dense_slots(count, hits, cap_out);
  constexpr int U = kDirectQuads;
  const uint64_t nq = n >> 2;
  const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t q0 = tid; q0 < nq; q0 += U * T) {
    int32_t key[4 * U], ship[4 * U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint64_t q = q0 + u * T;
      const int4 k = q < nq ? ld_stream(lkey4 + q) : make_int4(-1, -1, -1, -1);
      const int4 sh = q < nq ? ld_stream(lship4 + q) : make_int4(ship_gt, ship_gt, ship_gt, ship_gt);
      key[4 * u] = k.x; key[4 * u + 1] = k.y; key[4 * u + 2] = k.z; key[4 * u + 3] = k.w;
      ship[4 * u] = sh.x; ship[4 * u + 1] = sh.y; ship[4 * u + 2] = sh.z; ship[4 * u + 3] = sh.w;
    }
    // rows that look their key up: passing, in range, and a key other than the previous
    // looked-up row's in the quad
    uint32_t want = 0, pass = 0;
#pragma unroll
    for (int u = 0; u < U; u++) {
      int32_t last = INT32_MIN;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = 4 * u + i;
        const bool p = ship[r] > ship_gt && key[r] >= 0 && key[r] <= key_max;
        pass |= (uint32_t)p << r;
        if (p && key[r] != last) { want |= 1u << r; last = key[r]; }
      }
    }
    uint32_t word[4 * U];
#pragma unroll
    for (int r = 0; r < 4 * U; r++) word[r] = (want >> r & 1u) ? __ldg(okbm + ((uint32_t)key[r] >> 5)) : 0u;
    int32_t slot[4 * U];
#pragma unroll
    for (int r = 0; r < 4 * U; r++)
      slot[r] = ((want >> r & 1u) && (word[r] >> ((uint32_t)key[r] & 31u) & 1u)) ? __ldg(omap + key[r]) : -1;
    // rows that did not look up take the slot of the previous row of the quad (same key)
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int i = 1; i < 4; i++) {
        const int r = 4 * u + i;
        if (!(want >> r & 1u)) slot[r] = slot[r - 1];
      }
    uint32_t join = 0;
#pragma unroll
    for (int r = 0; r < 4 * U; r++) join |= (uint32_t)((pass >> r & 1u) && slot[r] >= 0) << r;
    if (!join) continue;
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint32_t jq = (join >> (4 * u)) & 0xFu;
      if (!jq) continue;
      const uint64_t q = q0 + u * T;
      const longlong2 e01 = ld_stream(lext2 + 2 * q), e23 = ld_stream(lext2 + 2 * q + 1);
      const int4 d = ld_stream(ldisc4 + q);
      const int64_t ev[4] = {e01.x, e01.y, e23.x, e23.y};
      const int32_t dv[4] = {d.x, d.y, d.z, d.w};
      unsigned long long acc = 0;
      uint32_t cnt = 0;
      int32_t cur = -1;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = 4 * u + i;
        if (!(jq >> i & 1u)) continue;
        if (slot[r] != cur && cnt) {
          atomicAdd(&ht[cur].rev, acc);
          atomicAdd(&hits[cur], cnt);
          acc = 0;
          cnt = 0;
        }
        cur = slot[r];
        acc += (unsigned long long)(ev[i] * (int64_t)(100 - dv[i]));
        cnt++;
      }
      if (cnt) {
        atomicAdd(&ht[cur].rev, acc);
        atomicAdd(&hits[cur], cnt);
      }
    }
  }
  // rows past the last whole quad (at most 3)
  const uint64_t r = (nq << 2) + tid;
  if (r < n) {
    const int32_t* k1 = reinterpret_cast<const int32_t*>(lkey4);
    const int32_t* s1 = reinterpret_cast<const int32_t*>(lship4);
    const int32_t k = k1[r];
    if (s1[r] > ship_gt && k >= 0 && k <= key_max && bitmap_test(okbm, k)) {
      const int32_t sl = omap[k];
      const int64_t e = reinterpret_cast<const int64_t*>(lext2)[r];
      const int32_t dd = reinterpret_cast<const int32_t*>(ldisc4)[r];
      atomicAdd(&ht[sl].rev, (unsigned long long)(e * (int64_t)(100 - dd)));
      atomicAdd(&hits[sl], 1u);
    }
  }
}

// Top-k of the table: the revenue histogram pass, then the select-and-rank pass
// (q3_table_hist / q3_table_select).
__global__ void __launch_bounds__(kTopkThreads) q3_hist_kernel(const Q3Slot* __restrict__ ht,
                                                               const uint32_t* __restrict__ hits, const uint32_t* cap_p,
                                                               uint32_t* state, unsigned long long* groups) {
  __shared__ uint32_t sh[kRevBins];
  q3_table_hist(ht, hits, *cap_p, state, groups, sh);
}

__global__ void __launch_bounds__(kTopkThreads) q3_select_kernel(const Q3Slot* __restrict__ ht,
                                                                 const uint32_t* __restrict__ hits,
                                                                 const uint32_t* cap_p, int k, uint32_t* state,
                                                                 u128* cand, u128* out) {
  __shared__ u128 sm[kTopkScratch];
  __shared__ u128 carry[GPUDB_Q3_MAX_K];
  q3_table_select(ht, hits, *cap_p, k, state, cand, out, sm, carry);
}

// ---- radix mode ----------------------------------------------------------------------
constexpr int kFactThreads = 256;
constexpr int kFactQuads = 4;   // 16-byte quads of ship dates and keys per thread per block step

// Fact rows that may join: ship_date > ship_gt and the order key in the hashed key set of
// the kept orders, compacted to (order_key, ext * (100 - disc)). A block step covers
// kFactThreads * 16 rows (load q of thread t is quad q * kFactThreads + t of the step, 128-bit
// loads where the columns allow): ship dates and keys load together, then the key-set words
// of the rows whose date passes (all in flight together), then one block_reserve (a single
// atomicAdd on the output count per 4096 rows; one per warp step made the counter the
// bottleneck) and ext/discount only for the rows kept.
__global__ void __launch_bounds__(kFactThreads) q3_fact_filter_kernel(
    const int32_t* __restrict__ lkey, const int32_t* __restrict__ lship, const int64_t* __restrict__ lext,
    const int32_t* __restrict__ ldisc, uint64_t n, int32_t ship_gt, const uint32_t* __restrict__ kset,
    uint32_t kset_mask, int32_t* __restrict__ out_key, int64_t* __restrict__ out_val, uint32_t* count) {
  __shared__ uint32_t sh[33];
  constexpr int R = 4 * kFactQuads;
  constexpr uint64_t kStep = (uint64_t)kFactThreads * R;
  const bool vec = ((reinterpret_cast<uintptr_t>(lkey) | reinterpret_cast<uintptr_t>(lship)) & 15u) == 0;
  auto row_of = [&](uint64_t b, int j) {   // row j (quad j / 4, element j % 4) of this thread
    return b + 4 * ((uint64_t)(j >> 2) * kFactThreads + threadIdx.x) + (j & 3);
  };
  // whole blocks stay in the loop: block_reserve needs every thread of the block
  for (uint64_t b = (uint64_t)blockIdx.x * kStep; b < n; b += (uint64_t)gridDim.x * kStep) {
    int32_t k[R];
    uint32_t on = 0;
    if (vec && b + kStep <= n) {
#pragma unroll
      for (int q = 0; q < kFactQuads; q++) {
        const uint64_t r0 = row_of(b, 4 * q);
        const int4 sv = ld_stream(reinterpret_cast<const int4*>(lship + r0));
        const int4 kv = ld_stream(reinterpret_cast<const int4*>(lkey + r0));
        k[4 * q] = kv.x; k[4 * q + 1] = kv.y; k[4 * q + 2] = kv.z; k[4 * q + 3] = kv.w;
        on |= ((uint32_t)(sv.x > ship_gt) | (uint32_t)(sv.y > ship_gt) << 1 | (uint32_t)(sv.z > ship_gt) << 2 |
               (uint32_t)(sv.w > ship_gt) << 3) << (4 * q);
      }
    } else {
#pragma unroll
      for (int j = 0; j < R; j++) {
        const uint64_t r = row_of(b, j);
        const bool in = r < n;
        k[j] = in ? ld_stream(lkey + r) : 0;
        on |= (uint32_t)(in && ld_stream(lship + r) > ship_gt) << j;
      }
    }
    uint32_t take = 0;
#pragma unroll
    for (int j = 0; j < R; j++) {
      const uint32_t w = ((on >> j) & 1u) ? __ldg(kset + kset_word(k[j], kset_mask)) : 0u;
      take |= ((w >> ((uint32_t)k[j] & 31u)) & 1u) << j;
    }
    uint32_t pos = block_reserve<kFactThreads>(__popc(take), count, sh);
#pragma unroll
    for (int j = 0; j < R; j++)
      if ((take >> j) & 1u) {
        const uint64_t r = row_of(b, j);
        out_key[pos] = k[j];
        out_val[pos] = ld_stream(lext + r) * (int64_t)(100 - ld_stream(ldisc + r));
        pos++;
      }
  }
}

constexpr uint32_t kQ3PartCap = 4096;               // shared slots per partition table
constexpr uint32_t kQ3PartChunk = kQ3PartCap / 2;   // build rows per chunk
constexpr int kQ3PartGroups = 4;                    // 32-row groups a warp loads at once in q3_partition_kernel

constexpr size_t q3_partition_smem() { return (size_t)kQ3PartCap * (8 + 4 + 4 + 4); }

// One block per partition: shared table of the partition's orders (in chunks), probe of its
// fact rows with shared 64-bit atomics, then the chunk's groups (orders with a joined row)
// are appended to the dense slot array (one reservation per block per chunk); the top-k runs
// over the dense slots afterwards, as in the other modes.
__global__ void __launch_bounds__(kTopkThreads) q3_partition_kernel(
    const int32_t* __restrict__ bk, const int32_t* __restrict__ bdate, const uint32_t* __restrict__ boff,
    const int32_t* __restrict__ pk, const int64_t* __restrict__ pval, const uint32_t* __restrict__ poff,
    Q3Slot* __restrict__ dense, uint32_t* __restrict__ dense_hits, uint32_t* dense_count, uint32_t* status) {
  extern __shared__ __align__(16) unsigned char q3p_pool[];
  __shared__ uint32_t sh[33];
  unsigned long long* hrev = reinterpret_cast<unsigned long long*>(q3p_pool);
  int32_t* hkey = reinterpret_cast<int32_t*>(hrev + kQ3PartCap);
  int32_t* hdate = hkey + kQ3PartCap;
  uint32_t* hhit = reinterpret_cast<uint32_t*>(hdate + kQ3PartCap);
  const uint32_t part = blockIdx.x, mask = kQ3PartCap - 1;
  const uint32_t b0 = boff[part], b1 = boff[part + 1], p0 = poff[part], p1 = poff[part + 1];
  constexpr uint32_t kPerThread = kQ3PartCap / kTopkThreads;
  for (uint32_t c0 = b0; c0 < b1; c0 += kQ3PartChunk) {
    const uint32_t c1 = min(c0 + kQ3PartChunk, b1);
    for (uint32_t i = threadIdx.x; i < kQ3PartCap; i += kTopkThreads) { hkey[i] = kEmptyKey; hrev[i] = 0; hhit[i] = 0; }
    __syncthreads();
    for (uint32_t i = c0 + threadIdx.x; i < c1; i += kTopkThreads) {
      const int32_t key = bk[i];
      uint32_t s = key_slot(key, mask);
      for (uint32_t t = 0; t < kQ3PartCap; t++, s = (s + 1) & mask) {
        const int32_t prev = atomicCAS(&hkey[s], kEmptyKey, key);
        if (prev == kEmptyKey) { hdate[s] = bdate[i]; break; }
        if (prev == key) { set_status(status, ST_DUPLICATE); break; }
      }
    }
    __syncthreads();
    // an order's fact rows arrive mostly adjacent (compacted in row order; the partitioning
    // moves a sub-tile's rows of one digit together): whole warps take 32 rows at a time, runs
    // of equal keys are summed across their lanes (segmented shuffle scan) and the last lane of
    // a run probes and adds once for the run. A warp loads kQ3PartGroups groups of 32 rows
    // before it works on the first, so their loads are in flight together.
    const int lane = threadIdx.x & 31;
    for (uint32_t gbase = p0 + (threadIdx.x & ~31u) * kQ3PartGroups; gbase < p1;
         gbase += kTopkThreads * kQ3PartGroups) {
     int32_t gkey[kQ3PartGroups];
     long long gval[kQ3PartGroups];
#pragma unroll
     for (int g = 0; g < kQ3PartGroups; g++) {
       const uint32_t i = gbase + g * 32 + lane;
       gkey[g] = i < p1 ? pk[i] : kEmptyKey;
       gval[g] = i < p1 ? (long long)pval[i] : 0ll;
     }
#pragma unroll
     for (int g = 0; g < kQ3PartGroups; g++) {
      const uint32_t i = gbase + g * 32 + lane;
      const bool valid = i < p1;
      const int32_t key = gkey[g];
      long long v = gval[g];
      uint32_t c = valid ? 1u : 0u;
      const int32_t prev = __shfl_up_sync(FULL_MASK, key, 1);
      const uint32_t heads = __ballot_sync(FULL_MASK, lane == 0 || key != prev);
      const int seg = 31 - __clz(heads & lanemask_le());   // first lane of this lane's run
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const long long ov = __shfl_up_sync(FULL_MASK, v, d);
        const uint32_t oc = __shfl_up_sync(FULL_MASK, c, d);
        if (lane - d >= seg) { v += ov; c += oc; }
      }
      const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
      if (!tail || !valid || key == kEmptyKey) continue;
      uint32_t s = key_slot(key, mask);
      for (uint32_t t = 0; t < kQ3PartCap; t++, s = (s + 1) & mask) {
        const int32_t hk = hkey[s];
        if (hk == key) { atomicAdd(&hrev[s], (unsigned long long)v); atomicAdd(&hhit[s], c); break; }
        if (hk == kEmptyKey) break;
      }
     }
    }
    __syncthreads();
    // append the chunk's groups: thread t owns slots [t * kPerThread, (t + 1) * kPerThread)
    uint32_t mine = 0;
#pragma unroll
    for (uint32_t j = 0; j < kPerThread; j++) mine += hhit[threadIdx.x * kPerThread + j] != 0;
    uint32_t pos = block_reserve<kTopkThreads>(mine, dense_count, sh);
#pragma unroll
    for (uint32_t j = 0; j < kPerThread; j++) {
      const uint32_t s = threadIdx.x * kPerThread + j;
      if (hhit[s]) {
        *reinterpret_cast<ulonglong2*>(dense + pos) =
            make_ulonglong2((unsigned long long)(uint32_t)hkey[s] | ((unsigned long long)(uint32_t)hdate[s] << 32), hrev[s]);
        dense_hits[pos] = hhit[s];
        pos++;
      }
    }
    __syncthreads();
  }
}

}  // namespace

int q3_radix(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_lineitem* li,
             const gpudb_q3_params& p, uint8_t* result) {
  gpudb_ctx* ctx = call.ctx();
  cudaStream_t s = call.stream();
  const uint32_t words = (uint32_t)(cu.key_max >> 5) + 1;
  const uint64_t n_or = std::max<uint64_t>(od.n_rows, 1), n_li = std::max<uint64_t>(li->n_rows, 1);
  // default fan-out: about 16K orders rows per partition (~1.6K after the filters of the
  // default query), and at least 512 partitions so that every SM has some
  const int bits = p.radix_bits > 0 ? std::min(p.radix_bits, (int)kRadixMaxBits)
                 : ctx->radix_bits > 0 ? ctx->radix_bits
                                       : std::min(kRxPassBits, std::max(9, radix_bits_for(od.n_rows, 16384)));
  const uint64_t parts = 1ull << bits;
  // hashed set of the kept order keys: 16 bits per orders row, a power of two of words
  uint64_t kwords = 32;
  while (kwords < n_or / 2 && kwords < (1ull << 28)) kwords <<= 1;
  const uint64_t n_or_a = (n_or + 31) / 32 * 32;   // 128-byte aligned column starts
  void *bitmap, *bstage, *fstage, *count, *bpart, *fpart, *offs, *cand, *kset;
  int rc = scratch(ctx, "q3.bitmap", (size_t)words * 4, &bitmap);
  if (!rc) rc = scratch(ctx, "q3r.kset", (size_t)kwords * 4, &kset);
  if (!rc) rc = scratch(ctx, "q3r.build", n_or_a * 4 * 4 + 256, &bstage);        // key, date, tmp key, tmp date
  if (!rc) rc = scratch(ctx, "q3r.fact", n_li * 12 * 2 + 1024, &fstage);           // key, value, tmp
  if (!rc) rc = scratch(ctx, "q3.count", 256, &count);
  if (!rc) rc = scratch(ctx, "q3r.bpart", n_or_a * 8 + 256, &bpart);
  if (!rc) rc = scratch(ctx, "q3r.fpart", n_li * 12 + 1024, &fpart);
  if (!rc) rc = scratch(ctx, "q3r.offs", (2 * (parts + 1) + 64) * 4, &offs);
  const uint64_t dslots = std::max<uint64_t>(128, (n_or + 127) / 128 * 128);
  void *dense, *dhits, *tstate;
  if (!rc) rc = scratch(ctx, "q3.cand", (size_t)kTopkCandCap * sizeof(u128), &cand);
  if (!rc) rc = scratch(ctx, "q3r.dense", (size_t)dslots * sizeof(Q3Slot), &dense);
  if (!rc) rc = scratch(ctx, "q3r.dhits", (size_t)dslots * 4, &dhits);
  if (!rc) rc = scratch(ctx, "q3.topk", (size_t)kTopkStateWords * 4, &tstate);
  if (rc) return rc;
  uint32_t* cnt = static_cast<uint32_t*>(count);   // [0] orders, [1] fact rows, [2] groups, [3] top-k capacity
  GPUDB_CUDA(ctx, cudaMemsetAsync(bitmap, 0, (size_t)words * 4, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(kset, 0, (size_t)kwords * 4, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(count, 0, 16, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(tstate, 0, (size_t)kTopkStateWords * 4, s));
  const int sms = ctx->sm_count;
  auto grid = [&](uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 16)); };
  uint32_t* ks = static_cast<uint32_t*>(kset);
  const uint32_t kmask = (uint32_t)(kwords - 1);
  int32_t* bkey = static_cast<int32_t*>(bstage);
  int32_t* bdate = bkey + n_or_a;
  int32_t* bkey_t = bdate + n_or_a;
  int32_t* bdate_t = bkey_t + n_or_a;
  int32_t* fkey = static_cast<int32_t*>(fstage);
  int64_t* fval = reinterpret_cast<int64_t*>(static_cast<uint8_t*>(fstage) + ((n_li * 4 + 255) / 256) * 256);
  int32_t* fkey_t = reinterpret_cast<int32_t*>(fval + n_li);
  int64_t* fval_t = reinterpret_cast<int64_t*>(static_cast<uint8_t*>(static_cast<void*>(fkey_t)) + ((n_li * 4 + 255) / 256) * 256);
  int32_t* bk = static_cast<int32_t*>(bpart);
  int32_t* bd = bk + n_or_a;
  int32_t* pk = static_cast<int32_t*>(fpart);
  int64_t* pv = reinterpret_cast<int64_t*>(static_cast<uint8_t*>(fpart) + ((n_li * 4 + 255) / 256) * 256);
  uint32_t* boff = static_cast<uint32_t*>(offs);
  uint32_t* poff = boff + parts + 16;
  if (cu.n_rows)
    GPUDB_LAUNCH(call, bitmap_build_kernel, grid(cu.n_rows), 256, 0, cu.cust_key, cu.segment, p.segment, cu.n_rows,
                 cu.key_max, (uint32_t*)bitmap, call.status());
  if ((rc = launch_orders_filter<false>(call, cu, od, p, (const uint32_t*)bitmap, staging_out(bkey, bdate, ks, kmask), cnt)))
    return rc;
  rc = radix_partition_run<int32_t, false>(call, bkey, bdate, n_or, cnt, bits, bk, bd, boff, bkey_t, bdate_t);
  if (rc) return rc;
  // fact rows that may join, compacted (a few percent of the table), then partitioned
  const int fgrid = (int)std::max<uint64_t>(
      1, std::min<uint64_t>((n_li + kFactThreads * 16 - 1) / (kFactThreads * 16), (uint64_t)sms * 8));
  rc = stream_lineitem(call, li, LI_ORDER | LI_SHIP | LI_EXT | LI_DISC, 0, [&](const gpudb_lineitem& c) {
    if (c.n_rows == 0) return (int)GPUDB_OK;
    GPUDB_LAUNCH(call, q3_fact_filter_kernel, fgrid, kFactThreads, 0, c.order_key, c.ship_date, c.ext_price, c.discount,
                 c.n_rows, p.ship_date_gt, (const uint32_t*)ks, kmask, fkey, fval, cnt + 1);
    return (int)GPUDB_OK;
  });
  if (!rc) rc = radix_partition_run<int64_t, false>(call, fkey, fval, n_li, cnt + 1, bits, pk, pv, poff, fkey_t, fval_t);
  if (rc) return rc;
  u128* cbuf = static_cast<u128*>(cand);
  unsigned long long* groups = reinterpret_cast<unsigned long long*>(result);
  u128* rows = reinterpret_cast<u128*>(result + 16);
  const size_t psmem = q3_partition_smem();
  GPUDB_CUDA(ctx, kernel_smem(ctx, (const void*)q3_partition_kernel, psmem));
  GPUDB_LAUNCH(call, q3_partition_kernel, (unsigned)parts, kTopkThreads, psmem, (const int32_t*)bk, (const int32_t*)bd,
               (const uint32_t*)boff, (const int32_t*)pk, (const int64_t*)pv, (const uint32_t*)poff, (Q3Slot*)dense,
               (uint32_t*)dhits, cnt + 2, call.status());
  GPUDB_LAUNCH(call, q3_seal_kernel, 1, 256, 0, (const uint32_t*)(cnt + 2), (uint32_t*)dhits, cnt + 3);
  uint32_t* ts = static_cast<uint32_t*>(tstate);
  GPUDB_LAUNCH(call, q3_hist_kernel, q3_topk_grid((uint32_t)dslots, ctx->sm_count, 1, 4), kTopkThreads, 0,
               (const Q3Slot*)dense, (const uint32_t*)dhits, (const uint32_t*)(cnt + 3), ts, groups);
  GPUDB_LAUNCH(call, q3_select_kernel, q3_topk_grid((uint32_t)dslots, ctx->sm_count, 1, 2), kTopkThreads, 0,
               (const Q3Slot*)dense, (const uint32_t*)dhits, (const uint32_t*)(cnt + 3), p.k, ts, cbuf, rows);
  return GPUDB_OK;
}

// Direct-map Q3: customer bitmap, the orders filter into dense slots + order-key bitmap +
// direct map, the probe, and the top-k passes over the dense slots. Result payload as in
// q3_global. The orders' key_max bounds the map (od.key_max + 1 int32).
int q3_direct(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_lineitem* li,
              const gpudb_q3_params& p, uint8_t* result) {
  gpudb_ctx* ctx = call.ctx();
  cudaStream_t s = call.stream();
  const uint32_t words = (uint32_t)(cu.key_max >> 5) + 1;
  const uint64_t n_or = od.n_rows;
  const uint64_t slots = std::max<uint64_t>(128, (n_or + 127) / 128 * 128);
  const int32_t key_max = std::max<int32_t>(od.key_max, 0);
  const size_t okbm_bytes = ((size_t)((uint32_t)key_max >> 5) + 1) * 4;
  void *bitmap, *okbm, *omap, *ht, *hits, *count, *tstate, *cand;
  int rc = scratch(ctx, "q3.bitmap", (size_t)words * 4, &bitmap);
  if (!rc) rc = scratch(ctx, "q3.okbm", okbm_bytes, &okbm);
  if (!rc) rc = scratch(ctx, "q3d.map", ((size_t)key_max + 1) * 4, &omap);   // never cleared
  if (!rc) rc = scratch(ctx, "q3d.slots", (size_t)slots * sizeof(Q3Slot), &ht);
  if (!rc) rc = scratch(ctx, "q3d.hits", (size_t)slots * 4, &hits);
  if (!rc) rc = scratch(ctx, "q3.count", 256, &count);
  if (!rc) rc = scratch(ctx, "q3.topk", (size_t)kTopkStateWords * 4, &tstate);
  if (!rc) rc = scratch(ctx, "q3.cand", (size_t)kTopkCandCap * sizeof(u128), &cand);
  if (rc) return rc;
  uint32_t* cnt = static_cast<uint32_t*>(count);   // [0] orders, [1] top-k capacity
  GPUDB_CUDA(ctx, cudaMemsetAsync(bitmap, 0, (size_t)words * 4, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(okbm, 0, okbm_bytes, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(count, 0, 16, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(tstate, 0, (size_t)kTopkStateWords * 4, s));
  const int sms = ctx->sm_count;
  if (cu.n_rows) {
    const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((cu.n_rows + 255) / 256, (uint64_t)sms * 16));
    GPUDB_LAUNCH(call, bitmap_build_kernel, g, 256, 0, cu.cust_key, cu.segment, p.segment, cu.n_rows, cu.key_max,
                 (uint32_t*)bitmap, call.status());
  }
  const FilterOut out{nullptr, nullptr, (Q3Slot*)ht, (uint32_t*)hits, (int32_t*)omap, (uint32_t*)okbm, key_max};
  if ((rc = launch_orders_filter<true>(call, cu, od, p, (const uint32_t*)bitmap, out, cnt))) return rc;
  const uint32_t mask = LI_ORDER | LI_SHIP | LI_EXT | LI_DISC;
  rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) {
    if (c.n_rows == 0) return (int)GPUDB_OK;
    auto a16 = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    if (a16(c.order_key) && a16(c.ship_date) && a16(c.ext_price) && a16(c.discount)) {
      const uint64_t per_block = 256 * 4 * kDirectQuads;
      const unsigned g = (unsigned)std::max<uint64_t>(
          1, std::min<uint64_t>((c.n_rows + per_block - 1) / per_block,
                                (uint64_t)sms * kernel_occupancy(ctx, (const void*)q3_direct_quad_kernel, 256, 0)));
      GPUDB_LAUNCH(call, q3_direct_quad_kernel, g, 256, 0, (const int4*)c.order_key, (const int4*)c.ship_date,
                   (const longlong2*)c.ext_price, (const int4*)c.discount, c.n_rows, p.ship_date_gt,
                   (const uint32_t*)okbm, (const int32_t*)omap, key_max, (Q3Slot*)ht, (uint32_t*)hits,
                   (const uint32_t*)cnt, cnt + 1);
    } else {
      const uint64_t per_block = 256 * kDirectBatches;
      const unsigned g = (unsigned)std::max<uint64_t>(
          1, std::min<uint64_t>((c.n_rows + per_block - 1) / per_block, (uint64_t)sms * 8));
      GPUDB_LAUNCH(call, q3_direct_probe_kernel, g, 256, 0, c.order_key, c.ship_date, c.ext_price, c.discount,
                   c.n_rows, p.ship_date_gt, (const uint32_t*)okbm, (const int32_t*)omap, key_max, (Q3Slot*)ht,
                   (uint32_t*)hits, (const uint32_t*)cnt, cnt + 1);
    }
    return (int)GPUDB_OK;
  });
  if (rc) return rc;
  u128* cbuf = static_cast<u128*>(cand);
  unsigned long long* groups = reinterpret_cast<unsigned long long*>(result);
  u128* rows = reinterpret_cast<u128*>(result + 16);
  uint32_t* ts = static_cast<uint32_t*>(tstate);
  const uint32_t max_cap = (uint32_t)slots;
  GPUDB_LAUNCH(call, q3_hist_kernel, q3_topk_grid(max_cap, sms, 1, 4), kTopkThreads, 0, (const Q3Slot*)ht,
               (const uint32_t*)hits, (const uint32_t*)(cnt + 1), ts, groups);
  GPUDB_LAUNCH(call, q3_select_kernel, q3_topk_grid(max_cap, sms, 1, 2), kTopkThreads, 0, (const Q3Slot*)ht,
               (const uint32_t*)hits, (const uint32_t*)(cnt + 1), p.k, ts, cbuf, rows);
  return GPUDB_OK;
}

// Whether the direct map of the orders' key range fits 30% of the device's memory (the
// reference's choice between its direct map and its hash table, src/q3.cpp:246).
bool q3_direct_fits(gpudb_ctx* ctx, const gpudb_orders& od) {
  if (od.key_max < 0) return false;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  (void)ctx;
  return ((double)od.key_max + 1.0) * 4.0 <= 0.3 * (double)total_b;
}

// Global-table Q3 (steps 1-6 above). Result payload: {u64 groups, u128 rows[k]}.
int q3_global(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_lineitem* li,
              const gpudb_q3_params& p, uint8_t* result) {
  gpudb_ctx* ctx = call.ctx();
  cudaStream_t s = call.stream();
  const uint32_t words = (uint32_t)(cu.key_max >> 5) + 1;
  const uint64_t n_or = od.n_rows;
  uint32_t max_cap = 2048;
  while (max_cap < (n_or << ctx->ht_shift) && max_cap < (1u << 31)) max_cap <<= 1;
  void *bitmap, *stage, *count, *ht, *hits, *cand, *okbm = nullptr;
  // order-key bitmap for the probe's miss test when the orders carry a key bound
  const bool use_okbm = n_or && od.key_max >= 0;
  const size_t okbm_bytes = use_okbm ? ((size_t)((uint32_t)od.key_max >> 5) + 1) * 4 : 0;
  int rc = scratch(ctx, "q3.bitmap", (size_t)words * 4, &bitmap);
  if (!rc && use_okbm) rc = scratch(ctx, "q3.okbm", okbm_bytes, &okbm);
  if (!rc) rc = scratch(ctx, "q3.stage", std::max<size_t>(n_or, 1) * 8, &stage);
  if (!rc) rc = scratch(ctx, "q3.count", 256, &count);
  if (!rc) rc = scratch(ctx, "q3.ht", (size_t)max_cap * sizeof(Q3Slot), &ht);
  if (!rc) rc = scratch(ctx, "q3.hits", (size_t)max_cap * 4, &hits);
  void* tstate;
  if (!rc) rc = scratch(ctx, "q3.topk", (size_t)kTopkStateWords * 4, &tstate);
  if (!rc) rc = scratch(ctx, "q3.cand", (size_t)kTopkCandCap * sizeof(u128), &cand);
  if (rc) return rc;
  uint32_t* cnt = static_cast<uint32_t*>(count);
  uint32_t* cap = cnt + 1;
  GPUDB_CUDA(ctx, cudaMemsetAsync(bitmap, 0, (size_t)words * 4, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(count, 0, 16, s));   // [0] count, [1] capacity, [2] okbm off, [3] ticket
  if (use_okbm) GPUDB_CUDA(ctx, cudaMemsetAsync(okbm, 0, okbm_bytes, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(tstate, 0, (size_t)kTopkStateWords * 4, s));
  const int sms = ctx->sm_count;
  auto grid = [&](uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 16)); };
  if (cu.n_rows)
    GPUDB_LAUNCH(call, bitmap_build_kernel, grid(cu.n_rows), 256, 0, cu.cust_key, cu.segment, p.segment, cu.n_rows,
                 cu.key_max, (uint32_t*)bitmap, call.status());
  int32_t* skey = static_cast<int32_t*>(stage);
  int32_t* sdate = skey + std::max<uint64_t>(n_or, 1);
  if ((rc = launch_orders_filter<false>(call, cu, od, p, (const uint32_t*)bitmap, staging_out(skey, sdate), cnt)))
    return rc;
  GPUDB_LAUNCH(call, table_clear_kernel, grid(max_cap), 256, 0, (const uint32_t*)cnt, 2048u, max_cap, ctx->ht_shift, cap,
               (Q3Slot*)ht, (uint32_t*)hits);
  GPUDB_LAUNCH(call, orders_insert_kernel, grid(n_or / 4), 256, 0, (const int32_t*)skey, (const int32_t*)sdate,
               (const uint32_t*)cnt, (const uint32_t*)cap, (Q3Slot*)ht, (uint32_t*)okbm, od.key_max, cnt + 2,
               call.status());
  const uint32_t mask = LI_ORDER | LI_SHIP | LI_EXT | LI_DISC;
  rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) {
    if (c.n_rows == 0) return (int)GPUDB_OK;
    const unsigned g = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((c.n_rows + 256 * kProbeBatches - 1) / (256 * kProbeBatches), (uint64_t)sms * 8));
    GPUDB_LAUNCH(call, q3_probe_kernel, g, 256, 0, c.order_key, c.ship_date, c.ext_price, c.discount, c.n_rows,
                 p.ship_date_gt, (Q3Slot*)ht, (uint32_t*)hits, (const uint32_t*)cap, (const uint32_t*)okbm, od.key_max,
                 (const uint32_t*)(cnt + 2));
    return (int)GPUDB_OK;
  });
  if (rc) return rc;
  u128* cbuf = static_cast<u128*>(cand);
  unsigned long long* groups = reinterpret_cast<unsigned long long*>(result);
  u128* rows = reinterpret_cast<u128*>(result + 16);
  uint32_t* ts = static_cast<uint32_t*>(tstate);
  GPUDB_LAUNCH(call, q3_hist_kernel, q3_topk_grid(max_cap, sms, 1, 4), kTopkThreads, 0, (const Q3Slot*)ht, (const uint32_t*)hits,
               (const uint32_t*)cap, ts, groups);
  GPUDB_LAUNCH(call, q3_select_kernel, q3_topk_grid(max_cap, sms, 1, 2), kTopkThreads, 0, (const Q3Slot*)ht, (const uint32_t*)hits,
               (const uint32_t*)cap, p.k, ts, cbuf, rows);
  return GPUDB_OK;
}

}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_q3_join_topk(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_orders* od,
                                  const gpudb_lineitem* li, const gpudb_q3_params* p, gpudb_q3_result* out,
                                  gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!cu || !od || !p || !out) return fail(ctx, GPUDB_E_INVALID, "q3: tables, params and result are required");
  if (p->k < 1 || p->k > GPUDB_Q3_MAX_K) return fail(ctx, GPUDB_E_INVALID, "q3: k must be in 1..%d", GPUDB_Q3_MAX_K);
  if (p->join_mode < GPUDB_JOIN_GLOBAL || p->join_mode > GPUDB_JOIN_AUTO)
    return fail(ctx, GPUDB_E_INVALID, "q3: unknown join mode %d", p->join_mode);
  if (cu->n_rows && (!cu->cust_key || !cu->segment)) return fail(ctx, GPUDB_E_INVALID, "q3: customer columns are NULL");
  if (cu->key_max < 0 && cu->n_rows) return fail(ctx, GPUDB_E_INVALID, "q3: customer.key_max is required");
  if (od->n_rows && (!od->order_key || !od->cust_key || !od->order_date))
    return fail(ctx, GPUDB_E_INVALID, "q3: orders columns are NULL");
  if (od->n_rows > (1ull << 30)) return fail(ctx, GPUDB_E_INVALID, "q3: orders larger than 2^30 rows");
  int rc = lineitem_check(ctx, li, LI_ORDER | LI_SHIP | LI_EXT | LI_DISC);
  if (rc) return rc;
  gpudb_customer c = *cu;
  if (c.key_max < 0) c.key_max = 0;
  const gpudb_orders o = *od;
  const gpudb_q3_params pp = *p;
  int mode = pp.join_mode;
  if (mode == GPUDB_JOIN_AUTO)
    mode = ctx->q3_auto_mode >= 0 ? ctx->q3_auto_mode : q3_direct_fits(ctx, o) ? GPUDB_JOIN_DIRECT : GPUDB_JOIN_GLOBAL;
  if (mode == GPUDB_JOIN_DIRECT && o.key_max < 0 && pp.join_mode == GPUDB_JOIN_AUTO) mode = GPUDB_JOIN_GLOBAL;
  if (mode == GPUDB_JOIN_DIRECT && o.n_rows && o.key_max < 0)
    return fail(ctx, GPUDB_E_INVALID, "q3: the direct mode needs orders.key_max");
  Call call(ctx, ex, t);
  const size_t bytes = 16 + (size_t)GPUDB_Q3_MAX_K * sizeof(u128);
  if ((rc = call.begin(bytes))) return rc;
  uint8_t* res = call.result<uint8_t>();
  rc = mode == GPUDB_JOIN_GLOBAL ? q3_global(call, c, o, li, pp, res)
     : mode == GPUDB_JOIN_DIRECT ? q3_direct(call, c, o, li, pp, res)
                                 : q3_radix(call, c, o, li, pp, res);
  if (rc) return rc;
  const int k = pp.k;
  return call.finish(bytes, [out, k, mode](const uint8_t* h) {
    q3_result_from(h, k, out, mode);
    return GPUDB_OK;
  });
}

namespace gpudb {

void q3_result_from(const uint8_t* h, int k, gpudb_q3_result* out, int mode) {
  uint64_t groups;
  std::memcpy(&groups, h, 8);
  out->n_groups = groups;
  out->join_mode = mode;
  out->n_rows = (uint32_t)std::min<uint64_t>(groups, (uint64_t)k);
  for (uint32_t i = 0; i < out->n_rows; i++) {
    u128 c;
    std::memcpy(&c, h + 16 + i * sizeof(u128), sizeof c);
    int64_t rev;
    int32_t date, key;
    topk_decompose(c, &rev, &date, &key);
    out->rows[i].order_key = key;
    out->rows[i].order_date = date;
    out->rows[i].revenue = rev;
  }
}

}  // namespace gpudb
