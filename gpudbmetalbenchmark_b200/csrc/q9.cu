// Q9-like star join + (nation, year) aggregate.
// Reference: kernels/q9.metal:44-394 (part filter, supplier direct map, partsupp hash
// table, orders hash table / year map, probe + global CAS aggregation), src/q9.cpp:8-557
// (driver, SF100 streaming), src/infra.h:743-776 (post-processing order).
//
// B200 design:
//  - part filter -> bitmap (bitmap_build_kernel); supplier -> nation and order -> year as
//    uint8 direct maps (100 KB and max_order_key+1 bytes: 60 MB for 15M orders, mostly L2);
//  - partsupp rows whose part passes the bitmap are compacted, then inserted into an
//    open-addressing table keyed by the 64-bit (part, supp) composite with a 64-bit
//    atomicCAS; the table is sized on the device from the qualifying count;
//  - the fact table goes through in pieces of at most 64M rows, two kernels each:
//    li_filter_kernel streams part_key (128-bit loads), tests each part against a filter held
//    in shared memory (the exact bitmap, or a blocked Bloom filter whose ~1.3% false
//    positives the resolve turns away after gathering the part key, with one test of the
//    exact bitmap) and writes a bitmask of the rows that pass (~5.5%); q9_resolve_kernel expands the bitmask a
//    warp at a time (one set bit per lane) and gathers each row's six columns and its
//    lookups together (late materialisation, all resident threads' misses in flight);
//  - aggregation goes to a per-block shared-memory hash table keyed by (nation<<16 | year)
//    (CAS + 64-bit shared atomics); a group that finds no shared slot spills straight to the
//    global open-addressing table, and each block merges its shared table into the global
//    one once at the end (global atomics ~ blocks x groups, not rows);
//  - one block compacts the global table and sorts it by nation asc, year desc.
#include <algorithm>
#include <cstring>
#include <string>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"

namespace gpudb {
namespace {

constexpr uint32_t kGroupEmpty = 0xFFFFFFFFu;
constexpr unsigned long long kPsEmpty = ~0ull;
constexpr uint8_t kNoValue = 0xFF;

struct PsSlot {
  unsigned long long key;   // (uint32 part << 32) | uint32 supp
  long long cost;
};

__device__ __forceinline__ unsigned long long ps_key(int32_t part, int32_t supp) {
  return ((unsigned long long)(uint32_t)part << 32) | (uint32_t)supp;
}

__global__ void map_u8_kernel(const int32_t* __restrict__ keys, const uint8_t* __restrict__ vals, uint64_t n,
                              int32_t key_max, uint8_t* map, uint32_t* status) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t k = keys[i];
    const uint8_t v = vals[i];
    if (k < 0 || k > key_max) { set_status(status, ST_KEY_RANGE); continue; }
    if (v == kNoValue) { set_status(status, ST_DOMAIN); continue; }
    map[k] = v;
  }
}

// order key -> year - 1992, where year = 1992 + order_date / 365. Four rows per thread per
// step, all eight loads issued before any is used.
constexpr int kYearRows = 4;
__global__ void __launch_bounds__(256) year_map_kernel(const int32_t* __restrict__ keys,
                                                       const int32_t* __restrict__ dates, uint64_t n, int32_t key_max,
                                                       uint8_t* map, uint32_t* status) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x * kYearRows;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x * kYearRows + threadIdx.x; b < n; b += step) {
    int32_t k[kYearRows], d[kYearRows];
#pragma unroll
    for (int j = 0; j < kYearRows; j++) {
      const uint64_t i = b + (uint64_t)j * blockDim.x;
      k[j] = i < n ? ld_stream(keys + i) : 0;
      d[j] = i < n ? ld_stream(dates + i) : -1;
    }
#pragma unroll
    for (int j = 0; j < kYearRows; j++) {
      if (b + (uint64_t)j * blockDim.x >= n) break;
      if (k[j] < 0 || k[j] > key_max) { set_status(status, ST_KEY_RANGE); continue; }
      if (d[j] < 0 || d[j] / 365 >= kNoValue) { set_status(status, ST_DOMAIN); continue; }
      map[k[j]] = (uint8_t)(d[j] / 365);
    }
  }
}

constexpr int kPsRows = 4;   // rows per thread per block step of ps_filter_kernel

// Partsupp rows whose part passes the bitmap, compacted (block prefix sum, one atomicAdd
// per 1024 rows).
__global__ void __launch_bounds__(256) ps_filter_kernel(const int32_t* __restrict__ part, uint64_t n,
                                                        const uint32_t* __restrict__ bits, int32_t part_max,
                                                        uint32_t* stage, uint32_t* count) {
  __shared__ uint32_t sh[33];
  const uint64_t step = (uint64_t)gridDim.x * 256 * kPsRows;
  for (uint64_t b = (uint64_t)blockIdx.x * 256 * kPsRows; b < n; b += step) {   // whole blocks
    uint32_t take = 0;
#pragma unroll
    for (int j = 0; j < kPsRows; j++) {
      const uint64_t i = b + (uint64_t)j * 256 + threadIdx.x;
      if (i < n) {
        const int32_t p = part[i];
        take |= (uint32_t)(p >= 0 && p <= part_max && bitmap_test(bits, p)) << j;
      }
    }
    uint32_t pos = block_reserve<256>(__popc(take), count, sh);
#pragma unroll
    for (int j = 0; j < kPsRows; j++)
      if (take & (1u << j)) stage[pos++] = (uint32_t)(b + (uint64_t)j * 256 + threadIdx.x);
  }
}

__global__ void ps_clear_kernel(const uint32_t* count, uint32_t max_cap, int shift, uint32_t* cap_out, PsSlot* ht) {
  const uint32_t cap = table_capacity(*count, 1024, max_cap, shift);
  if (blockIdx.x == 0 && threadIdx.x == 0) *cap_out = cap;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += stride) {
    ht[i].key = kPsEmpty;
    ht[i].cost = 0;
  }
}

__global__ void ps_insert_kernel(const int32_t* __restrict__ part, const int32_t* __restrict__ supp,
                                 const int64_t* __restrict__ cost, const uint32_t* __restrict__ stage,
                                 const uint32_t* count, const uint32_t* cap_p, PsSlot* ht, uint32_t* status) {
  const uint32_t n = *count, cap = *cap_p, mask = cap - 1;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t r = stage[i];
    const int64_t c = cost[r];
    if (c < 0 || c >= (1ll << 32)) { set_status(status, ST_DOMAIN); continue; }
    const unsigned long long k = ps_key(part[r], supp[r]);
    uint32_t s = slot_hash64(k) & mask;
    bool done = false;
    for (uint32_t p = 0; p < cap && !done; p++, s = (s + 1) & mask) {
      const unsigned long long prev = atomicCAS(&ht[s].key, kPsEmpty, k);
      if (prev == kPsEmpty) { ht[s].cost = c; done = true; }
      else if (prev == k) { set_status(status, ST_DUPLICATE); done = true; }
    }
    if (!done) set_status(status, ST_CAPACITY);
  }
}

__device__ __forceinline__ bool ps_find(const PsSlot* ht, uint32_t cap, unsigned long long k, long long* cost) {
  const uint32_t mask = cap - 1;
  uint32_t s = slot_hash64(k) & mask;
  for (uint32_t p = 0; p < cap; p++, s = (s + 1) & mask) {
    const unsigned long long key = __ldg(&ht[s].key);
    if (key == k) { *cost = __ldg(&ht[s].cost); return true; }
    if (key == kPsEmpty) return false;
  }
  return false;
}

__device__ __forceinline__ void global_group_add(uint32_t* gkeys, unsigned long long* gvals, uint32_t gcap,
                                                 uint32_t key, unsigned long long v, uint32_t* status) {
  const uint32_t mask = gcap - 1;
  uint32_t s = slot_hash64(key) & mask;
  for (uint32_t p = 0; p < gcap; p++, s = (s + 1) & mask) {
    const uint32_t prev = atomicCAS(&gkeys[s], kGroupEmpty, key);
    if (prev == kGroupEmpty || prev == key) { atomicAdd(&gvals[s], v); return; }
  }
  set_status(status, ST_CAPACITY);
}

struct Q9Maps {
  const uint32_t* part_bits; int32_t part_max;   // part_bits: exact bitmap to confirm a Bloom filter's hits, or null
  const uint8_t* nation; int32_t supp_max;
  const PsSlot* ps; const uint32_t* ps_cap;
  const uint8_t* year; int32_t order_max;
};

constexpr int kQ9Threads = 256;

constexpr int kLiThreads = 1024;
constexpr int kLiQuads = 4;                  // 128-row groups per warp per block step
constexpr int kLiRows = 4 * kLiQuads;        // fact rows per thread per block step of li_filter_kernel
constexpr uint64_t kQ9Piece = 64ull << 20;   // fact rows per filter + resolve pair (bounds the pair buffer)

// Part filter forms of li_filter_kernel.
enum : int {
  kPartBloom = 0,   // blocked Bloom filter in shared memory (hits confirmed by the resolve)
  kPartExact = 1    // the exact bitmap, all of it in shared memory
};

// Fact rows whose part passes the filter -> bit (r & 31) of passbits[r >> 5] (rows of the
// piece). A block step covers kLiThreads * 16 rows in 128-row groups, four per warp; lane L
// tests rows 32k + L of a group (k = 0..3), loaded by four coalesced 4-byte loads (128 bytes
// a warp each, any alignment), so the vote (__ballot_sync) of the lanes' row-32k tests is the
// bitmask word k itself: one instruction a word, no shuffles, and lane 0 stores the group's
// four words as one 16-byte store. The next step's keys load while this one is tested.
// MODE: kPartExact tests the exact bitmap in shared memory (keys outside [0, part_max] fail);
// kPartBloom a blocked Bloom filter in shared memory, whose word index is in range for any
// key and whose hits (false positives, and keys outside the part range) the resolve
// confirms against the exact bitmap.
template <int MODE>
__global__ void __launch_bounds__(kLiThreads) li_filter_kernel(const int32_t* __restrict__ part, uint64_t n,
                                                               int32_t part_max, const uint32_t* __restrict__ filt,
                                                               uint32_t filt_words, uint32_t* __restrict__ passbits) {
  extern __shared__ uint32_t sfilt[];
  smem_filter_load(filt, filt_words, sfilt);
  const int lane = threadIdx.x & 31;
  constexpr uint64_t kStepRows = (uint64_t)kLiThreads * kLiRows;
  const uint64_t step = (uint64_t)gridDim.x * kStepRows;
  // first row of group g (0..kLiQuads-1) of this warp in the step at b
  auto group_of = [&](uint64_t b, int g) { return b + 128 * ((uint64_t)g * (kLiThreads / 32) + (threadIdx.x >> 5)); };
  int32_t nv[kLiRows];
  auto prefetch = [&](uint64_t b) {
    if (b + kStepRows <= n) {
#pragma unroll
      for (int g = 0; g < kLiQuads; g++)
#pragma unroll
        for (int k = 0; k < 4; k++) nv[4 * g + k] = ld_stream(part + group_of(b, g) + 32 * k + lane);
    }
  };
  uint64_t b = (uint64_t)blockIdx.x * kStepRows;
  prefetch(b);
  for (; b < n; b += step) {   // b is the same for the whole block: every lane votes
    int32_t p[kLiRows];
    const bool full = b + kStepRows <= n;
    if (full) {
#pragma unroll
      for (int j = 0; j < kLiRows; j++) p[j] = nv[j];
    } else {
#pragma unroll
      for (int g = 0; g < kLiQuads; g++)
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint64_t r = group_of(b, g) + 32 * k + lane;
          p[4 * g + k] = r < n ? ld_stream(part + r) : 0;
        }
    }
    prefetch(b + step);
#pragma unroll
    for (int g = 0; g < kLiQuads; g++) {
      const uint64_t r0 = group_of(b, g);
      uint32_t w[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int32_t key = p[4 * g + k];
        bool hit;
        if (MODE == kPartExact) {
          const bool in = (uint32_t)key <= (uint32_t)part_max;
          const uint32_t x = in ? (uint32_t)key : 0u;
          hit = in && ((sfilt[x >> 5] >> (x & 31u)) & 1u);
        } else {
          const uint32_t h = smem_filter_mix(key), m = smem_filter_bits(h);
          hit = (sfilt[smem_filter_word(h)] & m) == m;
        }
        if (!full) hit = hit && r0 + 32 * k + lane < n;
        w[k] = __ballot_sync(FULL_MASK, hit);
      }
      if (lane == 0 && r0 < n) *reinterpret_cast<uint4*>(passbits + (r0 >> 5)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// Position of the k-th (from 0) set bit of w: halving, by the bit counts of the low halves.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t w, uint32_t k) {
  uint32_t pos = 0;
#pragma unroll
  for (uint32_t width = 16; width >= 1; width >>= 1) {
    const uint32_t lo = __popc(w & ((1u << width) - 1u));
    if (k >= lo) { k -= lo; w >>= width; pos += width; }
  }
  return pos;
}

// The rows of the pass bitmask, 1024 rows (32 words) per warp step: the warp counts every
// word's bits, and in rounds of 32 each lane takes one set bit (its word found by a binary
// search over the word counts), so all lanes work whatever the density.
// For each row the five other columns are gathered together, then supplier -> nation,
// order -> year and (part, supp) -> cost; the profit goes to a shared (nation, year) table
// that spills to the global one.
__global__ void __launch_bounds__(kQ9Threads) q9_resolve_kernel(const uint32_t* __restrict__ passbits, uint64_t n,
                                                                 const int32_t* __restrict__ part,
                                                                 const int32_t* __restrict__ supp,
                                                                 const int32_t* __restrict__ order,
                                                                 const int64_t* __restrict__ ext,
                                                                 const int32_t* __restrict__ disc,
                                                                 const int32_t* __restrict__ qty, Q9Maps m,
                                                                 uint32_t* gkeys, unsigned long long* gvals, uint32_t gcap,
                                                                 uint32_t scap, uint32_t* status) {
  extern __shared__ unsigned long long q9_smem[];
  unsigned long long* svals = q9_smem;
  uint32_t* skeys = reinterpret_cast<uint32_t*>(svals + scap);
  for (uint32_t i = threadIdx.x; i < scap; i += blockDim.x) { skeys[i] = kGroupEmpty; svals[i] = 0; }
  __syncthreads();
  const uint32_t ps_cap = *m.ps_cap, smask = scap - 1;
  const int lane = threadIdx.x & 31;
  const uint64_t words = (n + 31) >> 5, groups = (words + 31) >> 5;
  const uint64_t W = (uint64_t)gridDim.x * (blockDim.x >> 5);
  uint32_t bad = 0;
  for (uint64_t g = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < groups; g += W) {
    const uint64_t w = g * 32 + lane;
    const uint32_t word = w < words ? ld_stream(passbits + w) : 0u;
    const uint32_t c = __popc(word);
    uint32_t incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(FULL_MASK, incl, d);
      if (lane >= d) incl += o;
    }
    const uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
    for (uint32_t j0 = 0; j0 < total; j0 += 32) {
      const uint32_t j = j0 + (uint32_t)lane;
      // source lane: the number of lanes whose inclusive count is <= j
      uint32_t src = 0;
#pragma unroll
      for (uint32_t stp = 16; stp >= 1; stp >>= 1)
        if (__shfl_sync(FULL_MASK, incl, src + stp - 1) <= j) src += stp;
      const uint32_t sw = __shfl_sync(FULL_MASK, word, src);
      const uint32_t sx = __shfl_sync(FULL_MASK, incl - c, src);
      if (j >= total) continue;
      const uint64_t r = ((g * 32 + src) << 5) + nth_set_bit(sw, j - sx);
      const int32_t pk = ld_stream(part + r);
      // a Bloom filter's false positive (about 1% of the other parts, or a key outside the
      // part range) stops after one gather and one test of the exact bitmap (L2-resident); the
      // exact filter has tested the range and the bit itself
      if (m.part_bits && ((uint32_t)pk > (uint32_t)m.part_max ||
                          !((__ldg(m.part_bits + ((uint32_t)pk >> 5)) >> ((uint32_t)pk & 31u)) & 1u)))
        continue;
      const int32_t sk = ld_stream(supp + r), o = ld_stream(order + r);
      const int64_t e = ld_stream(ext + r);
      const int32_t d = ld_stream(disc + r), q = ld_stream(qty + r);
      const bool s_ok = sk >= 0 && sk <= m.supp_max, o_ok = o >= 0 && o <= m.order_max;
      const uint8_t nat = s_ok ? __ldg(m.nation + sk) : kNoValue;
      const uint8_t yoff = o_ok ? __ldg(m.year + o) : kNoValue;
      long long cost = 0;
      const bool found = s_ok && ps_find(m.ps, ps_cap, ps_key(pk, sk), &cost);
      if (found && nat != kNoValue && yoff != kNoValue) {
        bad |= ((uint64_t)e >= (1ull << 36)) | ((uint32_t)d > 100u) | ((uint32_t)q >= 65536u);
        const long long profit = e * (int64_t)(100 - d) - cost * (int64_t)q * 100;
        const uint32_t key = ((uint32_t)nat << 16) | (uint32_t)(1992 + yoff);
        uint32_t h = slot_hash64(key) & smask;
        bool done = false;
        for (uint32_t t = 0; t < scap && !done; t++, h = (h + 1) & smask) {
          const uint32_t prev = atomicCAS(&skeys[h], kGroupEmpty, key);
          if (prev == kGroupEmpty || prev == key) { atomicAdd(&svals[h], (unsigned long long)profit); done = true; }
        }
        if (!done) global_group_add(gkeys, gvals, gcap, key, (unsigned long long)profit, status);   // shared table full
      }
    }
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) set_status(status, ST_DOMAIN);
  for (uint32_t i = threadIdx.x; i < scap; i += blockDim.x)
    if (skeys[i] != kGroupEmpty) global_group_add(gkeys, gvals, gcap, skeys[i], svals[i], status);
}

// One block: compact the global table and sort by nation asc, year desc (bitonic, in
// shared memory). out = {u32 n, pad, u64 pad, groups[n] of (nation, year, profit)}.
__global__ void __launch_bounds__(1024) q9_sort_kernel(const uint32_t* __restrict__ gkeys,
                                                       const unsigned long long* __restrict__ gvals, uint32_t gcap,
                                                       uint8_t* out) {
  extern __shared__ unsigned long long sort_smem[];
  unsigned long long* vals = sort_smem;                       // gcap
  uint32_t* keys = reinterpret_cast<uint32_t*>(vals + gcap);  // gcap
  __shared__ uint32_t count;
  if (threadIdx.x == 0) count = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < gcap; i += blockDim.x) {
    const uint32_t k = gkeys[i];
    if (k != kGroupEmpty) {
      const uint32_t pos = atomicAdd(&count, 1u);
      keys[pos] = ((k >> 16) << 16) | (0xFFFFu - (k & 0xFFFFu));   // nation asc, year desc
      vals[pos] = gvals[i];
    }
  }
  __syncthreads();
  const uint32_t n = count;
  uint32_t size = 1;
  while (size < n) size <<= 1;
  for (uint32_t i = n + threadIdx.x; i < size; i += blockDim.x) { keys[i] = 0xFFFFFFFFu; vals[i] = 0; }
  __syncthreads();
  for (uint32_t k = 2; k <= size; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < size; i += blockDim.x) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const bool up = (i & k) == 0;
          if ((keys[i] > keys[l]) == up) {
            uint32_t tk = keys[i]; keys[i] = keys[l]; keys[l] = tk;
            unsigned long long tv = vals[i]; vals[i] = vals[l]; vals[l] = tv;
          }
        }
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) *reinterpret_cast<uint32_t*>(out) = n;
  int32_t* g = reinterpret_cast<int32_t*>(out + 16);
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    g[4 * i + 0] = (int32_t)(keys[i] >> 16);
    g[4 * i + 1] = (int32_t)(0xFFFFu - (keys[i] & 0xFFFFu));
    *reinterpret_cast<long long*>(g + 4 * i + 2) = (long long)vals[i];
  }
}

uint32_t pow2_at_least(uint32_t v, uint32_t lo) {
  uint32_t p = lo;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_q9_star(gpudb_ctx* ctx, const gpudb_part* pa, const gpudb_supplier* su, const gpudb_partsupp* ps,
                             const gpudb_orders* od, const gpudb_lineitem* li, const gpudb_q9_params* p,
                             gpudb_q9_group* out, uint32_t capacity, uint32_t* n_groups, gpudb_timing* t,
                             const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!pa || !su || !ps || !od || !n_groups || (!out && capacity))
    return fail(ctx, GPUDB_E_INVALID, "q9: tables, n_groups and the output are required");
  if (pa->n_rows && (!pa->part_key || !pa->flag || pa->key_max < 0)) return fail(ctx, GPUDB_E_INVALID, "q9: part columns / key_max");
  if (su->n_rows && (!su->supp_key || !su->nation || su->key_max < 0)) return fail(ctx, GPUDB_E_INVALID, "q9: supplier columns / key_max");
  if (ps->n_rows && (!ps->part_key || !ps->supp_key || !ps->supply_cost)) return fail(ctx, GPUDB_E_INVALID, "q9: partsupp columns");
  if (od->n_rows && (!od->order_key || !od->order_date || od->key_max < 0)) return fail(ctx, GPUDB_E_INVALID, "q9: orders columns / key_max");
  if (ps->n_rows > (1ull << 30)) return fail(ctx, GPUDB_E_INVALID, "q9: partsupp larger than 2^30 rows");
  const uint32_t mask = LI_PART | LI_SUPP | LI_ORDER | LI_EXT | LI_DISC | LI_QTY;
  int rc = lineitem_check(ctx, li, mask);
  if (rc) return rc;
  gpudb_q9_params pp{};
  if (p) pp = *p;
  const uint32_t scap = pp.smem_slots ? (uint32_t)pp.smem_slots : (uint32_t)ctx->q9_smem_slots;
  const uint32_t gcap = pp.global_slots ? (uint32_t)pp.global_slots : (uint32_t)ctx->q9_global_slots;
  if ((scap & (scap - 1)) || scap < 32 || scap > 8192) return fail(ctx, GPUDB_E_INVALID, "q9: smem_slots must be a power of two in 32..8192");
  if ((gcap & (gcap - 1)) || gcap < 32 || gcap > 8192) return fail(ctx, GPUDB_E_INVALID, "q9: global_slots must be a power of two in 32..8192");

  Call call(ctx, ex, t);
  const size_t bytes = 16 + (size_t)gcap * 16;
  if ((rc = call.begin(bytes))) return rc;
  cudaStream_t s = call.stream();
  const int32_t part_max = pa->n_rows ? pa->key_max : 0, supp_max = su->n_rows ? su->key_max : 0;
  const int32_t order_max = od->n_rows ? od->key_max : 0;
  const uint32_t words = (uint32_t)(part_max >> 5) + 1;
  const uint32_t ps_max_cap =
      pow2_at_least((uint32_t)std::min<uint64_t>(ps->n_rows << ctx->ht_shift, 1u << 31), 1024);
  void *bits, *nation, *year, *stage, *count, *pst, *groups;
  rc = scratch(ctx, "q9.bits", (size_t)words * 4, &bits);
  if (!rc) rc = scratch(ctx, "q9.nation", (size_t)supp_max + 1, &nation);
  if (!rc) rc = scratch(ctx, "q9.year", (size_t)order_max + 1, &year);
  if (!rc) rc = scratch(ctx, "q9.stage", std::max<size_t>(ps->n_rows, 1) * 4, &stage);
  if (!rc) rc = scratch(ctx, "q9.count", 256, &count);
  if (!rc) rc = scratch(ctx, "q9.ps", (size_t)ps_max_cap * sizeof(PsSlot), &pst);
  if (!rc) rc = scratch(ctx, "q9.groups", (size_t)gcap * 12, &groups);
  // the part filter of li_filter_kernel: the exact bitmap in shared memory, else a Bloom
  // filter built from it. Two exact alternatives for 2M parts were measured slower: the exact
  // bitmap split between shared memory and global memory (121 us against 93 us for the Bloom
  // form: latency-bound on the global lookups for the keys above the shared part), and the
  // exact bitmap split over the shared memory of a 2-CTA cluster, read through distributed
  // shared memory (338 us: random 4-byte reads of the peer's shared memory stall on
  // long_scoreboard and the memory pipes).
  const int filt_mode = smem_filter_exact(part_max) ? kPartExact : kPartBloom;
  const bool filt_exact = filt_mode != kPartBloom;   // no false positives for the resolve to drop
  const uint32_t filt_words = filt_mode == kPartExact ? smem_filter_words(part_max) : kSmemFilterWords;
  void* hfilt = nullptr;
  if (!rc && filt_mode == kPartBloom) rc = scratch(ctx, "q9.partfilter", (size_t)kSmemFilterWords * 4, &hfilt);
  // pass bitmask of one piece of the fact table (rows whose part passed the part filter;
  // chunk_rows, when given, also sets the piece size of a device-resident table)
  const uint64_t piece =
      std::max<uint64_t>(1, std::min<uint64_t>(pp.chunk_rows ? (uint64_t)pp.chunk_rows : li->n_rows, kQ9Piece));
  void* passbits = nullptr;
  // (the filter writes whole 128-row groups: up to three words past (piece + 31) / 32)
  if (!rc) rc = scratch(ctx, "q9.passbits", ((piece + 31) / 32 + 32) * 4, &passbits);
  if (rc) return rc;
  uint32_t* cnt = static_cast<uint32_t*>(count);
  uint32_t* cap = cnt + 1;
  uint32_t* gkeys = reinterpret_cast<uint32_t*>(static_cast<unsigned long long*>(groups) + gcap);
  unsigned long long* gvals = static_cast<unsigned long long*>(groups);
  const size_t probe_smem = (size_t)scap * 12, sort_smem = (size_t)gcap * 12;
  // dynamic + static shared memory may pass the 48 KB default: always opt in (before any capture)
  GPUDB_CUDA(ctx, kernel_smem(ctx, (const void*)q9_resolve_kernel, probe_smem));
  const size_t filt_smem = (size_t)filt_words * 4;
  const void* li_kernel = filt_mode == kPartExact ? (const void*)li_filter_kernel<kPartExact>
                                                   : (const void*)li_filter_kernel<kPartBloom>;
  GPUDB_CUDA(ctx, kernel_smem(ctx, li_kernel, filt_smem));
  const int filter_per_sm = kernel_occupancy(ctx, li_kernel, kLiThreads, filt_smem);
  const int resolve_per_sm = kernel_occupancy(ctx, (const void*)q9_resolve_kernel, kQ9Threads, probe_smem);
  GPUDB_CUDA(ctx, kernel_smem(ctx, (const void*)q9_sort_kernel, sort_smem));
  const int sms = ctx->sm_count;
  auto grid = [&](uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 16)); };
  // Every device operation of the pipeline, in stream order (status and result through
  // call.status()/call.result()).
  // The part bitmap and the fact-row filter of the first piece stay on the call's stream; the
  // supplier and year maps and the partsupp table, which the filter does not need, go on the
  // context's side stream meanwhile, and the first resolve waits for both.
  auto enqueue = [&]() -> int {
    GPUDB_CUDA(ctx, cudaMemsetAsync(bits, 0, (size_t)words * 4, s));
    GPUDB_CUDA(ctx, cudaMemsetAsync(count, 0, 16, s));   // [0] partsupp count, [1] capacity
    GPUDB_CUDA(ctx, cudaMemsetAsync(gvals, 0, (size_t)gcap * 8, s));
    GPUDB_CUDA(ctx, cudaMemsetAsync(gkeys, 0xFF, (size_t)gcap * 4, s));
    if (pa->n_rows)
      GPUDB_LAUNCH(call, bitmap_build_kernel, grid(pa->n_rows), 256, 0, pa->part_key, pa->flag, -1, pa->n_rows,
                   part_max, (uint32_t*)bits, call.status());
    if (!filt_exact) {
      GPUDB_CUDA(ctx, cudaMemsetAsync(hfilt, 0, (size_t)kSmemFilterWords * 4, s));
      GPUDB_LAUNCH(call, hashed_filter_kernel, grid(words), 256, 0, (const uint32_t*)bits, words, (uint32_t*)hfilt);
    }
    int sr = call.side_begin();
    if (sr) return sr;
    const cudaStream_t side = call.stream();
    GPUDB_CUDA(ctx, cudaMemsetAsync(nation, 0xFF, (size_t)supp_max + 1, side));
    GPUDB_CUDA(ctx, cudaMemsetAsync(year, 0xFF, (size_t)order_max + 1, side));
    if (su->n_rows)
      GPUDB_LAUNCH(call, map_u8_kernel, grid(su->n_rows), 256, 0, su->supp_key, su->nation, su->n_rows, supp_max,
                   (uint8_t*)nation, call.status());
    if (od->n_rows)
      GPUDB_LAUNCH(call, year_map_kernel, grid((od->n_rows + kYearRows - 1) / kYearRows), 256, 0, od->order_key,
                   od->order_date, od->n_rows, order_max, (uint8_t*)year, call.status());
    if (ps->n_rows)
      GPUDB_LAUNCH(call, ps_filter_kernel, grid((ps->n_rows + kPsRows - 1) / kPsRows), 256, 0, ps->part_key, ps->n_rows,
                   (const uint32_t*)bits,
                   part_max, (uint32_t*)stage, cnt);
    GPUDB_LAUNCH(call, ps_clear_kernel, grid(ps_max_cap), 256, 0, (const uint32_t*)cnt, ps_max_cap, ctx->ht_shift, cap,
                 (PsSlot*)pst);
    GPUDB_LAUNCH(call, ps_insert_kernel, grid(ps->n_rows), 256, 0, ps->part_key, ps->supp_key, ps->supply_cost,
                 (const uint32_t*)stage, (const uint32_t*)cnt, (const uint32_t*)cap, (PsSlot*)pst, call.status());
    call.side_end();
    bool joined = false;
    const Q9Maps maps{filt_exact ? nullptr : (const uint32_t*)bits, part_max, (const uint8_t*)nation, supp_max, (const PsSlot*)pst,
                      (const uint32_t*)cap, (const uint8_t*)year, order_max};
    int r = stream_lineitem(call, li, mask, pp.chunk_rows, [&](const gpudb_lineitem& c) {
      for (uint64_t off = 0; off < c.n_rows; off += piece) {
        // (the previous piece's resolve is done with the bitmask: stream order)
        const uint64_t n = std::min<uint64_t>(piece, c.n_rows - off);
        const unsigned fg = (unsigned)std::max<uint64_t>(
            1, std::min<uint64_t>((n + kLiThreads * kLiRows - 1) / (kLiThreads * kLiRows),
                                  (uint64_t)sms * std::max(1, filter_per_sm)));
        const uint32_t* fsrc = (const uint32_t*)(filt_exact ? bits : hfilt);
        if (filt_mode == kPartExact)
          GPUDB_LAUNCH(call, li_filter_kernel<kPartExact>, fg, kLiThreads, filt_smem, c.part_key + off, n, part_max,
                       fsrc, filt_words, (uint32_t*)passbits);
        else
          GPUDB_LAUNCH(call, li_filter_kernel<kPartBloom>, fg, kLiThreads, filt_smem, c.part_key + off, n, part_max,
                       fsrc, filt_words, (uint32_t*)passbits);
        if (!joined) {
          const int jr = call.side_join();
          if (jr) return jr;
          joined = true;
        }
        const uint64_t warps_needed = (n + 1023) / 1024;
        const unsigned g = (unsigned)std::max<uint64_t>(
            1, std::min<uint64_t>((warps_needed + kQ9Threads / 32 - 1) / (kQ9Threads / 32),
                                  (uint64_t)sms * std::max(1, resolve_per_sm)));
        GPUDB_LAUNCH(call, q9_resolve_kernel, g, kQ9Threads, probe_smem, (const uint32_t*)passbits, n,
                     c.part_key + off, c.supp_key + off, c.order_key + off, c.ext_price + off, c.discount + off,
                     c.quantity + off, maps, gkeys, gvals, gcap, scap, call.status());
      }
      return (int)GPUDB_OK;
    });
    if (r) return r;
    if (!joined && (r = call.side_join())) return r;
    GPUDB_LAUNCH(call, q9_sort_kernel, 1, 1024, sort_smem, (const uint32_t*)gkeys, (const unsigned long long*)gvals,
                 gcap, call.result<uint8_t>());
    return GPUDB_OK;
  };
  // A device-resident call on the context's stream runs as a CUDA graph: captured the first
  // time its tables and parameters are seen (and again after a scratch buffer moves), then
  // replayed. The graph writes status and groups into a fixed scratch buffer; one copy moves
  // them into this call's result slot.
  const bool graph = ctx->use_graphs && li->location == GPUDB_MEM_DEVICE && s == ctx->stream;
  if (!graph) {
    if ((rc = enqueue())) return rc;
  } else {
    void* gout = nullptr;
    if ((rc = scratch(ctx, "q9.graph_out", kSlotHeader + bytes, &gout))) return rc;
    std::string key = "q9|";
    auto add = [&key](const void* p, size_t n) { key.append(static_cast<const char*>(p), n); };
    add(pa, sizeof *pa); add(su, sizeof *su); add(ps, sizeof *ps); add(od, sizeof *od); add(li, sizeof *li);
    add(&scap, sizeof scap); add(&gcap, sizeof gcap); add(&ctx->ht_shift, sizeof ctx->ht_shift);
    gpudb_ctx::Graph* g = graph_find(ctx, key);
    if (!g) {
      call.redirect(static_cast<uint8_t*>(gout));
      const uint32_t k0 = call.kernels();
      GPUDB_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      cudaError_t me = cudaMemsetAsync(gout, 0, kSlotHeader + bytes, s);
      int er = me == cudaSuccess ? enqueue() : cuda_fail(ctx, me, "cudaMemsetAsync");
      cudaGraph_t cg = nullptr;
      const cudaError_t ee = cudaStreamEndCapture(s, &cg);
      const uint32_t captured = call.kernels() - k0;
      call.uncount_launches(captured);
      cudaGraphExec_t exec = nullptr;
      if (er == GPUDB_OK && ee != cudaSuccess) er = cuda_fail(ctx, ee, "cudaStreamEndCapture");
      if (er == GPUDB_OK) {
        const cudaError_t ie = cudaGraphInstantiate(&exec, cg, 0);
        if (ie != cudaSuccess) er = cuda_fail(ctx, ie, "cudaGraphInstantiate");
      }
      if (cg) cudaGraphDestroy(cg);
      if (er != GPUDB_OK) return er;
      graph_store(ctx, key, exec, captured);
      g = graph_find(ctx, key);
      call.redirect(nullptr);
    }
    GPUDB_CUDA(ctx, cudaGraphLaunch(g->exec, s));
    call.count_launches(g->kernels);
    GPUDB_CUDA(ctx, cudaMemcpyAsync(call.slot_device(), gout, kSlotHeader + bytes, cudaMemcpyDeviceToDevice, s));
  }
  const uint32_t cap_out = capacity;
  const size_t copy = 16 + (size_t)std::min(gcap, capacity) * 16;
  return call.finish(copy, [out, cap_out, n_groups](const uint8_t* h) {
    uint32_t n;
    std::memcpy(&n, h, 4);
    *n_groups = n;
    const uint32_t m = std::min(n, cap_out);
    if (m) std::memcpy(out, h + 16, (size_t)m * sizeof(gpudb_q9_group));
    return GPUDB_OK;
  });
}
