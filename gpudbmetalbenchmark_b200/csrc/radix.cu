// Radix-partitioned joins: the C ABI of the partitioner, all-pairs equi-join and the
// semi-join count. Reference: sf100_radix_* and sf100_partition_join
// (kernels/microbenchmarks.metal:15-156), which the reference never launches.
//
// After both sides are partitioned with the same hash bits (radix.cuh), partition p of the
// build side can only match partition p of the probe side. One block per partition builds
// a shared-memory hash table from the build rows (chunks of at most kChunk rows, so any
// skew is handled by re-probing per chunk) and probes the partition's probe rows against
// it. Output positions come from warp-aggregated atomics on one global counter.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"
#include "micro.h"
#include "radix.cuh"

namespace gpudb {
namespace {

constexpr int kPJThreads = 256;
constexpr uint32_t kPJCap = 4096;          // shared hash-table slots (32 KB)
constexpr uint32_t kChunk = kPJCap / 2;    // build rows per chunk: <= 50% load
constexpr uint64_t kRowsPerPartition = 2048;   // average build rows per partition: one chunk

__device__ __forceinline__ uint32_t pj_slot(int32_t key) { return key_slot(key, kPJCap - 1); }

__device__ __forceinline__ void pj_build(const int32_t* __restrict__ bk, const int32_t* __restrict__ brow, uint32_t c0,
                                         uint32_t c1, int32_t* hkey, int32_t* hrow) {
  for (uint32_t i = threadIdx.x; i < kPJCap; i += kPJThreads) hkey[i] = kEmptyKey;
  __syncthreads();
  for (uint32_t i = c0 + threadIdx.x; i < c1; i += kPJThreads) {
    const int32_t k = bk[i];
    uint32_t s = pj_slot(k);
    // duplicates take their own slots (multi-map); a chunk never fills the table
    for (uint32_t t = 0; t < kPJCap; t++, s = (s + 1) & (kPJCap - 1))
      if (atomicCAS(&hkey[s], kEmptyKey, k) == kEmptyKey) { if (hrow) hrow[s] = brow[i]; break; }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kPJThreads) partition_pairs_kernel(
    const int32_t* __restrict__ bk, const int32_t* __restrict__ brow, const uint32_t* __restrict__ boff,
    const int32_t* __restrict__ pk, const int32_t* __restrict__ prow, const uint32_t* __restrict__ poff,
    int32_t* out_b, int32_t* out_p, uint64_t cap, unsigned long long* count) {
  __shared__ int32_t hkey[kPJCap], hrow[kPJCap];
  const uint32_t part = blockIdx.x;
  const uint32_t b0 = boff[part], b1 = boff[part + 1], p0 = poff[part], p1 = poff[part + 1];
  const int lane = threadIdx.x & 31;
  for (uint32_t c0 = b0; c0 < b1; c0 += kChunk) {
    pj_build(bk, brow, c0, min(c0 + kChunk, b1), hkey, hrow);
    // whole warps walk the probe rows so the warp-aggregated append is uniform
    for (uint32_t base = p0 + (threadIdx.x & ~31u); base < p1; base += kPJThreads) {
      const uint32_t i = base + lane;
      const bool valid = i < p1;
      const int32_t k = valid ? pk[i] : kEmptyKey;
      uint32_t m = 0;
      if (valid && k != kEmptyKey)
        for (uint32_t s = pj_slot(k), t = 0; t < kPJCap && hkey[s] != kEmptyKey; t++, s = (s + 1) & (kPJCap - 1))
          m += hkey[s] == k;
      uint32_t inc = m;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        uint32_t o = __shfl_up_sync(FULL_MASK, inc, d);
        if (lane >= d) inc += o;
      }
      const uint32_t total = __shfl_sync(FULL_MASK, inc, 31);
      unsigned long long start = 0;
      if (lane == 31 && total) start = atomicAdd(count, (unsigned long long)total);
      start = __shfl_sync(FULL_MASK, start, 31);
      unsigned long long pos = start + inc - m;
      if (m) {
        const int32_t r = prow[i];
        for (uint32_t s = pj_slot(k), t = 0; t < kPJCap && hkey[s] != kEmptyKey; t++, s = (s + 1) & (kPJCap - 1))
          if (hkey[s] == k) {
            if (pos < cap) { out_b[pos] = hrow[s]; out_p[pos] = r; }
            pos++;
          }
      }
    }
    __syncthreads();
  }
}

// Semi-join count: probe rows with at least one match. One 1024-thread block per partition
// with a kPCCap-slot shared table (128 KB), so a partition of up to kPCChunk build keys is one
// chunk and one 10-bit pass per side covers 15M build rows. Partitions whose build side needs
// more than one chunk mark matches in `flags` (one byte per partitioned probe row) and count
// them after the last chunk. Each thread keeps kPCRows build or probe keys in flight (the
// kernel waits on those loads otherwise). A key's slot comes from the bits of its partition
// hash above the `pbits` partition bits, so it is independent of the partition.
constexpr int kPCThreads = 1024;
constexpr uint32_t kPCCap = 32768;
constexpr uint32_t kPCChunk = kPCCap / 2;
constexpr uint64_t kCountRowsPerPartition = 15360;   // average build keys per partition (<= kPCChunk with margin)
constexpr int kPCRows = 16;

__device__ __forceinline__ uint32_t pc_slot(int32_t key, int pbits) {
  return (key_hash32(key) >> pbits) & (kPCCap - 1);
}

__global__ void __launch_bounds__(kPCThreads, 1) partition_count_kernel(
    const int32_t* __restrict__ bk, const uint32_t* __restrict__ boff, const int32_t* __restrict__ pk,
    const uint32_t* __restrict__ poff, int pbits, uint8_t* flags, unsigned long long* count) {
  extern __shared__ __align__(16) int32_t pc_key[];
  const uint32_t part = blockIdx.x, mask = kPCCap - 1;
  const uint32_t b0 = boff[part], b1 = boff[part + 1], p0 = poff[part], p1 = poff[part + 1];
  const bool multi = (b1 - b0) > kPCChunk;
  uint32_t c = 0;
  if (multi)
    for (uint32_t i = p0 + threadIdx.x; i < p1; i += kPCThreads) flags[i] = 0;
  for (uint32_t c0 = b0; c0 < b1; c0 += kPCChunk) {
    const uint32_t c1 = min(c0 + kPCChunk, b1);
    for (uint32_t i = threadIdx.x; i < kPCCap / 4; i += kPCThreads)
      reinterpret_cast<int4*>(pc_key)[i] = make_int4(kEmptyKey, kEmptyKey, kEmptyKey, kEmptyKey);
    __syncthreads();
    // duplicates take their own slots; a chunk fills at most half the table
    for (uint32_t i0 = c0 + threadIdx.x; i0 < c1; i0 += kPCRows * kPCThreads) {
      int32_t k[kPCRows];
#pragma unroll
      for (int u = 0; u < kPCRows; u++) {
        const uint32_t i = i0 + u * kPCThreads;
        k[u] = i < c1 ? __ldcs(bk + i) : kEmptyKey;
      }
#pragma unroll
      for (int u = 0; u < kPCRows; u++) {
        if (k[u] == kEmptyKey) continue;   // (an INT32_MIN key marks an empty slot and never matches)
        uint32_t s = pc_slot(k[u], pbits);
        for (uint32_t t = 0; t < kPCCap; t++, s = (s + 1) & mask)
          if (atomicCAS(&pc_key[s], kEmptyKey, k[u]) == kEmptyKey) break;
      }
    }
    __syncthreads();
    for (uint32_t i0 = p0 + threadIdx.x; i0 < p1; i0 += kPCRows * kPCThreads) {
      int32_t k[kPCRows];
#pragma unroll
      for (int u = 0; u < kPCRows; u++) {
        const uint32_t i = i0 + u * kPCThreads;
        k[u] = i < p1 ? __ldcs(pk + i) : kEmptyKey;
      }
      // (probing the kPCRows keys in lockstep rounds was slower: a warp then runs as many
      // rounds as the longest probe chain among its 512 keys)
#pragma unroll
      for (int u = 0; u < kPCRows; u++) {
        bool hit = false;
        if (k[u] != kEmptyKey)
          for (uint32_t s = pc_slot(k[u], pbits), t = 0; t < kPCCap; t++, s = (s + 1) & mask) {
            const int32_t h = pc_key[s];
            if (h == k[u]) { hit = true; break; }
            if (h == kEmptyKey) break;
          }
        if (multi) { if (hit) flags[i0 + u * kPCThreads] = 1; }
        else c += hit;
      }
    }
    __syncthreads();
  }
  if (multi)
    for (uint32_t i = p0 + threadIdx.x; i < p1; i += kPCThreads) c += flags[i];
  c = __reduce_add_sync(FULL_MASK, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

struct Sides {
  int32_t *bk, *brow, *pk, *prow;   // rows: null when only keys are partitioned
  uint32_t *boff, *poff;
};

// Partitions both sides with `bits` bits into scratch buffers: keys only, or keys with
// their row ids as payload.
int partition_both(Call& call, const int32_t* build, uint64_t nb, const int32_t* probe, uint64_t np, int bits,
                   bool rows, Sides* s) {
  gpudb_ctx* ctx = call.ctx();
  const uint64_t parts = 1ull << bits;
  const size_t nmax = std::max<uint64_t>(std::max(nb, np), 1);
  const int k = rows ? 2 : 1;
  void *keys, *offs;
  int rc = scratch(ctx, "rjoin.keys", (size_t)k * (nb + np + nmax + 3 * 48) * sizeof(int32_t), &keys);
  if (!rc) rc = scratch(ctx, "rjoin.offs", (2 * (parts + 1) + 64) * sizeof(uint32_t), &offs);
  if (rc) return rc;
  int32_t* p = static_cast<int32_t*>(keys);
  auto take = [&p](uint64_t n) { int32_t* q = p; p += (n + 16 + 31) / 32 * 32; return q; };   // 128-byte aligned
  s->bk = take(nb);
  s->pk = take(np);
  int32_t* ktmp = take(nmax);
  s->brow = rows ? take(nb) : nullptr;
  s->prow = rows ? take(np) : nullptr;
  int32_t* ptmp = rows ? take(nmax) : nullptr;
  s->boff = static_cast<uint32_t*>(offs);
  s->poff = s->boff + parts + 16;
  if (rows) {
    rc = radix_partition_run<int32_t, false>(call, build, nullptr, nb, nullptr, bits, s->bk, s->brow, s->boff, ktmp, ptmp);
    if (!rc) rc = radix_partition_run<int32_t, false>(call, probe, nullptr, np, nullptr, bits, s->pk, s->prow, s->poff, ktmp, ptmp);
  } else {
    rc = radix_partition_keys(call, build, nb, bits, s->bk, s->boff, ktmp);
    if (!rc) rc = radix_partition_keys(call, probe, np, bits, s->pk, s->poff, ktmp);
  }
  return rc;
}

}  // namespace

int radix_join_count(Call& call, const int32_t* build_keys, uint64_t n_build, const int32_t* probe_keys, uint64_t n_probe,
                     unsigned long long* count) {
  if (n_build == 0 || n_probe == 0) return GPUDB_OK;
  const int bits = radix_bits_for(n_build, kCountRowsPerPartition);
  Sides s;
  int rc = partition_both(call, build_keys, n_build, probe_keys, n_probe, bits, false, &s);
  if (rc) return rc;
  void* flags = nullptr;
  rc = scratch(call.ctx(), "rjoin.flags", n_probe + 16, &flags);
  if (rc) return rc;
  const size_t smem = kPCCap * sizeof(int32_t);
  GPUDB_CUDA(call.ctx(), kernel_smem(call.ctx(), (const void*)partition_count_kernel, smem));
  GPUDB_LAUNCH(call, partition_count_kernel, 1u << bits, kPCThreads, smem, (const int32_t*)s.bk, (const uint32_t*)s.boff,
               (const int32_t*)s.pk, (const uint32_t*)s.poff, bits, (uint8_t*)flags, count);
  return GPUDB_OK;
}

}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_radix_partition(gpudb_ctx* ctx, const int32_t* keys, const int32_t* payload, uint64_t n,
                                     int32_t bits, int32_t* keys_out, int32_t* payload_out, uint32_t* offsets,
                                     gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (bits < 0 || bits > kRadixMaxBits) return fail(ctx, GPUDB_E_INVALID, "radix: bits must be in 0..%d", kRadixMaxBits);
  if (!offsets || !keys_out || !payload_out || (n && !keys)) return fail(ctx, GPUDB_E_INVALID, "radix: NULL buffer");
  if (n >= (1ull << 32)) return fail(ctx, GPUDB_E_INVALID, "radix: at most 2^32-1 rows");
  Call call(ctx, ex, t);
  int rc = call.begin(16);
  if (rc) return rc;
  void* tmp = nullptr;
  rc = scratch(ctx, "radix.tmp", (2 * std::max<uint64_t>(n, 1) + 96) * sizeof(int32_t), &tmp);
  if (rc) return rc;
  int32_t* ktmp = static_cast<int32_t*>(tmp);
  int32_t* ptmp = ktmp + (std::max<uint64_t>(n, 1) + 16 + 31) / 32 * 32;   // 128-byte aligned
  rc = radix_partition_run<int32_t, true>(call, keys, payload, n, nullptr, bits, keys_out, payload_out, offsets, ktmp, ptmp);
  if (rc) return rc;
  return call.finish(16, [](const uint8_t*) { return GPUDB_OK; });
}

extern "C" int gpudb_radix_join_pairs(gpudb_ctx* ctx, const int32_t* build_keys, uint64_t n_build,
                                      const int32_t* probe_keys, uint64_t n_probe, int32_t* out_build_rows,
                                      int32_t* out_probe_rows, uint64_t capacity, uint64_t* n_pairs, gpudb_timing* t,
                                      const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!n_pairs || (n_build && !build_keys) || (n_probe && !probe_keys) ||
      (capacity && (!out_build_rows || !out_probe_rows)))
    return fail(ctx, GPUDB_E_INVALID, "radix join: NULL buffer");
  if (n_build >= (1ull << 31) || n_probe >= (1ull << 31)) return fail(ctx, GPUDB_E_INVALID, "radix join: at most 2^31-1 rows a side");
  Call call(ctx, ex, t);
  int rc = call.begin(16);
  if (rc) return rc;
  if (n_build && n_probe) {
    const int bits = radix_bits_for(n_build, kRowsPerPartition);
    Sides s;
    rc = partition_both(call, build_keys, n_build, probe_keys, n_probe, bits, true, &s);
    if (rc) return rc;
    GPUDB_LAUNCH(call, partition_pairs_kernel, 1u << bits, kPJThreads, 0, (const int32_t*)s.bk, (const int32_t*)s.brow,
                 (const uint32_t*)s.boff, (const int32_t*)s.pk, (const int32_t*)s.prow, (const uint32_t*)s.poff,
                 out_build_rows, out_probe_rows, capacity, call.result<unsigned long long>());
  }
  return call.finish(16, [n_pairs](const uint8_t* h) {
    std::memcpy(n_pairs, h, 8);
    return GPUDB_OK;
  });
}
