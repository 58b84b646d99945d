// Fused filter + aggregate scans over the lineitem columns:
//   Q6-like filtered global sum   (reference: kernels/q6.metal:12-70, src/q6.cpp:8-214)
//   Q1-like 6-group aggregate     (reference: kernels/q1.metal:39-243, src/q1.cpp:8-376)
//
// B200 design. Both kernels are HBM-bound streams: each thread walks "quads" of 4
// consecutive rows with 128-bit loads of every 4-byte column (one int4 = 4 rows) and two
// 128-bit loads of the 8-byte ext_price column, grid-strided so that a warp reads 512
// contiguous bytes per 4-byte column per step; loads use the streaming cache hint. Rows
// that fail the Q6 predicate never load ext_price (late materialisation). Per-thread
// accumulators live in registers; the block reduces them with warp shuffles, writes one
// partial per block, and the last block to finish folds the partials (one launch, no
// second-stage kernel, no atomics on the result, deterministic). Results accumulate into
// the output (+=) so a streamed table is one launch per chunk on the same output; a
// one-launch call on device-resident columns instead passes `hstatus` (its pinned host
// slot's status word, mapped) and the last block overwrites the output there, so the call
// needs no clear of its slot before the kernel and no copy back after it.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "scans.h"
#include "tma.cuh"

namespace gpudb {
namespace {

constexpr int kThreads = 256;

// ------------------------------------------------------------------------------------
// Q6
// ------------------------------------------------------------------------------------
struct Q6P { int32_t lo, hi, dlo, dhi, qlt; };

__device__ __forceinline__ bool q6_pass(int32_t s, int32_t d, int32_t q, const Q6P& p) {
  return (s >= p.lo) & (s < p.hi) & (d >= p.dlo) & (d <= p.dhi) & (q < p.qlt);
}

struct Q6Out { int64_t revenue; uint64_t matched; };

template <int T>
__device__ __forceinline__ void block_fold_q6(int64_t rev, uint64_t cnt, int64_t* part_rev, uint64_t* part_cnt,
                                              unsigned* ticket, Q6Out* out, uint32_t* hstatus) {
  __shared__ uint64_t sr[T / 32], sc[T / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t r = warp_sum_u64((uint64_t)rev), c = warp_sum_u64(cnt);
  if (lane == 0) { sr[warp] = r; sc[warp] = c; }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t a = 0, b = 0;
    for (int w = 0; w < T / 32; w++) { a += sr[w]; b += sc[w]; }
    part_rev[blockIdx.x] = (int64_t)a;
    part_cnt[blockIdx.x] = b;
  }
  if (!grid_last_block(ticket)) return;
  uint64_t a = 0, b = 0;
  for (unsigned i = threadIdx.x; i < gridDim.x; i += T) {
    a += (uint64_t)__ldcg(part_rev + i);
    b += __ldcg(part_cnt + i);
  }
  a = warp_sum_u64(a);
  b = warp_sum_u64(b);
  __syncthreads();
  if (lane == 0) { sr[warp] = a; sc[warp] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t ta = 0, tb = 0;
    for (int w = 0; w < T / 32; w++) { ta += sr[w]; tb += sc[w]; }
    if (hstatus) {   // one launch, the host slot: overwrite (the Q6 scan sets no status bits)
      out->revenue = (int64_t)ta;
      out->matched = tb;
      *hstatus = 0u;
    } else {
      out->revenue += (int64_t)ta;
      out->matched += tb;
    }
  }
}

template <int UNROLL>
__global__ void __launch_bounds__(kThreads) q6_vec_kernel(const int4* __restrict__ ship4, const int4* __restrict__ disc4,
                                                          const int4* __restrict__ qty4, const int64_t* __restrict__ ext,
                                                          uint64_t n, Q6P p, int64_t* part_rev, uint64_t* part_cnt,
                                                          unsigned* ticket, Q6Out* out, uint32_t* hstatus) {
  const uint64_t nq = n >> 2;
  const uint64_t T = (uint64_t)gridDim.x * kThreads;
  uint64_t q = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  int64_t rev = 0;
  uint32_t cnt = 0;
#define Q6_ROW(c, j)                                                      \
  if (q6_pass(s.c, d.c, k.c, p)) {                                        \
    rev += ld_stream(ext + 4 * qq + (j)) * (int64_t)d.c;                  \
    cnt++;                                                                \
  }
  for (; q + (UNROLL - 1) * T < nq; q += UNROLL * T) {
    int4 sv[UNROLL], dv[UNROLL], kv[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; u++) {
      sv[u] = ld_stream(ship4 + q + u * T);
      dv[u] = ld_stream(disc4 + q + u * T);
      kv[u] = ld_stream(qty4 + q + u * T);
    }
#pragma unroll
    for (int u = 0; u < UNROLL; u++) {
      const uint64_t qq = q + u * T;
      const int4 s = sv[u], d = dv[u], k = kv[u];
      Q6_ROW(x, 0) Q6_ROW(y, 1) Q6_ROW(z, 2) Q6_ROW(w, 3)
    }
  }
  for (; q < nq; q += T) {
    const uint64_t qq = q;
    const int4 s = ld_stream(ship4 + q), d = ld_stream(disc4 + q), k = ld_stream(qty4 + q);
    Q6_ROW(x, 0) Q6_ROW(y, 1) Q6_ROW(z, 2) Q6_ROW(w, 3)
  }
#undef Q6_ROW
  // 0..3 tail rows
  const uint64_t r = (nq << 2) + (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  if (r < n) {
    const int32_t* ship = reinterpret_cast<const int32_t*>(ship4);
    const int32_t* disc = reinterpret_cast<const int32_t*>(disc4);
    const int32_t* qty = reinterpret_cast<const int32_t*>(qty4);
    if (q6_pass(ship[r], disc[r], qty[r], p)) { rev += ext[r] * (int64_t)disc[r]; cnt++; }
  }
  block_fold_q6<kThreads>(rev, cnt, part_rev, part_cnt, ticket, out, hstatus);
}

// Any alignment: one row per thread per step.
__global__ void __launch_bounds__(kThreads) q6_row_kernel(const int32_t* ship, const int32_t* disc, const int32_t* qty,
                                                          const int64_t* ext, uint64_t n, Q6P p, int64_t* part_rev,
                                                          uint64_t* part_cnt, unsigned* ticket, Q6Out* out,
                                                          uint32_t* hstatus) {
  const uint64_t T = (uint64_t)gridDim.x * kThreads;
  int64_t rev = 0;
  uint32_t cnt = 0;
  for (uint64_t r = (uint64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += T)
    if (q6_pass(ship[r], disc[r], qty[r], p)) { rev += ext[r] * (int64_t)disc[r]; cnt++; }
  block_fold_q6<kThreads>(rev, cnt, part_rev, part_cnt, ticket, out, hstatus);
}

// ------------------------------------------------------------------------------------
// Q1
// ------------------------------------------------------------------------------------
// Exact-arithmetic domain (checked per qualifying row, ST_DOMAIN otherwise):
//   0 <= quantity < 2^16, 0 <= discount <= 100, 0 <= tax <= 100, 0 <= ext_price < 2^36,
//   and at most kQ1RowsPerThread rows per thread (enforced by the grid size).
// Per thread and group the kernel keeps four uint64 registers:
//   P   = sum(quantity << 32 | discount << 13 | 1)     (qty 28 bits, disc 19, count 13)
//   E   = sum(ext)          ED = sum(ext * disc)         EDT = sum(ext * (100 - disc) * tax)
// and derives sum_disc_price = 100 E - ED, sum_charge = 100 sum_disc_price + EDT in int128.
constexpr uint32_t kQ1RowsPerThread = 4000;
constexpr int kQ1Metrics = 6;          // count, qty, base, disc_price, charge, discount
constexpr int kQ1Raw = 6;              // count, qty, E, ED, EDT, dsum

struct Q1Acc {
  uint64_t P[6], E[6], ED[6], EDT[6];
  uint32_t bad;
};

__device__ __forceinline__ void q1_row(Q1Acc& a, int32_t s, int32_t qt, int64_t e, int32_t d, int32_t t, uint32_t f,
                                       uint32_t st, int32_t ship_le) {
  const bool pass = (s <= ship_le) & (f <= 2u) & (st <= 1u);
  const uint32_t g = pass ? f * 2u + st : 7u;
  a.bad |= pass & (((uint32_t)qt >= 65536u) | ((uint32_t)d > 100u) | ((uint32_t)t > 100u) |
                   ((uint64_t)e >= (1ull << 36)));
  const uint64_t ed = (uint64_t)e * (uint32_t)d;
  const uint64_t edt = ((uint64_t)e * 100u - ed) * (uint32_t)t;
  const uint64_t pk = ((uint64_t)(uint32_t)qt << 32) | ((uint64_t)(uint32_t)d << 13) | 1u;
  // Exactly one group takes the row. Predicated adds (no branch): a data-dependent `if`
  // per group compiles to divergent branches that stall on branch resolution.
#pragma unroll
  for (int k = 0; k < 6; k++) {
    asm("{\n\t.reg .pred p;\n\t"
        "setp.eq.u32 p, %4, %5;\n\t"
        "@p add.u64 %0, %0, %6;\n\t"
        "@p add.u64 %1, %1, %7;\n\t"
        "@p add.u64 %2, %2, %8;\n\t"
        "@p add.u64 %3, %3, %9;\n\t}"
        : "+l"(a.P[k]), "+l"(a.E[k]), "+l"(a.ED[k]), "+l"(a.EDT[k])
        : "r"(g), "r"((uint32_t)k), "l"(pk), "l"((uint64_t)e), "l"(ed), "l"(edt));
  }
}

template <int T>
__device__ __forceinline__ void q1_fold(Q1Acc& a, u128* partials, unsigned* ticket, u128* out, uint32_t* status) {
  __shared__ u128 red[T / 32][6 * kQ1Raw];
  __shared__ u128 tot[6 * kQ1Raw];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (__syncthreads_or(a.bad) && threadIdx.x == 0) set_status(status, ST_DOMAIN);
#pragma unroll
  for (int g = 0; g < 6; g++) {
    u128 v[kQ1Raw] = {a.P[g] & 0x1FFFu, a.P[g] >> 32, a.E[g], a.ED[g], a.EDT[g], (a.P[g] >> 13) & 0x7FFFFu};
#pragma unroll
    for (int m = 0; m < kQ1Raw; m++) {
      u128 w = warp_sum_u128(v[m]);
      if (lane == 0) red[warp][g * kQ1Raw + m] = w;
    }
  }
  __syncthreads();
  if (threadIdx.x < 6 * kQ1Raw) {
    u128 s = 0;
    for (int w = 0; w < T / 32; w++) s += red[w][threadIdx.x];
    partials[(size_t)blockIdx.x * 6 * kQ1Raw + threadIdx.x] = s;
  }
  if (!grid_last_block(ticket)) return;
  // the last block folds every block's partials: thread t sums metric t % 36 over the blocks
  // b = t / 36, t / 36 + kLanes, ... (all threads, independent loads in flight), then the
  // kLanes sums per metric are added up in shared memory (reusing `red`)
  constexpr int kMetrics = 6 * kQ1Raw;
  constexpr int kLanes = T / kMetrics;
  static_assert(kLanes >= 1 && kLanes <= T / 32, "fold lanes fit the reduction buffer");
  u128* fold = &red[0][0];
  __syncthreads();
  if (threadIdx.x < kLanes * kMetrics) {
    const int m = threadIdx.x % kMetrics, l = threadIdx.x / kMetrics;
    const uint64_t* pp = reinterpret_cast<const uint64_t*>(partials);
    u128 s = 0;
#pragma unroll 4
    for (unsigned b = l; b < gridDim.x; b += kLanes) {
      const size_t i = ((size_t)b * kMetrics + m) * 2;
      s += ((u128)__ldcg(pp + i + 1) << 64) | __ldcg(pp + i);
    }
    fold[l * kMetrics + m] = s;
  }
  __syncthreads();
  if (threadIdx.x < kMetrics) {
    u128 s = 0;
    for (int l = 0; l < kLanes; l++) s += fold[l * kMetrics + threadIdx.x];
    tot[threadIdx.x] = s;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    const int g = threadIdx.x;
    const u128* r = tot + g * kQ1Raw;
    const u128 disc_price = (u128)100 * r[2] - r[3];
    const u128 charge = (u128)100 * disc_price + r[4];
    u128* o = out + g * kQ1Metrics;
    o[0] += r[0];
    o[1] += r[1];
    o[2] += r[2];
    o[3] += disc_price;
    o[4] += charge;
    o[5] += r[5];
  }
}

// The shared-memory form's grid accumulators: kQ1AccCopies copies (block b adds into copy
// b % kQ1AccCopies, so fewer blocks queue on one address when they all finish together) of
// the 36 raw metrics, each held as three 64-bit words of 32-bit limbs. A block total v
// (below 2^96) adds limb j = (v >> 32j) & (2^32 - 1) into word j: a limb is below 2^32, so a
// word cannot overflow before 2^32 blocks, and the add needs no return value (no round trip,
// unlike a carry-propagating 128-bit add). The value is sum_j word_j * 2^32j, exact.
constexpr int kQ1AccCopies = 16;
constexpr size_t kQ1GaccWords = (size_t)kQ1AccCopies * 6 * kQ1Raw * 3;

__device__ __forceinline__ void red_add_limbs(unsigned long long* w, u128 v) {
  const unsigned long long l0 = (unsigned long long)v & 0xFFFFFFFFull;
  const unsigned long long l1 = (unsigned long long)(v >> 32) & 0xFFFFFFFFull;
  const unsigned long long l2 = (unsigned long long)(v >> 64);
  if (l0) atomicAdd(w, l0);
  if (l1) atomicAdd(w + 1, l1);
  if (l2) atomicAdd(w + 2, l2);
}

// Fold of the shared-memory form's per-thread sums acc[(metric * 6 + group) * T + thread]
// (metrics P, E, ED, EDT): each warp sums three of the 24 columns (P unpacked into count,
// quantity and discount sum) and adds the block's totals into its copy of the limb words of
// `gacc` (kQ1GaccWords); the last block turns them into the output and zeroes `gacc` for the
// next launch (it is zero when first allocated). No per-block partials are read back.
template <int T>
__device__ __forceinline__ void q1_smem_fold(const uint64_t* acc, uint32_t bad, unsigned long long* gacc, unsigned* ticket, u128* out,
                                             uint32_t* status, uint32_t* hstatus) {
  constexpr int W = T / 32;
  static_assert(24 % W == 0, "whole columns per warp");
  __shared__ u128 tot[6 * kQ1Raw];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // also orders every thread's shared-memory sums before the column reads
  if (__syncthreads_or(bad) && threadIdx.x == 0) set_status(status, ST_DOMAIN);
  for (int c = warp; c < 24; c += W) {
    const int metric = c / 6, g = c % 6;
    u128 s0 = 0, s1 = 0, s2 = 0;
#pragma unroll 4
    for (int i = lane; i < T; i += 32) {
      const uint64_t v = acc[c * T + i];
      if (metric == 0) {
        s0 += v & 0x1FFFu;
        s1 += v >> 32;
        s2 += (v >> 13) & 0x7FFFFu;
      } else {
        s0 += v;
      }
    }
    s0 = warp_sum_u128(s0);
    if (metric == 0) {
      s1 = warp_sum_u128(s1);
      s2 = warp_sum_u128(s2);
    }
    if (lane == 0) {
      // raw metrics: count, qty, E, ED, EDT, dsum
      unsigned long long* o = gacc + ((size_t)(blockIdx.x % kQ1AccCopies) * 6 * kQ1Raw + g * kQ1Raw) * 3;
      if (metric == 0) {
        red_add_limbs(o + 0 * 3, s0);
        red_add_limbs(o + 1 * 3, s1);
        red_add_limbs(o + 5 * 3, s2);
      } else {
        red_add_limbs(o + (1 + metric) * 3, s0);
      }
    }
  }
  if (!grid_last_block(ticket)) return;
  if (threadIdx.x < 6 * kQ1Raw) {
    u128 v = 0;
#pragma unroll
    for (int c = 0; c < kQ1AccCopies; c++) {
      unsigned long long* w = gacc + ((size_t)c * 6 * kQ1Raw + threadIdx.x) * 3;
      v += (u128)__ldcg(w) + ((u128)__ldcg(w + 1) << 32) + ((u128)__ldcg(w + 2) << 64);
      w[0] = 0;
      w[1] = 0;
      w[2] = 0;
    }
    tot[threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    const int g = threadIdx.x;
    const u128* r = tot + g * kQ1Raw;
    const u128 disc_price = (u128)100 * r[2] - r[3];
    const u128 charge = (u128)100 * disc_price + r[4];
    u128* o = out + g * kQ1Metrics;
    if (hstatus) {   // one launch, the host slot: overwrite
      o[0] = r[0];
      o[1] = r[1];
      o[2] = r[2];
      o[3] = disc_price;
      o[4] = charge;
      o[5] = r[5];
    } else {
      o[0] += r[0];
      o[1] += r[1];
      o[2] += r[2];
      o[3] += disc_price;
      o[4] += charge;
      o[5] += r[5];
    }
  }
  // the host slot takes the status every block has OR-ed in (visible past the ticket), and
  // the launch's own status word is left at zero for the next launch
  if (hstatus && threadIdx.x == 0) {
    *hstatus = __ldcg(status);
    *status = 0u;
  }
}

__global__ void __launch_bounds__(kThreads, 2) q1_vec_kernel(const int4* __restrict__ ship4, const int4* __restrict__ qty4,
                                                             const longlong2* __restrict__ ext2, const int4* __restrict__ disc4,
                                                             const int4* __restrict__ tax4, const uint32_t* __restrict__ flag4,
                                                             const uint32_t* __restrict__ stat4, uint64_t n, int32_t ship_le,
                                                             u128* partials, unsigned* ticket, u128* out, uint32_t* status) {
  Q1Acc a;
#pragma unroll
  for (int g = 0; g < 6; g++) a.P[g] = a.E[g] = a.ED[g] = a.EDT[g] = 0;
  a.bad = 0;
  const uint64_t nq = n >> 2;
  const uint64_t T = (uint64_t)gridDim.x * kThreads;
  for (uint64_t q = (uint64_t)blockIdx.x * kThreads + threadIdx.x; q < nq; q += T) {
    const int4 s = ld_stream(ship4 + q), k = ld_stream(qty4 + q), d = ld_stream(disc4 + q), t = ld_stream(tax4 + q);
    const longlong2 e01 = ld_stream(ext2 + 2 * q), e23 = ld_stream(ext2 + 2 * q + 1);
    const uint32_t f = ld_stream(flag4 + q), st = ld_stream(stat4 + q);
    q1_row(a, s.x, k.x, e01.x, d.x, t.x, f & 0xFF, st & 0xFF, ship_le);
    q1_row(a, s.y, k.y, e01.y, d.y, t.y, (f >> 8) & 0xFF, (st >> 8) & 0xFF, ship_le);
    q1_row(a, s.z, k.z, e23.x, d.z, t.z, (f >> 16) & 0xFF, (st >> 16) & 0xFF, ship_le);
    q1_row(a, s.w, k.w, e23.y, d.w, t.w, f >> 24, st >> 24, ship_le);
  }
  const uint64_t r = (nq << 2) + (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  if (r < n) {
    const int32_t* ship = reinterpret_cast<const int32_t*>(ship4);
    const int32_t* qty = reinterpret_cast<const int32_t*>(qty4);
    const int64_t* ext = reinterpret_cast<const int64_t*>(ext2);
    const int32_t* disc = reinterpret_cast<const int32_t*>(disc4);
    const int32_t* tax = reinterpret_cast<const int32_t*>(tax4);
    const uint8_t* flag = reinterpret_cast<const uint8_t*>(flag4);
    const uint8_t* stat = reinterpret_cast<const uint8_t*>(stat4);
    q1_row(a, ship[r], qty[r], ext[r], disc[r], tax[r], flag[r], stat[r], ship_le);
  }
  q1_fold<kThreads>(a, partials, ticket, out, status);
}

__global__ void __launch_bounds__(kThreads, 2) q1_row_kernel(const int32_t* ship, const int32_t* qty, const int64_t* ext,
                                                             const int32_t* disc, const int32_t* tax, const uint8_t* flag,
                                                             const uint8_t* stat, uint64_t n, int32_t ship_le,
                                                             u128* partials, unsigned* ticket, u128* out, uint32_t* status) {
  Q1Acc a;
#pragma unroll
  for (int g = 0; g < 6; g++) a.P[g] = a.E[g] = a.ED[g] = a.EDT[g] = 0;
  a.bad = 0;
  const uint64_t T = (uint64_t)gridDim.x * kThreads;
  for (uint64_t r = (uint64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += T)
    q1_row(a, ship[r], qty[r], ext[r], disc[r], tax[r], flag[r], stat[r], ship_le);
  q1_fold<kThreads>(a, partials, ticket, out, status);
}

// ---- Q1 with TMA-staged column tiles ----------------------------------------------------
// Persistent: one 512-thread block per SM walks tiles blockIdx, blockIdx+grid, ... of
// R = 2048*QPT rows. Thread 0 keeps STAGES tiles in flight: for each tile it posts the
// stage's byte count (26 R) on the stage's mbarrier and issues one bulk copy per column;
// all threads wait on the barrier (bounded), read their 4*QPT rows from shared memory with
// 128-bit loads, and a block barrier frees the stage for the next copy. Memory parallelism
// therefore costs shared memory instead of registers, which the 24 accumulators need.
// Shapes: QPT=1, STAGES=4 (2048-row tiles) and QPT=2, STAGES=2 (4096-row tiles, half the
// block barriers per row); both use 212,992 bytes of shared memory.
constexpr int kQ1TmaThreads = 512;

template <int QPT, int STAGES>
__global__ void __launch_bounds__(kQ1TmaThreads, 1) q1_tma_kernel(const int32_t* __restrict__ ship, const int32_t* __restrict__ qty,
                                                                  const int64_t* __restrict__ ext, const int32_t* __restrict__ disc,
                                                                  const int32_t* __restrict__ tax, const uint8_t* __restrict__ flag,
                                                                  const uint8_t* __restrict__ stat, uint64_t n, int32_t ship_le,
                                                                  u128* partials, unsigned* ticket, u128* out, uint32_t* status) {
  constexpr uint32_t R = 2048u * QPT;            // rows per tile
  constexpr uint32_t kStage = 26u * R;           // bytes per stage
  constexpr uint32_t oShip = 0, oQty = 4 * R, oExt = 8 * R, oDisc = 16 * R, oTax = 20 * R, oFlag = 24 * R,
                     oStat = 25 * R;
  extern __shared__ __align__(128) uint8_t q1_stage[];
  __shared__ __align__(8) uint64_t full[STAGES];
  Q1Acc a;
#pragma unroll
  for (int g = 0; g < 6; g++) a.P[g] = a.E[g] = a.ED[g] = a.EDT[g] = 0;
  a.bad = 0;
  const uint64_t tiles = n / R;
  const uint64_t mine = tiles > blockIdx.x ? (tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) mbar_init(&full[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto issue = [&](uint64_t j) {
    const int s = (int)(j % STAGES);
    const uint64_t r0 = (blockIdx.x + j * gridDim.x) * (uint64_t)R;
    uint8_t* st = q1_stage + (size_t)s * kStage;
    mbar_arrive_expect_tx(&full[s], kStage);
    bulk_copy_g2s(st + oShip, ship + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oQty, qty + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oExt, ext + r0, R * 8, &full[s]);
    bulk_copy_g2s(st + oDisc, disc + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oTax, tax + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oFlag, flag + r0, R, &full[s]);
    bulk_copy_g2s(st + oStat, stat + r0, R, &full[s]);
  };
  if (threadIdx.x == 0)
    for (uint64_t j = 0; j < mine && j < (uint64_t)STAGES; j++) issue(j);
  uint64_t j = 0;
  for (; j < mine; j++) {
    const int s = (int)(j % STAGES);
    const bool ok = mbar_wait(&full[s], (uint32_t)((j / STAGES) & 1), kMbarPollLimit);
    if (__syncthreads_or(!ok)) break;
    const uint8_t* st = q1_stage + (size_t)s * kStage;
#pragma unroll
    for (int q = 0; q < QPT; q++) {
      const int t = threadIdx.x + q * kQ1TmaThreads;   // quad of the tile
      const int4 sv = *reinterpret_cast<const int4*>(st + oShip + 16 * t);
      const int4 kv = *reinterpret_cast<const int4*>(st + oQty + 16 * t);
      const longlong2 e01 = *reinterpret_cast<const longlong2*>(st + oExt + 32 * t);
      const longlong2 e23 = *reinterpret_cast<const longlong2*>(st + oExt + 32 * t + 16);
      const int4 dv = *reinterpret_cast<const int4*>(st + oDisc + 16 * t);
      const int4 tv = *reinterpret_cast<const int4*>(st + oTax + 16 * t);
      const uint32_t f = *reinterpret_cast<const uint32_t*>(st + oFlag + 4 * t);
      const uint32_t g = *reinterpret_cast<const uint32_t*>(st + oStat + 4 * t);
      q1_row(a, sv.x, kv.x, e01.x, dv.x, tv.x, f & 0xFF, g & 0xFF, ship_le);
      q1_row(a, sv.y, kv.y, e01.y, dv.y, tv.y, (f >> 8) & 0xFF, (g >> 8) & 0xFF, ship_le);
      q1_row(a, sv.z, kv.z, e23.x, dv.z, tv.z, (f >> 16) & 0xFF, (g >> 16) & 0xFF, ship_le);
      q1_row(a, sv.w, kv.w, e23.y, dv.w, tv.w, f >> 24, g >> 24, ship_le);
    }
    __syncthreads();
    if (threadIdx.x == 0 && j + STAGES < mine) issue(j + STAGES);
  }
  if (j < mine && threadIdx.x == 0) {
    // a wait ran out: report it, and let the copies already issued land before leaving
    set_status(status, ST_TIMEOUT);
    for (uint64_t k = j; k < mine && k < j + STAGES; k++)
      mbar_wait(&full[k % STAGES], (uint32_t)((k / STAGES) & 1), kMbarPollLimit);
  }
  // rows after the last whole tile
  if (blockIdx.x == gridDim.x - 1)
    for (uint64_t r = tiles * R + threadIdx.x; r < n; r += kQ1TmaThreads)
      q1_row(a, ship[r], qty[r], ext[r], disc[r], tax[r], flag[r], stat[r], ship_le);
  q1_fold<kQ1TmaThreads>(a, partials, ticket, out, status);
}

// Same tiles through a producer/consumer ring: `full[s]` completes when a stage's bytes have
// landed, `empty[s]` when all 16 warps have read it. Warps release stages on their own (no
// block-wide barrier per tile) and thread 0 refills a stage as soon as it is released, so
// STAGES-1 tiles stay in flight while the warps compute.
template <int QPT, int STAGES>
__global__ void __launch_bounds__(kQ1TmaThreads, 1) q1_ring_kernel(const int32_t* __restrict__ ship, const int32_t* __restrict__ qty,
                                                                   const int64_t* __restrict__ ext, const int32_t* __restrict__ disc,
                                                                   const int32_t* __restrict__ tax, const uint8_t* __restrict__ flag,
                                                                   const uint8_t* __restrict__ stat, uint64_t n, int32_t ship_le,
                                                                   u128* partials, unsigned* ticket, u128* out, uint32_t* status) {
  constexpr uint32_t R = 2048u * QPT;
  constexpr uint32_t kStage = 26u * R;
  constexpr uint32_t oShip = 0, oQty = 4 * R, oExt = 8 * R, oDisc = 16 * R, oTax = 20 * R, oFlag = 24 * R,
                     oStat = 25 * R;
  constexpr uint32_t kWarps = kQ1TmaThreads / 32;
  extern __shared__ __align__(128) uint8_t q1_ring[];
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
  Q1Acc a;
#pragma unroll
  for (int g = 0; g < 6; g++) a.P[g] = a.E[g] = a.ED[g] = a.EDT[g] = 0;
  a.bad = 0;
  const uint64_t tiles = n / R;
  const uint64_t mine = tiles > blockIdx.x ? (tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], kWarps); }
    mbar_fence_init();
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  uint64_t issued = 0;       // thread 0: tiles whose copies were issued
  bool timed_out = false;
  auto issue = [&](uint64_t j) {
    const int s = (int)(j % STAGES);
    const uint64_t r0 = (blockIdx.x + j * gridDim.x) * (uint64_t)R;
    uint8_t* st = q1_ring + (size_t)s * kStage;
    mbar_arrive_expect_tx(&full[s], kStage);
    bulk_copy_g2s(st + oShip, ship + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oQty, qty + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oExt, ext + r0, R * 8, &full[s]);
    bulk_copy_g2s(st + oDisc, disc + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oTax, tax + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oFlag, flag + r0, R, &full[s]);
    bulk_copy_g2s(st + oStat, stat + r0, R, &full[s]);
  };
  uint64_t j = 0;
  for (; j < mine; j++) {
    if (threadIdx.x == 0) {
      // keep the ring full: reuse a stage only after every warp has released it
      while (issued < mine && issued < j + STAGES) {
        if (issued >= (uint64_t)STAGES &&
            !mbar_wait(&empty[issued % STAGES], (uint32_t)(((issued / STAGES) - 1) & 1), kMbarPollLimit)) {
          timed_out = true;
          break;
        }
        issue(issued++);
      }
    }
    const int s = (int)(j % STAGES);
    if (timed_out || !mbar_wait(&full[s], (uint32_t)((j / STAGES) & 1), kMbarPollLimit)) { timed_out = true; break; }
    const uint8_t* st = q1_ring + (size_t)s * kStage;
#pragma unroll
    for (int q = 0; q < QPT; q++) {
      const int t = threadIdx.x + q * kQ1TmaThreads;
      const int4 sv = *reinterpret_cast<const int4*>(st + oShip + 16 * t);
      const int4 kv = *reinterpret_cast<const int4*>(st + oQty + 16 * t);
      const longlong2 e01 = *reinterpret_cast<const longlong2*>(st + oExt + 32 * t);
      const longlong2 e23 = *reinterpret_cast<const longlong2*>(st + oExt + 32 * t + 16);
      const int4 dv = *reinterpret_cast<const int4*>(st + oDisc + 16 * t);
      const int4 tv = *reinterpret_cast<const int4*>(st + oTax + 16 * t);
      const uint32_t f = *reinterpret_cast<const uint32_t*>(st + oFlag + 4 * t);
      const uint32_t g = *reinterpret_cast<const uint32_t*>(st + oStat + 4 * t);
      q1_row(a, sv.x, kv.x, e01.x, dv.x, tv.x, f & 0xFF, g & 0xFF, ship_le);
      q1_row(a, sv.y, kv.y, e01.y, dv.y, tv.y, (f >> 8) & 0xFF, (g >> 8) & 0xFF, ship_le);
      q1_row(a, sv.z, kv.z, e23.x, dv.z, tv.z, (f >> 16) & 0xFF, (g >> 16) & 0xFF, ship_le);
      q1_row(a, sv.w, kv.w, e23.y, dv.w, tv.w, f >> 24, g >> 24, ship_le);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (timed_out) set_status(status, ST_TIMEOUT);
  if (threadIdx.x == 0)
    // copies this thread issued but never consumed must land before the block exits
    for (uint64_t k = j; k < issued; k++) mbar_wait(&full[k % STAGES], (uint32_t)((k / STAGES) & 1), kMbarPollLimit);
  if (blockIdx.x == gridDim.x - 1)
    for (uint64_t r = tiles * R + threadIdx.x; r < n; r += kQ1TmaThreads)
      q1_row(a, ship[r], qty[r], ext[r], disc[r], tax[r], flag[r], stat[r], ship_le);
  q1_fold<kQ1TmaThreads>(a, partials, ticket, out, status);
}

// Ring of TMA tiles as above, but each thread's 6 x 4 group accumulators live in shared
// memory ([metric][group][thread], conflict-free for a warp) and a row updates only its own
// group: 4 load-add-store per row instead of 24 predicated 64-bit adds.
template <int THREADS, int STAGES>
__global__ void __launch_bounds__(THREADS, 1) q1_ring_smem_kernel(const int32_t* __restrict__ ship, const int32_t* __restrict__ qty,
                                                                  const int64_t* __restrict__ ext, const int32_t* __restrict__ disc,
                                                                  const int32_t* __restrict__ tax, const uint8_t* __restrict__ flag,
                                                                  const uint8_t* __restrict__ stat, uint64_t n, int32_t ship_le,
                                                                  u128* partials, unsigned* ticket, u128* out, uint32_t* status) {
  constexpr uint32_t R = THREADS * 4u;            // one quad per thread per tile
  constexpr uint32_t kStage = 26u * R;
  constexpr uint32_t oShip = 0, oQty = 4 * R, oExt = 8 * R, oDisc = 16 * R, oTax = 20 * R, oFlag = 24 * R,
                     oStat = 25 * R;
  constexpr uint32_t kWarps = THREADS / 32;
  extern __shared__ __align__(128) uint8_t q1_dyn[];
  uint64_t* acc = reinterpret_cast<uint64_t*>(q1_dyn + (size_t)STAGES * kStage);   // [4][6][THREADS]
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
  const int t = threadIdx.x, lane = t & 31;
#pragma unroll
  for (int i = 0; i < 24; i++) acc[i * THREADS + t] = 0;
  uint32_t bad = 0;
  const uint64_t tiles = n / R;
  const uint64_t mine = tiles > blockIdx.x ? (tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  if (t == 0) {
    for (int s = 0; s < STAGES; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], kWarps); }
    mbar_fence_init();
  }
  __syncthreads();
  auto row = [&](int32_t s, int32_t qt, int64_t e, int32_t d, int32_t tx, uint32_t f, uint32_t st) {
    if (!((s <= ship_le) & (f <= 2u) & (st <= 1u))) return;
    bad |= ((uint32_t)qt >= 65536u) | ((uint32_t)d > 100u) | ((uint32_t)tx > 100u) | ((uint64_t)e >= (1ull << 36));
    const uint64_t ed = (uint64_t)e * (uint32_t)d;
    const uint64_t edt = ((uint64_t)e * 100u - ed) * (uint32_t)tx;
    const uint64_t pk = ((uint64_t)(uint32_t)qt << 32) | ((uint64_t)(uint32_t)d << 13) | 1u;
    uint64_t* p = acc + (f * 2u + st) * THREADS + t;
    p[0] += pk;
    p[6 * THREADS] += (uint64_t)e;
    p[12 * THREADS] += ed;
    p[18 * THREADS] += edt;
  };
  uint64_t issued = 0;
  bool timed_out = false;
  auto issue = [&](uint64_t j) {
    const int s = (int)(j % STAGES);
    const uint64_t r0 = (blockIdx.x + j * gridDim.x) * (uint64_t)R;
    uint8_t* st = q1_dyn + (size_t)s * kStage;
    mbar_arrive_expect_tx(&full[s], kStage);
    bulk_copy_g2s(st + oShip, ship + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oQty, qty + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oExt, ext + r0, R * 8, &full[s]);
    bulk_copy_g2s(st + oDisc, disc + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oTax, tax + r0, R * 4, &full[s]);
    bulk_copy_g2s(st + oFlag, flag + r0, R, &full[s]);
    bulk_copy_g2s(st + oStat, stat + r0, R, &full[s]);
  };
  uint64_t j = 0;
  for (; j < mine; j++) {
    if (t == 0) {
      while (issued < mine && issued < j + STAGES) {
        if (issued >= (uint64_t)STAGES &&
            !mbar_wait(&empty[issued % STAGES], (uint32_t)(((issued / STAGES) - 1) & 1), kMbarPollLimit)) {
          timed_out = true;
          break;
        }
        issue(issued++);
      }
    }
    const int s = (int)(j % STAGES);
    if (timed_out || !mbar_wait(&full[s], (uint32_t)((j / STAGES) & 1), kMbarPollLimit)) { timed_out = true; break; }
    const uint8_t* stg = q1_dyn + (size_t)s * kStage;
    const int4 sv = *reinterpret_cast<const int4*>(stg + oShip + 16 * t);
    const int4 kv = *reinterpret_cast<const int4*>(stg + oQty + 16 * t);
    const longlong2 e01 = *reinterpret_cast<const longlong2*>(stg + oExt + 32 * t);
    const longlong2 e23 = *reinterpret_cast<const longlong2*>(stg + oExt + 32 * t + 16);
    const int4 dv = *reinterpret_cast<const int4*>(stg + oDisc + 16 * t);
    const int4 tv = *reinterpret_cast<const int4*>(stg + oTax + 16 * t);
    const uint32_t f = *reinterpret_cast<const uint32_t*>(stg + oFlag + 4 * t);
    const uint32_t g = *reinterpret_cast<const uint32_t*>(stg + oStat + 4 * t);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);   // the tile is in registers: release the stage
    row(sv.x, kv.x, e01.x, dv.x, tv.x, f & 0xFF, g & 0xFF);
    row(sv.y, kv.y, e01.y, dv.y, tv.y, (f >> 8) & 0xFF, (g >> 8) & 0xFF);
    row(sv.z, kv.z, e23.x, dv.z, tv.z, (f >> 16) & 0xFF, (g >> 16) & 0xFF);
    row(sv.w, kv.w, e23.y, dv.w, tv.w, f >> 24, g >> 24);
  }
  if (timed_out) set_status(status, ST_TIMEOUT);
  if (t == 0)
    for (uint64_t k = j; k < issued; k++) mbar_wait(&full[k % STAGES], (uint32_t)((k / STAGES) & 1), kMbarPollLimit);
  if (blockIdx.x == gridDim.x - 1)
    for (uint64_t r = tiles * R + t; r < n; r += THREADS) row(ship[r], qty[r], ext[r], disc[r], tax[r], flag[r], stat[r]);
  Q1Acc a;
#pragma unroll
  for (int gi = 0; gi < 6; gi++) {
    a.P[gi] = acc[(0 * 6 + gi) * THREADS + t];
    a.E[gi] = acc[(1 * 6 + gi) * THREADS + t];
    a.ED[gi] = acc[(2 * 6 + gi) * THREADS + t];
    a.EDT[gi] = acc[(3 * 6 + gi) * THREADS + t];
  }
  a.bad = bad;
  q1_fold<THREADS>(a, partials, ticket, out, status);
}

// 128-bit loads straight from HBM with the accumulators in shared memory: registers stay low
// (several blocks per SM), and each thread keeps two quads (208 bytes) of loads in flight.
constexpr int kQ1SmemThreads = 256;
constexpr size_t kQ1AccBytes = (size_t)4 * 6 * kQ1SmemThreads * 8;   // 49,152

// Q6 requests evaluated on the rows a Q1 scan reads (one read of the table for both): their
// constants, and the two words (revenue, rows matched) each one adds into.
constexpr int kMaxRiders = 4;
struct Q6Riders {
  Q6P p[kMaxRiders];
  unsigned long long* out[kMaxRiders];
};

// MINB: resident blocks per SM the registers are sized for (2: the default; 3: variant 8,
// more loads in flight for tables that end in one short wave). NQ6: Q6 requests riding along
// (register sums per request, added into their words at the end). QPI: 16-byte quads per
// thread per step (2 by default; 4: variant 9; 1 with four blocks per SM: variant 10).
template <int MINB, int NQ6, int QPI = 2>
__global__ void __launch_bounds__(kQ1SmemThreads, MINB) q1_vec_smem_kernel(const int4* __restrict__ ship4, const int4* __restrict__ qty4,
                                                                     const longlong2* __restrict__ ext2, const int4* __restrict__ disc4,
                                                                     const int4* __restrict__ tax4, const uint32_t* __restrict__ flag4,
                                                                     const uint32_t* __restrict__ stat4, uint64_t n, int32_t ship_le,
                                                                     unsigned long long* gacc, unsigned* ticket, u128* out, uint32_t* status,
                                                                     uint32_t* hstatus, Q6Riders riders) {
  constexpr int T = kQ1SmemThreads;
  extern __shared__ __align__(16) uint64_t q1_acc[];   // [4 metrics][6 groups][T]
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 24; i++) q1_acc[i * T + t] = 0;
  uint32_t bad = 0;
  int64_t rrev[NQ6 > 0 ? NQ6 : 1];
  uint64_t rcnt[NQ6 > 0 ? NQ6 : 1];
#pragma unroll
  for (int r = 0; r < NQ6; r++) { rrev[r] = 0; rcnt[r] = 0; }
  auto row = [&](int32_t s, int32_t qt, int64_t e, int32_t d, int32_t tx, uint32_t f, uint32_t st) {
#pragma unroll
    for (int r = 0; r < NQ6; r++) {
      const bool m = q6_pass(s, d, qt, riders.p[r]);
      rrev[r] += m ? e * (int64_t)d : 0;
      rcnt[r] += m;
    }
    if (!((s <= ship_le) & (f <= 2u) & (st <= 1u))) return;
    bad |= ((uint32_t)qt >= 65536u) | ((uint32_t)d > 100u) | ((uint32_t)tx > 100u) | ((uint64_t)e >= (1ull << 36));
    const uint64_t ed = (uint64_t)e * (uint32_t)d;
    const uint64_t edt = ((uint64_t)e * 100u - ed) * (uint32_t)tx;
    const uint64_t pk = ((uint64_t)(uint32_t)qt << 32) | ((uint64_t)(uint32_t)d << 13) | 1u;
    uint64_t* p = q1_acc + (f * 2u + st) * T + t;
    p[0] += pk;
    p[6 * T] += (uint64_t)e;
    p[12 * T] += ed;
    p[18 * T] += edt;
  };
  auto quad = [&](const int4& s, const int4& k, const longlong2& e01, const longlong2& e23, const int4& d, const int4& x,
                  uint32_t f, uint32_t g) {
    row(s.x, k.x, e01.x, d.x, x.x, f & 0xFF, g & 0xFF);
    row(s.y, k.y, e01.y, d.y, x.y, (f >> 8) & 0xFF, (g >> 8) & 0xFF);
    row(s.z, k.z, e23.x, d.z, x.z, (f >> 16) & 0xFF, (g >> 16) & 0xFF);
    row(s.w, k.w, e23.y, d.w, x.w, f >> 24, g >> 24);
  };
  const uint64_t nq = n >> 2;
  const uint64_t S = (uint64_t)gridDim.x * T;
  uint64_t q = (uint64_t)blockIdx.x * T + t;
  // QPI quads per thread per step, all their loads issued before the first is used
  for (; q + (uint64_t)(QPI - 1) * S < nq; q += (uint64_t)QPI * S) {
    int4 sv[QPI], kv[QPI], dv[QPI], xv[QPI];
    longlong2 av[QPI], bv[QPI];
    uint32_t fv[QPI], gv[QPI];
#pragma unroll
    for (int u = 0; u < QPI; u++) {
      const uint64_t qq = q + (uint64_t)u * S;
      sv[u] = ld_stream(ship4 + qq);
      kv[u] = ld_stream(qty4 + qq);
      av[u] = ld_stream(ext2 + 2 * qq);
      bv[u] = ld_stream(ext2 + 2 * qq + 1);
      dv[u] = ld_stream(disc4 + qq);
      xv[u] = ld_stream(tax4 + qq);
      fv[u] = ld_stream(flag4 + qq);
      gv[u] = ld_stream(stat4 + qq);
    }
#pragma unroll
    for (int u = 0; u < QPI; u++) quad(sv[u], kv[u], av[u], bv[u], dv[u], xv[u], fv[u], gv[u]);
  }
  for (; q < nq; q += S)
    quad(ld_stream(ship4 + q), ld_stream(qty4 + q), ld_stream(ext2 + 2 * q), ld_stream(ext2 + 2 * q + 1),
         ld_stream(disc4 + q), ld_stream(tax4 + q), ld_stream(flag4 + q), ld_stream(stat4 + q));
  const uint64_t r = (nq << 2) + (uint64_t)blockIdx.x * T + t;
  if (r < n) {
    row(reinterpret_cast<const int32_t*>(ship4)[r], reinterpret_cast<const int32_t*>(qty4)[r],
        reinterpret_cast<const int64_t*>(ext2)[r], reinterpret_cast<const int32_t*>(disc4)[r],
        reinterpret_cast<const int32_t*>(tax4)[r], reinterpret_cast<const uint8_t*>(flag4)[r],
        reinterpret_cast<const uint8_t*>(stat4)[r]);
  }
#pragma unroll
  for (int r = 0; r < NQ6; r++) {
    const unsigned long long v = warp_sum_u64((unsigned long long)rrev[r]), c = warp_sum_u64(rcnt[r]);
    if ((t & 31) == 0) {
      if (v) atomicAdd(riders.out[r], v);
      if (c) atomicAdd(riders.out[r] + 1, c);
    }
  }
  q1_smem_fold<T>(q1_acc, bad, gacc, ticket, out, status, hstatus);
}

bool aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

int grid_for(gpudb_ctx* ctx, const void* kernel, uint64_t work_items, int min_blocks) {
  const int per_sm = kernel_occupancy(ctx, kernel, kThreads, 0);
  uint64_t want = (work_items + kThreads - 1) / kThreads;
  uint64_t cap = (uint64_t)ctx->sm_count * per_sm;
  uint64_t g = std::min<uint64_t>(want, cap);
  g = std::max<uint64_t>(g, (uint64_t)min_blocks);
  return (int)std::max<uint64_t>(g, 1);
}

// Per-launch scratch: partials of every block + the last-block ticket (new scratch is
// zeroed; each launch's last block resets the ticket).
int scan_scratch(gpudb_ctx* ctx, const char* name, size_t partial_bytes, void** partials, unsigned** ticket) {
  void* p = nullptr;
  const size_t need = partial_bytes + 256;
  int rc = scratch(ctx, name, need, &p);
  if (rc) return rc;
  *ticket = reinterpret_cast<unsigned*>(p);
  *partials = static_cast<uint8_t*>(p) + 256;
  return GPUDB_OK;
}

}  // namespace

// Enqueue one Q6 scan of device-resident columns, adding into `out` (device), or with
// `hstatus` overwriting `out` in the call's mapped host slot (a direct result).
int launch_q6(Call& call, const gpudb_lineitem& c, const gpudb_q6_params& p, void* out, uint32_t* hstatus) {
  gpudb_ctx* ctx = call.ctx();
  if (c.n_rows == 0) return GPUDB_OK;
  const Q6P pp{p.ship_lo, p.ship_hi, p.disc_lo, p.disc_hi, p.qty_lt};
  const bool vec = aligned(c.ship_date, 16) && aligned(c.discount, 16) && aligned(c.quantity, 16) && aligned(c.ext_price, 8);
  // 1 one row per thread; 2/3/4: 128-bit loads, 1/2/4 quads per thread per step. Auto (0):
  // the autotuner's choice on B200 -- one row per thread below 2^24 rows (the columns stay
  // in L2 across calls), one quad per step above
  int variant = ctx->q6_variant ? ctx->q6_variant : (c.n_rows < (1u << 24) ? 1 : 2);
  if (!vec) variant = 1;
  const int unroll = variant == 2 ? 1 : variant == 4 ? 4 : 2;
  const void* kfn = variant == 1 ? (const void*)q6_row_kernel
                    : unroll == 1 ? (const void*)q6_vec_kernel<1>
                    : unroll == 4 ? (const void*)q6_vec_kernel<4> : (const void*)q6_vec_kernel<2>;
  const int grid = variant == 1 ? grid_for(ctx, kfn, c.n_rows, 1) : grid_for(ctx, kfn, (c.n_rows / 4 + 1) / unroll, 1);
  void* part = nullptr;
  unsigned* ticket = nullptr;
  int rc = scan_scratch(ctx, "q6.partials", (size_t)grid * 16, &part, &ticket);
  if (rc) return rc;
  int64_t* prev = static_cast<int64_t*>(part);
  uint64_t* pcnt = reinterpret_cast<uint64_t*>(prev + grid);
  if (variant != 1) {
    auto k = unroll == 1 ? q6_vec_kernel<1> : unroll == 4 ? q6_vec_kernel<4> : q6_vec_kernel<2>;
    GPUDB_LAUNCH(call, k, grid, kThreads, 0, (const int4*)c.ship_date, (const int4*)c.discount,
                 (const int4*)c.quantity, c.ext_price, c.n_rows, pp, prev, pcnt, ticket, (Q6Out*)out, hstatus);
  } else {
    GPUDB_LAUNCH(call, q6_row_kernel, grid, kThreads, 0, c.ship_date, c.discount, c.quantity, c.ext_price, c.n_rows,
                 pp, prev, pcnt, ticket, (Q6Out*)out, hstatus);
  }
  return GPUDB_OK;
}

// Enqueue one Q1 scan of device-resident columns, adding into `out` (device, 36 x u128).
// The shared-memory Q1 kernel (16-byte aligned columns): a grid of SMs x occupancy blocks
// (at most kQ1RowsPerThread rows a thread) over the limb accumulators of "q1.acc".
// With `hstatus` (a direct result: `out` and `hstatus` in the call's mapped host slot) the
// launch's status word is the one in the scratch header beside the ticket, which the last
// block copies to the host slot and leaves at zero.
using Q1SmemKernel = void (*)(const int4*, const int4*, const longlong2*, const int4*, const int4*, const uint32_t*,
                              const uint32_t*, uint64_t, int32_t, unsigned long long*, unsigned*, u128*, uint32_t*,
                              uint32_t*, Q6Riders);
static int launch_q1_smem(Call& call, const gpudb_lineitem& c, const gpudb_q1_params& p, void* out, uint32_t* status,
                          Q1SmemKernel kern, const Q6Riders& riders, uint32_t* hstatus = nullptr) {
  gpudb_ctx* ctx = call.ctx();
  const size_t smem = kQ1AccBytes;
  GPUDB_CUDA(ctx, kernel_smem(ctx, (const void*)kern, smem));
  const int per_sm = kernel_occupancy(ctx, (const void*)kern, kQ1SmemThreads, smem);
  const uint64_t min_blocks = (c.n_rows + (uint64_t)kQ1SmemThreads * kQ1RowsPerThread - 1) /
                              ((uint64_t)kQ1SmemThreads * kQ1RowsPerThread);
  const uint64_t want = (c.n_rows / 4 + kQ1SmemThreads - 1) / kQ1SmemThreads;
  const int grid = (int)std::max<uint64_t>(
      1, std::max(min_blocks, std::min<uint64_t>(want, (uint64_t)ctx->sm_count * std::max(per_sm, 1))));
  // the limb accumulators and a ticket, both left at zero by every launch's last block
  void* part = nullptr;
  unsigned* ticket = nullptr;
  int rc = scan_scratch(ctx, "q1.acc", kQ1GaccWords * sizeof(unsigned long long), &part, &ticket);
  if (rc) return rc;
  if (hstatus) status = ticket + 1;
  GPUDB_LAUNCH(call, kern, grid, kQ1SmemThreads, smem, (const int4*)c.ship_date, (const int4*)c.quantity,
               (const longlong2*)c.ext_price, (const int4*)c.discount, (const int4*)c.tax, (const uint32_t*)c.flag,
               (const uint32_t*)c.status, c.n_rows, p.ship_le, (unsigned long long*)part, ticket, (u128*)out, status,
               hstatus,
               riders);
  return GPUDB_OK;
}

// The Q1 variant a launch over `c` runs (the auto choice resolved, and the choices that the
// columns' alignment rules out replaced): 7-10 are the one-launch shared-memory kernels.
static int q1_variant(const gpudb_ctx* ctx, const gpudb_lineitem& c) {
  const bool vec = aligned(c.ship_date, 16) && aligned(c.quantity, 16) && aligned(c.ext_price, 16) &&
                   aligned(c.discount, 16) && aligned(c.tax, 16) && aligned(c.flag, 4) && aligned(c.status, 4);
  const bool tma_ok = vec && aligned(c.flag, 16) && aligned(c.status, 16) && c.n_rows >= 4096;
  int variant = ctx->scan_variant;
  if (variant == 0) variant = vec ? 7 : 3;
  if (variant >= 7 && variant <= 10) return vec ? variant : 3;
  if ((variant == 1 || variant >= 4) && !tma_ok) variant = vec ? 2 : 3;
  if (variant == 2 && !vec) variant = 3;
  return variant;
}

static Q1SmemKernel q1_smem_kernel(int variant) {
  return variant == 8  ? q1_vec_smem_kernel<3, 0, 2>
       : variant == 9  ? q1_vec_smem_kernel<2, 0, 4>
       : variant == 10 ? q1_vec_smem_kernel<4, 0, 1>
                       : q1_vec_smem_kernel<2, 0, 2>;
}

int launch_q1(Call& call, const gpudb_lineitem& c, const gpudb_q1_params& p, void* out, uint32_t* status) {
  gpudb_ctx* ctx = call.ctx();
  if (!status) status = call.status();
  if (c.n_rows == 0) return GPUDB_OK;
  // 0 auto, 1 TMA 2048-row tiles x 4 stages, 2 vector loads, 3 one row per thread,
  // 4 TMA 4096-row tiles x 2 stages, 5/6 TMA rings, 7-10 shared-memory sums
  const int variant = q1_variant(ctx, c);
  if (variant >= 7 && variant <= 10) return launch_q1_smem(call, c, p, out, status, q1_smem_kernel(variant), Q6Riders{});
  if (variant == 1 || variant >= 4) {
    const uint32_t R = (variant == 1 || variant == 5) ? 2048u : variant == 6 ? 1024u : 4096u;
    const int threads = variant == 6 ? 256 : kQ1TmaThreads;
    auto kernel = variant == 1 ? q1_tma_kernel<1, 4>
                  : variant == 4 ? q1_tma_kernel<2, 2>
                  : variant == 5 ? q1_ring_kernel<1, 4>
                                 : q1_ring_smem_kernel<256, 6>;
    const uint64_t tiles = c.n_rows / R;
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)ctx->sm_count, tiles));
    // 212,992 bytes of tiles; the shared-accumulator ring: 6 x 26,624 tiles + 49,152 accumulators
    const size_t smem = variant == 6 ? (size_t)6 * 26 * 1024 + 4 * 6 * 256 * 8 : (size_t)26 * 2048 * 4;
    GPUDB_CUDA(ctx, kernel_smem(ctx, (const void*)kernel, smem));
    void* part = nullptr;
    unsigned* ticket = nullptr;
    int rc = scan_scratch(ctx, "q1.partials", (size_t)grid * 6 * kQ1Raw * sizeof(u128), &part, &ticket);
    if (rc) return rc;
    // keep every thread under kQ1RowsPerThread rows: split very large tables into launches
    const uint64_t per_launch = ((uint64_t)grid * threads * (kQ1RowsPerThread - 8) / R) * R;
    for (uint64_t r0 = 0; r0 < c.n_rows; r0 += per_launch) {
      const uint64_t rows = std::min<uint64_t>(per_launch, c.n_rows - r0);
      GPUDB_LAUNCH(call, kernel, grid, threads, smem, c.ship_date + r0, c.quantity + r0, c.ext_price + r0,
                   c.discount + r0, c.tax + r0, c.flag + r0, c.status + r0, rows, p.ship_le, (u128*)part, ticket,
                   (u128*)out, status);
    }
    return GPUDB_OK;
  }
  const int min_blocks = (int)((c.n_rows + (uint64_t)kThreads * kQ1RowsPerThread - 1) / ((uint64_t)kThreads * kQ1RowsPerThread));
  const int grid = variant == 2 ? grid_for(ctx, (const void*)q1_vec_kernel, c.n_rows / 4 + 1, min_blocks)
                                : grid_for(ctx, (const void*)q1_row_kernel, c.n_rows, min_blocks);
  void* part = nullptr;
  unsigned* ticket = nullptr;
  int rc = scan_scratch(ctx, "q1.partials", (size_t)grid * 6 * kQ1Raw * sizeof(u128), &part, &ticket);
  if (rc) return rc;
  if (variant == 2) {
    GPUDB_LAUNCH(call, q1_vec_kernel, grid, kThreads, 0, (const int4*)c.ship_date, (const int4*)c.quantity,
                 (const longlong2*)c.ext_price, (const int4*)c.discount, (const int4*)c.tax, (const uint32_t*)c.flag,
                 (const uint32_t*)c.status, c.n_rows, p.ship_le, (u128*)part, ticket, (u128*)out, status);
  } else {
    GPUDB_LAUNCH(call, q1_row_kernel, grid, kThreads, 0, c.ship_date, c.quantity, c.ext_price, c.discount, c.tax,
                 c.flag, c.status, c.n_rows, p.ship_le, (u128*)part, ticket, (u128*)out, status);
  }
  return GPUDB_OK;
}

int launch_q1_riders(Call& call, const gpudb_lineitem& c, const gpudb_q1_params& p, void* out, uint32_t* status,
                     int n6, const gpudb_q6_params* q6, void* const* q6out) {
  const bool vec = aligned(c.ship_date, 16) && aligned(c.quantity, 16) && aligned(c.ext_price, 16) &&
                   aligned(c.discount, 16) && aligned(c.tax, 16) && aligned(c.flag, 4) && aligned(c.status, 4);
  if (n6 <= 0 || n6 > kMaxRiders || !vec || c.n_rows == 0 || call.ctx()->scan_variant != 0) {
    int rc = launch_q1(call, c, p, out, status);   // one kernel per request
    for (int r = 0; !rc && r < n6; r++) rc = launch_q6(call, c, q6[r], q6out[r]);
    return rc;
  }
  Q6Riders rd{};
  for (int r = 0; r < n6; r++) {
    rd.p[r] = Q6P{q6[r].ship_lo, q6[r].ship_hi, q6[r].disc_lo, q6[r].disc_hi, q6[r].qty_lt};
    rd.out[r] = static_cast<unsigned long long*>(q6out[r]);
  }
  static constexpr Q1SmemKernel kRiding[kMaxRiders] = {q1_vec_smem_kernel<2, 1>, q1_vec_smem_kernel<2, 2>,
                                                       q1_vec_smem_kernel<2, 3>, q1_vec_smem_kernel<2, 4>};
  return launch_q1_smem(call, c, p, out, status, kRiding[n6 - 1], rd);
}

}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_q6_sum(gpudb_ctx* ctx, const gpudb_lineitem* li, const gpudb_q6_params* p,
                            gpudb_q6_result* out, gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!p || !out) return fail(ctx, GPUDB_E_INVALID, "q6: params and result are required");
  const uint32_t mask = LI_SHIP | LI_DISC | LI_QTY | LI_EXT;
  int rc = lineitem_check(ctx, li, mask);
  if (rc) return rc;
  Call call(ctx, ex, t);
  // device-resident columns: one launch, whose last block writes the result into the host slot
  const bool direct = li->location == GPUDB_MEM_DEVICE && li->n_rows > 0;
  if ((rc = direct ? call.begin_direct(sizeof(int64_t) * 2) : call.begin(sizeof(int64_t) * 2))) return rc;
  const gpudb_q6_params pp = *p;
  if (uint8_t* d = call.direct_slot()) {
    rc = launch_q6(call, *li, pp, d + kSlotHeader, reinterpret_cast<uint32_t*>(d));
  } else {
    void* dout = call.result<void>();
    rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) { return launch_q6(call, c, pp, dout); });
  }
  if (rc) return rc;
  return call.finish(sizeof(int64_t) * 2, [out](const uint8_t* h) {
    std::memcpy(&out->revenue, h, 8);
    std::memcpy(&out->rows_matched, h + 8, 8);
    return GPUDB_OK;
  });
}

extern "C" int gpudb_q1_group6(gpudb_ctx* ctx, const gpudb_lineitem* li, const gpudb_q1_params* p,
                               gpudb_q1_result* out, gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!p || !out) return fail(ctx, GPUDB_E_INVALID, "q1: params and result are required");
  const uint32_t mask = LI_SHIP | LI_QTY | LI_EXT | LI_DISC | LI_TAX | LI_FLAG | LI_STATUS;
  int rc = lineitem_check(ctx, li, mask);
  if (rc) return rc;
  Call call(ctx, ex, t);
  const size_t bytes = kQ1ResultBytes;
  static_assert(kQ1ResultBytes == 6 * kQ1Metrics * sizeof(u128), "Q1 result layout");
  // device-resident columns and a one-launch kernel: its last block writes the result into
  // the host slot
  const int variant = li->location == GPUDB_MEM_DEVICE && li->n_rows > 0 ? q1_variant(ctx, *li) : 0;
  const bool direct = variant >= 7 && variant <= 10;
  if ((rc = direct ? call.begin_direct(bytes) : call.begin(bytes))) return rc;
  const gpudb_q1_params pp = *p;
  if (uint8_t* d = call.direct_slot()) {
    rc = launch_q1_smem(call, *li, pp, d + kSlotHeader, nullptr, q1_smem_kernel(variant), Q6Riders{},
                        reinterpret_cast<uint32_t*>(d));
  } else {
    void* dout = call.result<void>();
    rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) { return launch_q1(call, c, pp, dout); });
  }
  if (rc) return rc;
  return call.finish(bytes, [out](const uint8_t* h) {
    q1_result_from(h, out);
    return GPUDB_OK;
  });
}

namespace gpudb {

void q1_result_from(const uint8_t* h, gpudb_q1_result* out) {
  std::memset(out, 0, sizeof *out);
  for (int g = 0; g < 6; g++) {
    uint64_t w[12];
    std::memcpy(w, h + g * kQ1Metrics * 16, sizeof w);
    if (w[0] == 0 && w[1] == 0) continue;
    gpudb_q1_group& o = out->groups[out->n_groups++];
    o.flag = (uint8_t)(g / 2);
    o.status = (uint8_t)(g % 2);
    o.count = w[0];
    gpudb_i128* f[5] = {&o.sum_qty, &o.sum_base_price, &o.sum_disc_price, &o.sum_charge, &o.sum_discount};
    for (int m = 0; m < 5; m++) { f[m]->lo = w[2 + 2 * m]; f[m]->hi = (int64_t)w[3 + 2 * m]; }
  }
}

}  // namespace gpudb
