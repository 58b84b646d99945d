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
// the output (+=) so a streamed table is one launch per chunk on the same output.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "engine.h"

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
                                              unsigned* ticket, Q6Out* out) {
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
    out->revenue += (int64_t)ta;
    out->matched += tb;
  }
}

template <int UNROLL>
__global__ void __launch_bounds__(kThreads) q6_vec_kernel(const int4* __restrict__ ship4, const int4* __restrict__ disc4,
                                                          const int4* __restrict__ qty4, const int64_t* __restrict__ ext,
                                                          uint64_t n, Q6P p, int64_t* part_rev, uint64_t* part_cnt,
                                                          unsigned* ticket, Q6Out* out) {
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
  block_fold_q6<kThreads>(rev, cnt, part_rev, part_cnt, ticket, out);
}

// Any alignment: one row per thread per step.
__global__ void __launch_bounds__(kThreads) q6_row_kernel(const int32_t* ship, const int32_t* disc, const int32_t* qty,
                                                          const int64_t* ext, uint64_t n, Q6P p, int64_t* part_rev,
                                                          uint64_t* part_cnt, unsigned* ticket, Q6Out* out) {
  const uint64_t T = (uint64_t)gridDim.x * kThreads;
  int64_t rev = 0;
  uint32_t cnt = 0;
  for (uint64_t r = (uint64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += T)
    if (q6_pass(ship[r], disc[r], qty[r], p)) { rev += ext[r] * (int64_t)disc[r]; cnt++; }
  block_fold_q6<kThreads>(rev, cnt, part_rev, part_cnt, ticket, out);
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
#pragma unroll
  for (int k = 0; k < 6; k++) {
    if (g == (uint32_t)k) {
      a.P[k] += pk;
      a.E[k] += (uint64_t)e;
      a.ED[k] += ed;
      a.EDT[k] += edt;
    }
  }
}

__device__ __forceinline__ void q1_fold(Q1Acc& a, u128* partials, unsigned* ticket, u128* out, uint32_t* status) {
  __shared__ u128 red[kThreads / 32][6 * kQ1Raw];
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
    for (int w = 0; w < kThreads / 32; w++) s += red[w][threadIdx.x];
    partials[(size_t)blockIdx.x * 6 * kQ1Raw + threadIdx.x] = s;
  }
  if (!grid_last_block(ticket)) return;
  if (threadIdx.x < 6 * kQ1Raw) {
    u128 s = 0;
    const uint64_t* pp = reinterpret_cast<const uint64_t*>(partials);
    for (unsigned b = 0; b < gridDim.x; b++) {
      size_t i = ((size_t)b * 6 * kQ1Raw + threadIdx.x) * 2;
      s += ((u128)__ldcg(pp + i + 1) << 64) | __ldcg(pp + i);
    }
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
  q1_fold(a, partials, ticket, out, status);
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
  q1_fold(a, partials, ticket, out, status);
}

bool aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

int grid_for(gpudb_ctx* ctx, const void* kernel, uint64_t work_items, int min_blocks) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
  uint64_t want = (work_items + kThreads - 1) / kThreads;
  uint64_t cap = (uint64_t)ctx->sm_count * per_sm;
  uint64_t g = std::min<uint64_t>(want, cap);
  g = std::max<uint64_t>(g, (uint64_t)min_blocks);
  return (int)std::max<uint64_t>(g, 1);
}

// Per-launch scratch: partials of every block + the last-block ticket (zeroed once).
int scan_scratch(gpudb_ctx* ctx, const char* name, size_t partial_bytes, void** partials, unsigned** ticket) {
  void* p = nullptr;
  const size_t need = partial_bytes + 256;
  Buffer& b = ctx->scratch[name];
  const bool fresh = b.bytes < need;
  int rc = scratch(ctx, name, need, &p);
  if (rc) return rc;
  if (fresh) GPUDB_CUDA(ctx, cudaMemset(p, 0, need));
  *ticket = reinterpret_cast<unsigned*>(p);
  *partials = static_cast<uint8_t*>(p) + 256;
  return GPUDB_OK;
}

}  // namespace

// Enqueue one Q6 scan of device-resident columns, adding into `out` (device).
int launch_q6(Call& call, const gpudb_lineitem& c, const gpudb_q6_params& p, void* out) {
  gpudb_ctx* ctx = call.ctx();
  if (c.n_rows == 0) return GPUDB_OK;
  const Q6P pp{p.ship_lo, p.ship_hi, p.disc_lo, p.disc_hi, p.qty_lt};
  const bool vec = aligned(c.ship_date, 16) && aligned(c.discount, 16) && aligned(c.quantity, 16) && aligned(c.ext_price, 8);
  const int grid = vec ? grid_for(ctx, (const void*)q6_vec_kernel<2>, (c.n_rows / 4 + 1) / 2, 1)
                       : grid_for(ctx, (const void*)q6_row_kernel, c.n_rows, 1);
  void* part = nullptr;
  unsigned* ticket = nullptr;
  int rc = scan_scratch(ctx, "q6.partials", (size_t)grid * 16, &part, &ticket);
  if (rc) return rc;
  int64_t* prev = static_cast<int64_t*>(part);
  uint64_t* pcnt = reinterpret_cast<uint64_t*>(prev + grid);
  if (vec) {
    GPUDB_LAUNCH(call, q6_vec_kernel<2>, grid, kThreads, 0, (const int4*)c.ship_date, (const int4*)c.discount,
                 (const int4*)c.quantity, c.ext_price, c.n_rows, pp, prev, pcnt, ticket, (Q6Out*)out);
  } else {
    GPUDB_LAUNCH(call, q6_row_kernel, grid, kThreads, 0, c.ship_date, c.discount, c.quantity, c.ext_price, c.n_rows,
                 pp, prev, pcnt, ticket, (Q6Out*)out);
  }
  return GPUDB_OK;
}

// Enqueue one Q1 scan of device-resident columns, adding into `out` (device, 36 x u128).
int launch_q1(Call& call, const gpudb_lineitem& c, const gpudb_q1_params& p, void* out) {
  gpudb_ctx* ctx = call.ctx();
  if (c.n_rows == 0) return GPUDB_OK;
  const bool vec = aligned(c.ship_date, 16) && aligned(c.quantity, 16) && aligned(c.ext_price, 16) &&
                   aligned(c.discount, 16) && aligned(c.tax, 16) && aligned(c.flag, 4) && aligned(c.status, 4);
  const int min_blocks = (int)((c.n_rows + (uint64_t)kThreads * kQ1RowsPerThread - 1) / ((uint64_t)kThreads * kQ1RowsPerThread));
  const int grid = vec ? grid_for(ctx, (const void*)q1_vec_kernel, c.n_rows / 4 + 1, min_blocks)
                       : grid_for(ctx, (const void*)q1_row_kernel, c.n_rows, min_blocks);
  void* part = nullptr;
  unsigned* ticket = nullptr;
  int rc = scan_scratch(ctx, "q1.partials", (size_t)grid * 6 * kQ1Raw * sizeof(u128), &part, &ticket);
  if (rc) return rc;
  if (vec) {
    GPUDB_LAUNCH(call, q1_vec_kernel, grid, kThreads, 0, (const int4*)c.ship_date, (const int4*)c.quantity,
                 (const longlong2*)c.ext_price, (const int4*)c.discount, (const int4*)c.tax, (const uint32_t*)c.flag,
                 (const uint32_t*)c.status, c.n_rows, p.ship_le, (u128*)part, ticket, (u128*)out, call.status());
  } else {
    GPUDB_LAUNCH(call, q1_row_kernel, grid, kThreads, 0, c.ship_date, c.quantity, c.ext_price, c.discount, c.tax,
                 c.flag, c.status, c.n_rows, p.ship_le, (u128*)part, ticket, (u128*)out, call.status());
  }
  return GPUDB_OK;
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
  if ((rc = call.begin(sizeof(int64_t) * 2))) return rc;
  const gpudb_q6_params pp = *p;
  void* dout = call.result<void>();
  rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) { return launch_q6(call, c, pp, dout); });
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
  const size_t bytes = 6 * kQ1Metrics * sizeof(u128);
  if ((rc = call.begin(bytes))) return rc;
  const gpudb_q1_params pp = *p;
  void* dout = call.result<void>();
  rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) { return launch_q1(call, c, pp, dout); });
  if (rc) return rc;
  return call.finish(bytes, [out](const uint8_t* h) {
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
    return GPUDB_OK;
  });
}
