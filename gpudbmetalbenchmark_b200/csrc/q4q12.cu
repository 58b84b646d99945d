// Q4 (order priority checking) and Q12 (shipping modes and order priority): bitmap
// semi-joins between orders and lineitem with a handful of count bins.
// Reference: kernels/q4.metal:21-94 and src/q4.cpp:8-282 (late-delivery bitmap from lineitem,
// then orders by date window + bitmap, 5 priority bins); kernels/q12.metal:22-99 and
// src/q12.cpp:8-277 (priority bitmap from orders, then lineitem by ship mode + date
// predicates + bitmap, 4 bins).
//
// B200 design (both HBM-bound scans; no tensor-core work):
//  - bitmaps over order keys 0..key_max; a warp sets the bits of its rows with one atomicOr
//    per distinct word (__match_any_sync groups lanes of the same word, a masked OR-reduce
//    combines their bits), so clustered keys cost one atomic per warp and scattered keys one
//    per row;
//  - the scans load every column of a row together (four rows per thread per block step,
//    coalesced), keep their bins in registers, reduce them per warp and per block, and add
//    one 64-bit atomic per bin per block into the result slot;
//  - lineitem may be host-resident: it streams through the double-buffered chunk ring.
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"

namespace gpudb {
namespace {

constexpr int kThreads = 256;
constexpr int kRows = 4;   // rows per thread per block step

// Adds the block's per-thread bins into out[0..B) (one atomic per nonzero bin per block).
template <int B>
__device__ __forceinline__ void block_add_bins(const uint32_t (&c)[B], unsigned long long* out) {
  __shared__ unsigned long long sb[B];
  if (threadIdx.x < B) sb[threadIdx.x] = 0;
  __syncthreads();
#pragma unroll
  for (int b = 0; b < B; b++) {
    const uint32_t w = __reduce_add_sync(FULL_MASK, c[b]);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(&sb[b], (unsigned long long)w);
  }
  __syncthreads();
  if (threadIdx.x < B && sb[threadIdx.x]) atomicAdd(out + threadIdx.x, sb[threadIdx.x]);
}

// ---- Q4 ------------------------------------------------------------------------------------
// Late-delivery bitmap (kernels/q4.metal:21-37): order keys of lineitem rows with
// commit_date < receipt_date; keys outside 0..key_max match no order and are skipped.
__global__ void __launch_bounds__(kThreads) q4_late_kernel(const int32_t* __restrict__ key,
                                                           const int32_t* __restrict__ commit,
                                                           const int32_t* __restrict__ receipt, uint64_t n,
                                                           int32_t key_max, uint32_t* bits) {
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {   // whole warps
    int32_t k[kRows], c[kRows], r[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      k[j] = in ? ld_stream(key + i) : -1;
      c[j] = in ? ld_stream(commit + i) : 0;
      r[j] = in ? ld_stream(receipt + i) : 0;
    }
#pragma unroll
    for (int j = 0; j < kRows; j++) warp_bitmap_or(c[j] < r[j] && k[j] >= 0 && k[j] <= key_max, k[j], bits);
  }
}

// Orders in [date_lo, date_hi) whose key is in the late bitmap, counted by priority 1..5
// (kernels/q4.metal:40-72). An order key outside 0..key_max is a key-range error.
__global__ void __launch_bounds__(kThreads) q4_count_kernel(const int32_t* __restrict__ okey,
                                                            const int32_t* __restrict__ odate,
                                                            const uint8_t* __restrict__ oprio, uint64_t n,
                                                            int32_t date_lo, int32_t date_hi, int32_t key_max,
                                                            const uint32_t* __restrict__ bits,
                                                            unsigned long long* out, uint32_t* status) {
  uint32_t cnt[5] = {0, 0, 0, 0, 0};
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {
    int32_t k[kRows], d[kRows];
    uint32_t p[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      d[j] = in ? ld_stream(odate + i) : date_hi;
      k[j] = in ? ld_stream(okey + i) : 0;
      p[j] = in ? ld_stream(oprio + i) : 0u;
    }
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      if (d[j] < date_lo || d[j] >= date_hi) continue;
      if (k[j] < 0 || k[j] > key_max) { set_status(status, ST_KEY_RANGE); continue; }
      if (!bitmap_test(bits, k[j])) continue;
#pragma unroll
      for (int q = 0; q < 5; q++) cnt[q] += p[j] == (uint32_t)(q + 1);
    }
  }
  block_add_bins(cnt, out);
}

// ---- Q12 -----------------------------------------------------------------------------------
// Priority bitmap (kernels/q12.metal:87-99): orders with priority 1..high_max.
__global__ void __launch_bounds__(kThreads) q12_prio_kernel(const int32_t* __restrict__ okey,
                                                            const uint8_t* __restrict__ oprio, uint64_t n,
                                                            int32_t high_max, int32_t key_max, uint32_t* bits,
                                                            uint32_t* status) {
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {   // whole warps
    int32_t k[kRows];
    uint32_t p[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      k[j] = in ? ld_stream(okey + i) : 0;
      p[j] = in ? ld_stream(oprio + i) : 0u;
    }
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      bool on = p[j] >= 1u && p[j] <= (uint32_t)high_max;
      if (on && (k[j] < 0 || k[j] > key_max)) { set_status(status, ST_KEY_RANGE); on = false; }
      warp_bitmap_or(on, k[j], bits);
    }
  }
}

struct Q12Args {
  int32_t receipt_lo, receipt_hi, mode0, mode1, key_max;
};

// Lineitem rows of ship mode mode0 / mode1 with receipt in [lo, hi), commit < receipt and
// ship < commit, counted high or low by the priority bitmap (kernels/q12.metal:22-66).
// Bins: out[0..1] high for mode0/mode1, out[2..3] low.
__global__ void __launch_bounds__(kThreads) q12_count_kernel(const int32_t* __restrict__ lkey,
                                                             const int32_t* __restrict__ lship,
                                                             const int32_t* __restrict__ lcommit,
                                                             const int32_t* __restrict__ lreceipt,
                                                             const uint8_t* __restrict__ lmode, uint64_t n, Q12Args a,
                                                             const uint32_t* __restrict__ bits,
                                                             unsigned long long* out) {
  uint32_t cnt[4] = {0, 0, 0, 0};
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {
    int32_t k[kRows], s[kRows], c[kRows], r[kRows], m[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      m[j] = in ? (int32_t)ld_stream(lmode + i) : -1;
      r[j] = in ? ld_stream(lreceipt + i) : 0;
      c[j] = in ? ld_stream(lcommit + i) : 0;
      s[j] = in ? ld_stream(lship + i) : 0;
      k[j] = in ? ld_stream(lkey + i) : -1;
    }
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const int mi = m[j] == a.mode0 ? 0 : (m[j] == a.mode1 ? 1 : -1);
      if (mi < 0 || r[j] < a.receipt_lo || r[j] >= a.receipt_hi || c[j] >= r[j] || s[j] >= c[j]) continue;
      const bool high = k[j] >= 0 && k[j] <= a.key_max && bitmap_test(bits, k[j]);
      cnt[(high ? 0 : 2) + mi]++;
    }
  }
  block_add_bins(cnt, out);
}

unsigned scan_grid(gpudb_ctx* ctx, uint64_t n) {
  return (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((n + kThreads * kRows - 1) / (kThreads * kRows), (uint64_t)ctx->sm_count * 8));
}

int orders_check(gpudb_ctx* ctx, const gpudb_orders* od, bool need_date) {
  if (!od) return fail(ctx, GPUDB_E_INVALID, "orders is NULL");
  if (od->n_rows && (!od->order_key || !od->priority || (need_date && !od->order_date)))
    return fail(ctx, GPUDB_E_INVALID, "orders: order_key, priority%s are required", need_date ? ", order_date" : "");
  if (od->n_rows && od->key_max < 0) return fail(ctx, GPUDB_E_INVALID, "orders.key_max must be >= 0");
  return GPUDB_OK;
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_q4_priority(gpudb_ctx* ctx, const gpudb_orders* od, const gpudb_lineitem* li,
                                 const gpudb_q4_params* p, gpudb_q4_result* out, gpudb_timing* t,
                                 const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!p || !out) return fail(ctx, GPUDB_E_INVALID, "q4: params and result are required");
  int rc = orders_check(ctx, od, true);
  const uint32_t mask = LI_ORDER | LI_COMMIT | LI_RECEIPT;
  if (!rc) rc = lineitem_check(ctx, li, mask);
  if (rc) return rc;
  Call call(ctx, ex, t);
  if ((rc = call.begin(40))) return rc;
  cudaStream_t s = call.stream();
  const int32_t key_max = od->n_rows ? od->key_max : 0;
  const uint32_t words = (uint32_t)(key_max >> 5) + 1;
  void* bits = nullptr;
  if ((rc = scratch(ctx, "q4.late", (size_t)words * 4, &bits))) return rc;
  GPUDB_CUDA(ctx, cudaMemsetAsync(bits, 0, (size_t)words * 4, s));
  if (od->n_rows) {
    rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) {
      if (c.n_rows)
        GPUDB_LAUNCH(call, q4_late_kernel, scan_grid(ctx, c.n_rows), kThreads, 0, c.order_key, c.commit_date,
                     c.receipt_date, c.n_rows, key_max, (uint32_t*)bits);
      return (int)GPUDB_OK;
    });
    if (rc) return rc;
    GPUDB_LAUNCH(call, q4_count_kernel, scan_grid(ctx, od->n_rows), kThreads, 0, od->order_key, od->order_date,
                 od->priority, od->n_rows, p->date_lo, p->date_hi, key_max, (const uint32_t*)bits,
                 call.result<unsigned long long>(), call.status());
  }
  return call.finish(40, [out](const uint8_t* h) {
    std::memcpy(out->count, h, 40);
    return GPUDB_OK;
  });
}

extern "C" int gpudb_q12_shipmode(gpudb_ctx* ctx, const gpudb_orders* od, const gpudb_lineitem* li,
                                  const gpudb_q12_params* p, gpudb_q12_result* out, gpudb_timing* t,
                                  const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!p || !out) return fail(ctx, GPUDB_E_INVALID, "q12: params and result are required");
  int rc = orders_check(ctx, od, false);
  const uint32_t mask = LI_ORDER | LI_SHIP | LI_COMMIT | LI_RECEIPT | LI_MODE;
  if (!rc) rc = lineitem_check(ctx, li, mask);
  if (rc) return rc;
  Call call(ctx, ex, t);
  if ((rc = call.begin(32))) return rc;
  cudaStream_t s = call.stream();
  const int32_t key_max = od->n_rows ? od->key_max : 0;
  const uint32_t words = (uint32_t)(key_max >> 5) + 1;
  void* bits = nullptr;
  if ((rc = scratch(ctx, "q12.high", (size_t)words * 4, &bits))) return rc;
  GPUDB_CUDA(ctx, cudaMemsetAsync(bits, 0, (size_t)words * 4, s));
  if (od->n_rows)
    GPUDB_LAUNCH(call, q12_prio_kernel, scan_grid(ctx, od->n_rows), kThreads, 0, od->order_key, od->priority,
                 od->n_rows, p->high_max, key_max, (uint32_t*)bits, call.status());
  // with no orders every row is low (an empty bitmap); its key bound is then -1
  const Q12Args a{p->receipt_lo, p->receipt_hi, p->mode[0], p->mode[1], od->n_rows ? key_max : -1};
  rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) {
    if (c.n_rows)
      GPUDB_LAUNCH(call, q12_count_kernel, scan_grid(ctx, c.n_rows), kThreads, 0, c.order_key, c.ship_date,
                   c.commit_date, c.receipt_date, c.ship_mode, c.n_rows, a, (const uint32_t*)bits,
                   call.result<unsigned long long>());
    return (int)GPUDB_OK;
  });
  if (rc) return rc;
  return call.finish(32, [out](const uint8_t* h) {
    std::memcpy(out, h, 32);
    return GPUDB_OK;
  });
}
