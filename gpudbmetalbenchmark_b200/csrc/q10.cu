// Q10 (returned item reporting): revenue of returned lineitems per customer for the orders
// of a date window, and the k customers of largest revenue.
// Reference: kernels/q10.metal:8-54 (orders direct map order key -> customer for the window,
// then returned lineitems add float revenue per customer with atomic float adds),
// src/q10.cpp:8-140 (driver, top-20 heap on the host).
//
// B200 design:
//  1. bitmap_build_kernel: the customer table's keys -> bitmap (the join with customer).
//  2. q10_orders_kernel: orders in the window set their bit in an order-key bitmap (one
//     atomicOr per distinct word of a warp) and write their customer into a direct map
//     order key -> customer. The map is read only where the bit is set, so it is never
//     cleared (at SF-10 it is 240 MB; the bitmap 7.5 MB).
//  3. q10_probe_kernel: lineitem rows with flag 2 ('R') test the bitmap (L2-resident),
//     read the map, and add ext_price * (100 - discount) to their customer's int64 revenue
//     (ext/discount loaded only for those rows).
//  4. q10_hist_kernel + q10_select_kernel: the top-k of the per-customer revenue array by the
//     revenue-histogram select of the Q3 top-k (q3.h): a log-scale histogram, the bin that
//     holds the k-th best, the customers in bins at or above it, ranked in the last block.
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"
#include "q3.h"

namespace gpudb {
namespace {

constexpr int kThreads = 256;
constexpr int kRows = 4;

__global__ void __launch_bounds__(kThreads) q10_orders_kernel(const int32_t* __restrict__ okey,
                                                              const int32_t* __restrict__ ocust,
                                                              const int32_t* __restrict__ odate, uint64_t n,
                                                              int32_t date_lo, int32_t date_hi, int32_t key_max,
                                                              uint32_t* okbm, int32_t* map, uint32_t* status) {
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {   // whole warps
    int32_t k[kRows], d[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      d[j] = in ? ld_stream(odate + i) : date_hi;
      k[j] = in ? ld_stream(okey + i) : 0;
    }
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      bool on = d[j] >= date_lo && d[j] < date_hi;
      if (on && (k[j] < 0 || k[j] > key_max)) { set_status(status, ST_KEY_RANGE); on = false; }
      if (on) map[k[j]] = ld_stream(ocust + b + (uint64_t)j * kThreads + threadIdx.x);
      warp_bitmap_or(on, k[j], okbm);
    }
  }
}

// The bitmap words of a thread's kRows rows are loaded in one phase and the map entries of the
// rows whose bit is set in the next, so the loads of each phase are in flight together.
__global__ void __launch_bounds__(kThreads) q10_probe_kernel(const int32_t* __restrict__ lkey,
                                                             const uint8_t* __restrict__ lflag,
                                                             const int64_t* __restrict__ lext,
                                                             const int32_t* __restrict__ ldisc, uint64_t n,
                                                             int32_t order_max, const uint32_t* __restrict__ okbm,
                                                             const int32_t* __restrict__ map, int32_t cust_max,
                                                             const uint32_t* __restrict__ custbm,
                                                             unsigned long long* rev) {
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {
    int32_t k[kRows];
    bool want[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      const uint32_t f = in ? ld_stream(lflag + i) : 0u;
      k[j] = in ? ld_stream(lkey + i) : -1;
      want[j] = f == 2u && k[j] >= 0 && k[j] <= order_max;
    }
    uint32_t w[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) w[j] = want[j] ? __ldg(okbm + ((uint32_t)k[j] >> 5)) : 0u;
    int32_t c[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) c[j] = (w[j] >> ((uint32_t)k[j] & 31u) & 1u) ? __ldg(map + k[j]) : -1;
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      if (c[j] < 0 || c[j] > cust_max || !bitmap_test(custbm, c[j])) continue;
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      atomicAdd(rev + c[j], (unsigned long long)(ld_stream(lext + i) * (int64_t)(100 - ld_stream(ldisc + i))));
    }
  }
}

// Customers with revenue > 0: counted into *n_cust, and a histogram of rev_bin into
// state[0..kRevBins).
__global__ void __launch_bounds__(kThreads) q10_hist_kernel(const unsigned long long* __restrict__ rev, uint64_t n,
                                                            uint32_t* state, unsigned long long* n_cust) {
  __shared__ uint32_t sh[kRevBins];
  for (int i = threadIdx.x; i < kRevBins; i += kThreads) sh[i] = 0;
  __syncthreads();
  uint32_t cnt = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kThreads) {
    const long long v = (long long)ld_stream(rev + i);
    if (v > 0) {
      atomicAdd(&sh[rev_bin((unsigned long long)v)], 1u);
      cnt++;
    }
  }
  cnt = __reduce_add_sync(FULL_MASK, cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(n_cust, (unsigned long long)cnt);
  __syncthreads();
  for (int i = threadIdx.x; i < kRevBins; i += kThreads)
    if (sh[i]) atomicAdd(&state[i], sh[i]);
}

// The customers in bins >= b* (the bin holding the k-th best) are appended and ranked by
// (revenue desc, key asc) in the last block; more than kTopkCandCap candidates fall back to a
// tiled block top-k of the whole array.
__global__ void __launch_bounds__(kTopkThreads) q10_select_kernel(const unsigned long long* __restrict__ rev,
                                                                  uint64_t n, int k, uint32_t* state, u128* cand,
                                                                  u128* out) {
  __shared__ u128 sm[kTopkScratch];
  __shared__ u128 carry[GPUDB_Q3_MAX_K];
  __shared__ uint32_t wsum[kTopkWarps];
  __shared__ uint32_t bstar;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
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
  const uint64_t stride = (uint64_t)gridDim.x * kTopkThreads;
  const uint64_t end = (n + 31) & ~31ull;   // whole warps: warp_append is collective
  for (uint64_t i = (uint64_t)blockIdx.x * kTopkThreads + t; i < end; i += stride) {
    const long long v = i < n ? (long long)ld_stream(rev + i) : 0ll;
    const bool take = v > 0 && rev_bin((unsigned long long)v) >= bs;
    if (__any_sync(FULL_MASK, take)) {
      const uint32_t pos = warp_append(take, ncand);
      if (take && pos < kTopkCandCap) cand[pos] = topk_compose(v, 0, (int32_t)i);
    }
  }
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
    block_topk_stream(n, k, [&](uint64_t i) {
      const long long v = (long long)__ldcg(rev + i);
      return v > 0 ? topk_compose(v, 0, (int32_t)i) : (u128)0;
    }, carry, sm);
  }
  for (int i = t; i < k; i += kTopkThreads) out[i] = carry[i];
}

unsigned grid_for(gpudb_ctx* ctx, uint64_t n, int per_thread, int per_sm) {
  return (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((n + (uint64_t)kThreads * per_thread - 1) / ((uint64_t)kThreads * per_thread),
                            (uint64_t)ctx->sm_count * per_sm));
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_q10_returned(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_orders* od,
                                  const gpudb_lineitem* li, const gpudb_q10_params* p, gpudb_q10_result* out,
                                  gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!cu || !od || !p || !out) return fail(ctx, GPUDB_E_INVALID, "q10: tables, params and result are required");
  if (p->k < 1 || p->k > GPUDB_Q3_MAX_K) return fail(ctx, GPUDB_E_INVALID, "q10: k must be in 1..%d", GPUDB_Q3_MAX_K);
  if (cu->n_rows && (!cu->cust_key || cu->key_max < 0))
    return fail(ctx, GPUDB_E_INVALID, "q10: customer.cust_key and key_max >= 0 are required");
  if (od->n_rows && (!od->order_key || !od->cust_key || !od->order_date || od->key_max < 0))
    return fail(ctx, GPUDB_E_INVALID, "q10: orders.order_key, cust_key, order_date and key_max >= 0 are required");
  const uint32_t mask = LI_ORDER | LI_FLAG | LI_EXT | LI_DISC;
  int rc = lineitem_check(ctx, li, mask);
  if (rc) return rc;
  Call call(ctx, ex, t);
  const size_t bytes = 16 + (size_t)GPUDB_Q3_MAX_K * sizeof(u128);
  if ((rc = call.begin(bytes))) return rc;
  cudaStream_t s = call.stream();
  const int32_t cust_max = cu->n_rows ? cu->key_max : 0, order_max = od->n_rows ? od->key_max : 0;
  const uint32_t cwords = (uint32_t)(cust_max >> 5) + 1, owords = (uint32_t)(order_max >> 5) + 1;
  void *custbm, *okbm, *map, *rev, *tstate, *cand;
  rc = scratch(ctx, "q10.custbm", (size_t)cwords * 4, &custbm);
  if (!rc) rc = scratch(ctx, "q10.okbm", (size_t)owords * 4, &okbm);
  if (!rc) rc = scratch(ctx, "q10.map", ((size_t)order_max + 1) * 4, &map);
  if (!rc) rc = scratch(ctx, "q10.rev", ((size_t)cust_max + 1) * 8, &rev);
  if (!rc) rc = scratch(ctx, "q10.topk", (size_t)kTopkStateWords * 4, &tstate);
  if (!rc) rc = scratch(ctx, "q10.cand", (size_t)kTopkCandCap * sizeof(u128), &cand);
  if (rc) return rc;
  GPUDB_CUDA(ctx, cudaMemsetAsync(custbm, 0, (size_t)cwords * 4, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(okbm, 0, (size_t)owords * 4, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(rev, 0, ((size_t)cust_max + 1) * 8, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(tstate, 0, (size_t)kTopkStateWords * 4, s));
  uint8_t* res = call.result<uint8_t>();
  if (cu->n_rows)
    GPUDB_LAUNCH(call, bitmap_build_kernel, grid_for(ctx, cu->n_rows, 1, 16), kThreads, 0, cu->cust_key, nullptr, -1,
                 cu->n_rows, cust_max, (uint32_t*)custbm, call.status());
  if (od->n_rows)
    GPUDB_LAUNCH(call, q10_orders_kernel, grid_for(ctx, od->n_rows, kRows, 8), kThreads, 0, od->order_key, od->cust_key,
                 od->order_date, od->n_rows, p->date_lo, p->date_hi, order_max, (uint32_t*)okbm, (int32_t*)map,
                 call.status());
  if (od->n_rows && cu->n_rows) {
    rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) {
      if (c.n_rows)
        GPUDB_LAUNCH(call, q10_probe_kernel, grid_for(ctx, c.n_rows, kRows, 8), kThreads, 0, c.order_key, c.flag,
                     c.ext_price, c.discount, c.n_rows, order_max, (const uint32_t*)okbm, (const int32_t*)map,
                     cust_max, (const uint32_t*)custbm, (unsigned long long*)rev);
      return (int)GPUDB_OK;
    });
    if (rc) return rc;
  }
  const uint64_t n_rev = (uint64_t)cust_max + 1;
  const int sms = ctx->sm_count;
  GPUDB_LAUNCH(call, q10_hist_kernel, grid_for(ctx, n_rev, 1, 4), kThreads, 0, (const unsigned long long*)rev, n_rev,
               (uint32_t*)tstate, reinterpret_cast<unsigned long long*>(res));
  const unsigned sel = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(n_rev / kTopkSlotsPerBlock, (uint64_t)sms * 2));
  GPUDB_LAUNCH(call, q10_select_kernel, sel, kTopkThreads, 0, (const unsigned long long*)rev, n_rev, p->k,
               (uint32_t*)tstate, (u128*)cand, reinterpret_cast<u128*>(res + 16));
  const int k = p->k;
  return call.finish(bytes, [out, k](const uint8_t* h) {
    std::memset(out, 0, sizeof *out);
    std::memcpy(&out->n_customers, h, 8);
    const u128* rows = reinterpret_cast<const u128*>(h + 16);
    uint32_t n = 0;
    for (int i = 0; i < k; i++) {
      if (rows[i] == 0) break;
      int64_t rv;
      int32_t date, key;
      topk_decompose(rows[i], &rv, &date, &key);
      out->rows[n].cust_key = key;
      out->rows[n].revenue = rv;
      n++;
    }
    out->n_rows = n;
    return GPUDB_OK;
  });
}
