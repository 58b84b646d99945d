// Q5 (local supplier volume): revenue of lineitems whose customer and supplier share a
// nation of one region, for the orders of a date window, by nation.
// Reference: kernels/q5.metal:19-125 (customer / supplier -> nation direct maps of the
// region's nations, orders of the window -> customer nation, lineitem probe with the
// same-nation test and float atomic adds into 25 bins), src/q5.cpp:8-200 (driver, nation
// bitmap of the region on the host, sort by revenue).
//
// B200 design:
//  1. nation_map_kernel (customers, suppliers): key -> nation byte for the nations of the
//     mask; the maps start at 0xFF (not in the region) and are small (a byte per key).
//  2. q5_orders_kernel: orders of the window whose customer is in the region set their bit
//     in an order-key bitmap (one atomicOr per distinct word of a warp) and write the
//     customer's nation into a byte map order key -> nation that is read only where the bit
//     is set, so it is never cleared.
//  3. q5_probe_kernel: lineitem (order and supplier keys, 4 rows per thread) tests the bitmap,
//     reads the order's nation and the supplier's, and for equal nations adds ext_price *
//     (100 - discount) (loaded only for those rows) into 25 shared-memory int64 bins per
//     block, added to the result once per block.
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"

namespace gpudb {
namespace {

constexpr int kThreads = 256;
constexpr int kRows = 4;
constexpr uint8_t kNone = 0xFF;

__global__ void __launch_bounds__(kThreads) q5_orders_kernel(const int32_t* __restrict__ okey,
                                                             const int32_t* __restrict__ ocust,
                                                             const int32_t* __restrict__ odate, uint64_t n,
                                                             int32_t date_lo, int32_t date_hi, int32_t order_max,
                                                             int32_t cust_max, const uint8_t* __restrict__ cmap,
                                                             uint32_t* okbm, uint8_t* omap, uint32_t* status) {
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {   // whole warps
    int32_t k[kRows], d[kRows], c[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      d[j] = in ? ld_stream(odate + i) : date_hi;
      k[j] = in ? ld_stream(okey + i) : 0;
      c[j] = in ? ld_stream(ocust + i) : -1;
    }
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      bool on = d[j] >= date_lo && d[j] < date_hi;
      if (on && (k[j] < 0 || k[j] > order_max)) { set_status(status, ST_KEY_RANGE); on = false; }
      const uint8_t nt = on && c[j] >= 0 && c[j] <= cust_max ? cmap[c[j]] : kNone;
      on = nt != kNone;
      if (on) omap[k[j]] = nt;
      warp_bitmap_or(on, k[j], okbm);
    }
  }
}

__global__ void __launch_bounds__(kThreads) q5_probe_kernel(const int32_t* __restrict__ lkey,
                                                            const int32_t* __restrict__ lsupp,
                                                            const int64_t* __restrict__ lext,
                                                            const int32_t* __restrict__ ldisc, uint64_t n,
                                                            int32_t order_max, int32_t supp_max,
                                                            const uint32_t* __restrict__ okbm,
                                                            const uint8_t* __restrict__ omap,
                                                            const uint8_t* __restrict__ smap, long long* out) {
  __shared__ long long bins[GPUDB_NATIONS];
  if (threadIdx.x < GPUDB_NATIONS) bins[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {
    int32_t k[kRows], s[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      k[j] = in ? ld_stream(lkey + i) : -1;
      s[j] = in ? ld_stream(lsupp + i) : -1;
    }
    uint32_t nt[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      nt[j] = kNone;
      if (k[j] >= 0 && k[j] <= order_max && s[j] >= 0 && s[j] <= supp_max && bitmap_test(okbm, k[j])) {
        const uint32_t a = __ldg(omap + k[j]);
        nt[j] = a == __ldg(smap + s[j]) ? a : kNone;
      }
    }
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      if (nt[j] == kNone) continue;
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      atomicAdd(reinterpret_cast<unsigned long long*>(&bins[nt[j]]),
                (unsigned long long)(ld_stream(lext + i) * (int64_t)(100 - ld_stream(ldisc + i))));
    }
  }
  __syncthreads();
  if (threadIdx.x < GPUDB_NATIONS && bins[threadIdx.x])
    atomicAdd(reinterpret_cast<unsigned long long*>(out + threadIdx.x), (unsigned long long)bins[threadIdx.x]);
}

unsigned grid_for(gpudb_ctx* ctx, uint64_t n, int per_thread, int per_sm) {
  return (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((n + (uint64_t)kThreads * per_thread - 1) / ((uint64_t)kThreads * per_thread),
                            (uint64_t)ctx->sm_count * per_sm));
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_q5_local_supplier(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_supplier* su,
                                       const gpudb_orders* od, const gpudb_lineitem* li, const gpudb_q5_params* p,
                                       gpudb_q5_result* out, gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!cu || !su || !od || !p || !out) return fail(ctx, GPUDB_E_INVALID, "q5: tables, params and result are required");
  if (cu->n_rows && (!cu->cust_key || !cu->nation || cu->key_max < 0))
    return fail(ctx, GPUDB_E_INVALID, "q5: customer.cust_key, nation and key_max >= 0 are required");
  if (su->n_rows && (!su->supp_key || !su->nation || su->key_max < 0))
    return fail(ctx, GPUDB_E_INVALID, "q5: supplier.supp_key, nation and key_max >= 0 are required");
  if (od->n_rows && (!od->order_key || !od->cust_key || !od->order_date || od->key_max < 0))
    return fail(ctx, GPUDB_E_INVALID, "q5: orders.order_key, cust_key, order_date and key_max >= 0 are required");
  const uint32_t mask = LI_ORDER | LI_SUPP | LI_EXT | LI_DISC;
  int rc = lineitem_check(ctx, li, mask);
  if (rc) return rc;
  Call call(ctx, ex, t);
  if ((rc = call.begin(GPUDB_NATIONS * 8))) return rc;
  cudaStream_t s = call.stream();
  const int32_t cust_max = cu->n_rows ? cu->key_max : 0, supp_max = su->n_rows ? su->key_max : 0;
  const int32_t order_max = od->n_rows ? od->key_max : 0;
  const uint32_t owords = (uint32_t)(order_max >> 5) + 1;
  void *cmap, *smap, *okbm, *omap;
  rc = scratch(ctx, "q5.cmap", (size_t)cust_max + 1, &cmap);
  if (!rc) rc = scratch(ctx, "q5.smap", (size_t)supp_max + 1, &smap);
  if (!rc) rc = scratch(ctx, "q5.okbm", (size_t)owords * 4, &okbm);
  if (!rc) rc = scratch(ctx, "q5.omap", (size_t)order_max + 1, &omap);
  if (rc) return rc;
  GPUDB_CUDA(ctx, cudaMemsetAsync(cmap, kNone, (size_t)cust_max + 1, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(smap, kNone, (size_t)supp_max + 1, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(okbm, 0, (size_t)owords * 4, s));
  if (cu->n_rows)
    GPUDB_LAUNCH(call, nation_map_kernel, grid_for(ctx, cu->n_rows, 1, 8), kThreads, 0, cu->cust_key, cu->nation,
                 cu->n_rows, cust_max, p->nation_mask, (uint8_t*)cmap, call.status());
  if (su->n_rows)
    GPUDB_LAUNCH(call, nation_map_kernel, grid_for(ctx, su->n_rows, 1, 8), kThreads, 0, su->supp_key, su->nation,
                 su->n_rows, supp_max, p->nation_mask, (uint8_t*)smap, call.status());
  if (od->n_rows && cu->n_rows)
    GPUDB_LAUNCH(call, q5_orders_kernel, grid_for(ctx, od->n_rows, kRows, 8), kThreads, 0, od->order_key, od->cust_key,
                 od->order_date, od->n_rows, p->date_lo, p->date_hi, order_max, cust_max, (const uint8_t*)cmap,
                 (uint32_t*)okbm, (uint8_t*)omap, call.status());
  if (od->n_rows && cu->n_rows && su->n_rows) {
    rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) {
      if (c.n_rows)
        GPUDB_LAUNCH(call, q5_probe_kernel, grid_for(ctx, c.n_rows, kRows, 8), kThreads, 0, c.order_key, c.supp_key,
                     c.ext_price, c.discount, c.n_rows, order_max, supp_max, (const uint32_t*)okbm,
                     (const uint8_t*)omap, (const uint8_t*)smap, call.result<long long>());
      return (int)GPUDB_OK;
    });
    if (rc) return rc;
  }
  return call.finish(GPUDB_NATIONS * 8, [out](const uint8_t* h) {
    std::memcpy(out->revenue, h, GPUDB_NATIONS * 8);
    return GPUDB_OK;
  });
}
