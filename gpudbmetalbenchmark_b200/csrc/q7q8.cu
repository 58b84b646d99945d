// Q7 (volume shipping between two nations) and Q8 (a nation's market share in its region),
// both binned by calendar year.
// Reference: kernels/q7.metal:12-109 (supplier and customer maps of the two nations, orders ->
// customer map, lineitem probe in the ship window with pair and year bins of float atomics);
// kernels/q8.metal:9-76 (orders of the window with a customer of the region -> customer and
// year maps, lineitem probe of the part-type bitmap: total and the nation's volume per year).
//
// B200 design (as Q5/Q10): byte maps key -> nation for the dimension tables; for orders, a
// bitmap of the orders that can contribute plus an uncleared byte map order -> value (Q7: the
// customer's nation, Q8: the year index), read only where the bit is set; a lineitem probe
// that adds the exact int64 revenue into shared-memory bins (2 x 8 or 8 + 8) per block. Years
// are calendar years of day numbers: the host passes the first day of every year of the window
// (at most GPUDB_MAX_YEARS) and a kernel counts the boundaries a date has passed.
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"

namespace gpudb {
namespace {

constexpr int kThreads = 256;
constexpr int kRows = 4;
constexpr uint8_t kNone = 0xFF;
constexpr int kYears = GPUDB_MAX_YEARS;

// First day (day number, 0 = 1992-01-01) of every year of a window, and their count.
struct Years {
  int32_t first_year, n;
  int32_t start[kYears + 1];   // start[y] = first day of year first_year + y
};

int year_len(int y) { return ((y % 4 == 0 && y % 100 != 0) || y % 400 == 0) ? 366 : 365; }
int year_of_day(int32_t d, int32_t* year_start) {
  int y = 1992, s = 0;
  while (d < s) { y--; s -= year_len(y); }
  while (d >= s + year_len(y)) { s += year_len(y); y++; }
  *year_start = s;
  return y;
}

// The window's years; false when it is empty or spans more than kYears years.
bool years_of(int32_t lo, int32_t hi, Years* Y) {
  if (hi < lo) return false;
  int32_t s0, s1;
  const int y0 = year_of_day(lo, &s0), y1 = year_of_day(hi, &s1);
  if (y1 - y0 + 1 > kYears) return false;
  Y->first_year = y0;
  Y->n = y1 - y0 + 1;
  int32_t s = s0;
  for (int i = 0; i <= Y->n; i++) { Y->start[i] = s; s += year_len(y0 + i); }
  for (int i = Y->n + 1; i <= kYears; i++) Y->start[i] = INT32_MAX;
  return true;
}

__device__ __forceinline__ int year_index(int32_t d, const Years& Y) {
  int y = 0;
#pragma unroll
  for (int i = 1; i < kYears; i++) y += d >= Y.start[i];
  return y;
}

// Adds the block's shared-memory bins to out[0..B).
template <int B>
__device__ __forceinline__ void flush_bins(long long* bins, long long* out) {
  __syncthreads();
  if (threadIdx.x < B && bins[threadIdx.x])
    atomicAdd(reinterpret_cast<unsigned long long*>(out + threadIdx.x), (unsigned long long)bins[threadIdx.x]);
}

// ---- Q7 ------------------------------------------------------------------------------------
// Every order whose customer is of nation a or b: bit in okbm, the customer's nation in omap.
__global__ void __launch_bounds__(kThreads) q7_orders_kernel(const int32_t* __restrict__ okey,
                                                             const int32_t* __restrict__ ocust, uint64_t n,
                                                             int32_t order_max, int32_t cust_max,
                                                             const uint8_t* __restrict__ cmap, uint32_t* okbm,
                                                             uint8_t* omap, uint32_t* status) {
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {   // whole warps
    int32_t k[kRows], c[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      k[j] = in ? ld_stream(okey + i) : 0;
      c[j] = in ? ld_stream(ocust + i) : -1;
    }
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const bool row = b + (uint64_t)j * kThreads + threadIdx.x < n;
      bool on = row;
      if (row && (k[j] < 0 || k[j] > order_max)) { set_status(status, ST_KEY_RANGE); on = false; }
      const uint8_t nt = on && c[j] >= 0 && c[j] <= cust_max ? cmap[c[j]] : kNone;
      on = nt != kNone;
      if (on) omap[k[j]] = nt;
      warp_bitmap_or(on, k[j], okbm);
    }
  }
}

struct Q7Args {
  int32_t a, b, ship_lo, ship_hi, order_max, supp_max;
  Years Y;
};

// Lineitems shipped in [ship_lo, ship_hi] between a supplier and a customer of the two nations:
// bins[pair * kYears + year].
__global__ void __launch_bounds__(kThreads) q7_probe_kernel(const int32_t* __restrict__ lkey,
                                                            const int32_t* __restrict__ lsupp,
                                                            const int32_t* __restrict__ lship,
                                                            const int64_t* __restrict__ lext,
                                                            const int32_t* __restrict__ ldisc, uint64_t n, Q7Args a,
                                                            const uint32_t* __restrict__ okbm,
                                                            const uint8_t* __restrict__ omap,
                                                            const uint8_t* __restrict__ smap, long long* out) {
  __shared__ long long bins[2 * kYears];
  if (threadIdx.x < 2 * kYears) bins[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {
    int32_t k[kRows], s[kRows], d[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      d[j] = in ? ld_stream(lship + i) : a.ship_hi + 1;
      k[j] = in ? ld_stream(lkey + i) : -1;
      s[j] = in ? ld_stream(lsupp + i) : -1;
    }
    int bin[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      bin[j] = -1;
      if (d[j] < a.ship_lo || d[j] > a.ship_hi || k[j] < 0 || k[j] > a.order_max || s[j] < 0 || s[j] > a.supp_max ||
          !bitmap_test(okbm, k[j]))
        continue;
      const int c = __ldg(omap + k[j]), sn = __ldg(smap + s[j]);
      const int pair = (sn == a.a && c == a.b) ? 0 : (sn == a.b && c == a.a) ? 1 : -1;
      if (pair >= 0) bin[j] = pair * kYears + year_index(d[j], a.Y);
    }
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      if (bin[j] < 0) continue;
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      atomicAdd(reinterpret_cast<unsigned long long*>(&bins[bin[j]]),
                (unsigned long long)(ld_stream(lext + i) * (int64_t)(100 - ld_stream(ldisc + i))));
    }
  }
  flush_bins<2 * kYears>(bins, out);
}

// ---- Q8 ------------------------------------------------------------------------------------
// Orders of [date_lo, date_hi] whose customer is in the region: bit in okbm, year index in omap.
__global__ void __launch_bounds__(kThreads) q8_orders_kernel(const int32_t* __restrict__ okey,
                                                             const int32_t* __restrict__ ocust,
                                                             const int32_t* __restrict__ odate, uint64_t n,
                                                             int32_t date_lo, int32_t date_hi, int32_t order_max,
                                                             int32_t cust_max, const uint8_t* __restrict__ cmap,
                                                             Years Y, uint32_t* okbm, uint8_t* omap, uint32_t* status) {
  const uint64_t step = (uint64_t)gridDim.x * kThreads * kRows;
  for (uint64_t b = (uint64_t)blockIdx.x * kThreads * kRows; b < n; b += step) {   // whole warps
    int32_t k[kRows], c[kRows], d[kRows];
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      const uint64_t i = b + (uint64_t)j * kThreads + threadIdx.x;
      const bool in = i < n;
      d[j] = in ? ld_stream(odate + i) : date_hi + 1;
      k[j] = in ? ld_stream(okey + i) : 0;
      c[j] = in ? ld_stream(ocust + i) : -1;
    }
#pragma unroll
    for (int j = 0; j < kRows; j++) {
      bool on = d[j] >= date_lo && d[j] <= date_hi;
      if (on && (k[j] < 0 || k[j] > order_max)) { set_status(status, ST_KEY_RANGE); on = false; }
      on = on && c[j] >= 0 && c[j] <= cust_max && cmap[c[j]] != kNone;
      if (on) omap[k[j]] = (uint8_t)year_index(d[j], Y);
      warp_bitmap_or(on, k[j], okbm);
    }
  }
}

struct Q8Args {
  int32_t part_max, order_max, supp_max;
};

// Lineitems of parts of the type (part bitmap) and orders of okbm: bins[year] += revenue,
// bins[kYears + year] too when the supplier is of the nation. Every row's part is tested
// against a filter in shared memory (smem_filter_*: the exact part bitmap when it fits,
// else a hashed one whose hits are confirmed in `pbits`): a type is about 1 part in 150, so
// nearly every row is turned away without a global-memory access. Part keys stream with
// 128-bit loads, 16 rows per thread per step; order and supplier keys, the maps and ext/disc
// are loaded only for the rows that pass.
constexpr int kQ8Threads = 1024;
constexpr int kQ8Quads = 4;
constexpr int kQ8Rows = 4 * kQ8Quads;

__global__ void __launch_bounds__(kQ8Threads) q8_probe_kernel(const int32_t* __restrict__ lkey,
                                                              const int32_t* __restrict__ lpart,
                                                              const int32_t* __restrict__ lsupp,
                                                              const int64_t* __restrict__ lext,
                                                              const int32_t* __restrict__ ldisc, uint64_t n, Q8Args a,
                                                              const uint32_t* __restrict__ pbits,
                                                              const uint32_t* __restrict__ filt, uint32_t filt_words,
                                                              bool exact, const uint32_t* __restrict__ okbm,
                                                              const uint8_t* __restrict__ omap,
                                                              const uint8_t* __restrict__ smap, long long* out) {
  extern __shared__ uint32_t q8_filt[];
  __shared__ long long bins[2 * kYears];
  if (threadIdx.x < 2 * kYears) bins[threadIdx.x] = 0;
  smem_filter_load(filt, filt_words, q8_filt);   // ends with a block barrier
  const bool vec = (reinterpret_cast<uintptr_t>(lpart) & 15u) == 0;
  constexpr uint64_t kStepRows = (uint64_t)kQ8Threads * kQ8Rows;
  const uint64_t step = (uint64_t)gridDim.x * kStepRows;
  auto row_of = [&](uint64_t b, int q, int k) { return b + 4 * ((uint64_t)q * kQ8Threads + threadIdx.x) + k; };
  for (uint64_t b = (uint64_t)blockIdx.x * kStepRows; b < n; b += step) {
    int32_t p[kQ8Rows];
    if (vec && b + kStepRows <= n) {
#pragma unroll
      for (int q = 0; q < kQ8Quads; q++) {
        const int4 v = ld_stream(reinterpret_cast<const int4*>(lpart + row_of(b, q, 0)));
        p[4 * q] = v.x; p[4 * q + 1] = v.y; p[4 * q + 2] = v.z; p[4 * q + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < kQ8Quads; q++)
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint64_t r = row_of(b, q, k);
          p[4 * q + k] = r < n ? ld_stream(lpart + r) : -1;
        }
    }
    uint32_t ok = 0;
#pragma unroll
    for (int j = 0; j < kQ8Rows; j++) ok |= (uint32_t)(p[j] >= 0 && p[j] <= a.part_max) << j;
    uint32_t take = smem_filter_mask(q8_filt, exact, pbits, p, ok);
    while (take) {
      const int j = __ffs(take) - 1;
      take &= take - 1;
      const uint64_t i = row_of(b, j >> 2, j & 3);
      const int32_t k = ld_stream(lkey + i), s = ld_stream(lsupp + i);
      if (k < 0 || k > a.order_max || s < 0 || s > a.supp_max || !bitmap_test(okbm, k)) continue;
      const int y = __ldg(omap + k);
      const unsigned long long r = (unsigned long long)(ld_stream(lext + i) * (int64_t)(100 - ld_stream(ldisc + i)));
      atomicAdd(reinterpret_cast<unsigned long long*>(&bins[y]), r);
      if (__ldg(smap + s) != kNone) atomicAdd(reinterpret_cast<unsigned long long*>(&bins[kYears + y]), r);
    }
  }
  flush_bins<2 * kYears>(bins, out);
}

unsigned grid_for(gpudb_ctx* ctx, uint64_t n, int per_thread, int per_sm) {
  return (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((n + (uint64_t)kThreads * per_thread - 1) / ((uint64_t)kThreads * per_thread),
                            (uint64_t)ctx->sm_count * per_sm));
}

int check_dims(gpudb_ctx* ctx, const char* q, const gpudb_customer* cu, const gpudb_supplier* su,
               const gpudb_orders* od, bool need_date) {
  if (cu->n_rows && (!cu->cust_key || !cu->nation || cu->key_max < 0))
    return fail(ctx, GPUDB_E_INVALID, "%s: customer.cust_key, nation and key_max >= 0 are required", q);
  if (su->n_rows && (!su->supp_key || !su->nation || su->key_max < 0))
    return fail(ctx, GPUDB_E_INVALID, "%s: supplier.supp_key, nation and key_max >= 0 are required", q);
  if (od->n_rows && (!od->order_key || !od->cust_key || (need_date && !od->order_date) || od->key_max < 0))
    return fail(ctx, GPUDB_E_INVALID, "%s: orders keys, customer%s and key_max >= 0 are required", q,
                need_date ? ", date" : "");
  return GPUDB_OK;
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_q7_volume_shipping(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_supplier* su,
                                        const gpudb_orders* od, const gpudb_lineitem* li, const gpudb_q7_params* p,
                                        gpudb_q7_result* out, gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!cu || !su || !od || !p || !out) return fail(ctx, GPUDB_E_INVALID, "q7: tables, params and result are required");
  if (p->nation_a < 0 || p->nation_a >= GPUDB_NATIONS || p->nation_b < 0 || p->nation_b >= GPUDB_NATIONS)
    return fail(ctx, GPUDB_E_INVALID, "q7: nations must be in 0..%d", GPUDB_NATIONS - 1);
  Years Y;
  if (!years_of(p->ship_lo, p->ship_hi, &Y))
    return fail(ctx, GPUDB_E_INVALID, "q7: the ship window must span 1..%d calendar years", kYears);
  int rc = check_dims(ctx, "q7", cu, su, od, false);
  const uint32_t mask = LI_ORDER | LI_SUPP | LI_SHIP | LI_EXT | LI_DISC;
  if (!rc) rc = lineitem_check(ctx, li, mask);
  if (rc) return rc;
  Call call(ctx, ex, t);
  const size_t bytes = 2 * kYears * 8;
  if ((rc = call.begin(bytes))) return rc;
  cudaStream_t s = call.stream();
  const int32_t cust_max = cu->n_rows ? cu->key_max : 0, supp_max = su->n_rows ? su->key_max : 0;
  const int32_t order_max = od->n_rows ? od->key_max : 0;
  const uint32_t owords = (uint32_t)(order_max >> 5) + 1;
  void *cmap, *smap, *okbm, *omap;
  rc = scratch(ctx, "q7.cmap", (size_t)cust_max + 1, &cmap);
  if (!rc) rc = scratch(ctx, "q7.smap", (size_t)supp_max + 1, &smap);
  if (!rc) rc = scratch(ctx, "q7.okbm", (size_t)owords * 4, &okbm);
  if (!rc) rc = scratch(ctx, "q7.omap", (size_t)order_max + 1, &omap);
  if (rc) return rc;
  GPUDB_CUDA(ctx, cudaMemsetAsync(cmap, kNone, (size_t)cust_max + 1, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(smap, kNone, (size_t)supp_max + 1, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(okbm, 0, (size_t)owords * 4, s));
  const uint32_t pair_mask = (1u << p->nation_a) | (1u << p->nation_b);
  if (cu->n_rows)
    GPUDB_LAUNCH(call, nation_map_kernel, grid_for(ctx, cu->n_rows, 1, 8), kThreads, 0, cu->cust_key, cu->nation,
                 cu->n_rows, cust_max, pair_mask, (uint8_t*)cmap, call.status());
  if (su->n_rows)
    GPUDB_LAUNCH(call, nation_map_kernel, grid_for(ctx, su->n_rows, 1, 8), kThreads, 0, su->supp_key, su->nation,
                 su->n_rows, supp_max, pair_mask, (uint8_t*)smap, call.status());
  if (od->n_rows && cu->n_rows)
    GPUDB_LAUNCH(call, q7_orders_kernel, grid_for(ctx, od->n_rows, kRows, 8), kThreads, 0, od->order_key,
                 od->cust_key, od->n_rows, order_max, cust_max, (const uint8_t*)cmap, (uint32_t*)okbm, (uint8_t*)omap,
                 call.status());
  if (od->n_rows && cu->n_rows && su->n_rows) {
    const Q7Args a{p->nation_a, p->nation_b, p->ship_lo, p->ship_hi, order_max, supp_max, Y};
    rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) {
      if (c.n_rows)
        GPUDB_LAUNCH(call, q7_probe_kernel, grid_for(ctx, c.n_rows, kRows, 8), kThreads, 0, c.order_key, c.supp_key,
                     c.ship_date, c.ext_price, c.discount, c.n_rows, a, (const uint32_t*)okbm, (const uint8_t*)omap,
                     (const uint8_t*)smap, call.result<long long>());
      return (int)GPUDB_OK;
    });
    if (rc) return rc;
  }
  const int32_t fy = Y.first_year, ny = Y.n;
  return call.finish(bytes, [out, fy, ny](const uint8_t* h) {
    std::memset(out, 0, sizeof *out);
    out->first_year = fy;
    out->n_years = ny;
    std::memcpy(out->revenue, h, 2 * kYears * 8);
    return GPUDB_OK;
  });
}

extern "C" int gpudb_q8_market_share(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_supplier* su,
                                     const gpudb_part* pa, const gpudb_orders* od, const gpudb_lineitem* li,
                                     const gpudb_q8_params* p, gpudb_q8_result* out, gpudb_timing* t,
                                     const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!cu || !su || !pa || !od || !p || !out)
    return fail(ctx, GPUDB_E_INVALID, "q8: tables, params and result are required");
  if (p->nation < 0 || p->nation >= GPUDB_NATIONS) return fail(ctx, GPUDB_E_INVALID, "q8: nation must be in 0..24");
  if (p->part_type < 0 || p->part_type > 149) return fail(ctx, GPUDB_E_INVALID, "q8: part_type must be in 0..149");
  Years Y;
  if (!years_of(p->date_lo, p->date_hi, &Y))
    return fail(ctx, GPUDB_E_INVALID, "q8: the date window must span 1..%d calendar years", kYears);
  int rc = check_dims(ctx, "q8", cu, su, od, true);
  if (!rc && pa->n_rows && (!pa->part_key || !pa->type || pa->key_max < 0))
    rc = fail(ctx, GPUDB_E_INVALID, "q8: part.part_key, type and key_max >= 0 are required");
  const uint32_t mask = LI_ORDER | LI_PART | LI_SUPP | LI_EXT | LI_DISC;
  if (!rc) rc = lineitem_check(ctx, li, mask);
  if (rc) return rc;
  Call call(ctx, ex, t);
  const size_t bytes = 2 * kYears * 8;
  if ((rc = call.begin(bytes))) return rc;
  cudaStream_t s = call.stream();
  const int32_t cust_max = cu->n_rows ? cu->key_max : 0, supp_max = su->n_rows ? su->key_max : 0;
  const int32_t order_max = od->n_rows ? od->key_max : 0, part_max = pa->n_rows ? pa->key_max : 0;
  const uint32_t owords = (uint32_t)(order_max >> 5) + 1, pwords = (uint32_t)(part_max >> 5) + 1;
  void *cmap, *smap, *okbm, *omap, *pbits;
  rc = scratch(ctx, "q8.cmap", (size_t)cust_max + 1, &cmap);
  if (!rc) rc = scratch(ctx, "q8.smap", (size_t)supp_max + 1, &smap);
  if (!rc) rc = scratch(ctx, "q8.okbm", (size_t)owords * 4, &okbm);
  if (!rc) rc = scratch(ctx, "q8.omap", (size_t)order_max + 1, &omap);
  if (!rc) rc = scratch(ctx, "q8.pbits", (size_t)pwords * 4, &pbits);
  if (rc) return rc;
  GPUDB_CUDA(ctx, cudaMemsetAsync(cmap, kNone, (size_t)cust_max + 1, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(smap, kNone, (size_t)supp_max + 1, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(okbm, 0, (size_t)owords * 4, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(pbits, 0, (size_t)pwords * 4, s));
  if (pa->n_rows)
    GPUDB_LAUNCH(call, bitmap_build_kernel, grid_for(ctx, pa->n_rows, 1, 16), kThreads, 0, pa->part_key, pa->type,
                 p->part_type, pa->n_rows, part_max, (uint32_t*)pbits, call.status());
  if (cu->n_rows)
    GPUDB_LAUNCH(call, nation_map_kernel, grid_for(ctx, cu->n_rows, 1, 8), kThreads, 0, cu->cust_key, cu->nation,
                 cu->n_rows, cust_max, p->region_mask, (uint8_t*)cmap, call.status());
  if (su->n_rows)
    GPUDB_LAUNCH(call, nation_map_kernel, grid_for(ctx, su->n_rows, 1, 8), kThreads, 0, su->supp_key, su->nation,
                 su->n_rows, supp_max, 1u << p->nation, (uint8_t*)smap, call.status());
  if (od->n_rows && cu->n_rows)
    GPUDB_LAUNCH(call, q8_orders_kernel, grid_for(ctx, od->n_rows, kRows, 8), kThreads, 0, od->order_key,
                 od->cust_key, od->order_date, od->n_rows, p->date_lo, p->date_hi, order_max, cust_max,
                 (const uint8_t*)cmap, Y, (uint32_t*)okbm, (uint8_t*)omap, call.status());
  if (od->n_rows && cu->n_rows && su->n_rows && pa->n_rows) {
    const Q8Args a{part_max, order_max, supp_max};
    // the probe's part filter: the exact bitmap itself, or a hashed one built from it
    const bool exact = smem_filter_exact(part_max);
    const uint32_t fwords = smem_filter_words(part_max);
    void* hfilt = nullptr;
    if (!exact) {
      if ((rc = scratch(ctx, "q8.partfilter", (size_t)kSmemFilterWords * 4, &hfilt))) return rc;
      GPUDB_CUDA(ctx, cudaMemsetAsync(hfilt, 0, (size_t)kSmemFilterWords * 4, s));
      GPUDB_LAUNCH(call, hashed_filter_kernel, grid_for(ctx, pwords, 1, 8), kThreads, 0, (const uint32_t*)pbits, pwords,
                   (uint32_t*)hfilt);
    }
    const size_t fsmem = (size_t)fwords * 4;
    GPUDB_CUDA(ctx, kernel_smem(ctx, (const void*)q8_probe_kernel, fsmem));
    const int per_sm = kernel_occupancy(ctx, (const void*)q8_probe_kernel, kQ8Threads, fsmem);
    rc = stream_lineitem(call, li, mask, 0, [&](const gpudb_lineitem& c) {
      if (c.n_rows) {
        const uint64_t per_block = (uint64_t)kQ8Threads * kQ8Rows;
        const unsigned g = (unsigned)std::max<uint64_t>(
            1, std::min<uint64_t>((c.n_rows + per_block - 1) / per_block, (uint64_t)ctx->sm_count * std::max(1, per_sm)));
        GPUDB_LAUNCH(call, q8_probe_kernel, g, kQ8Threads, fsmem, c.order_key, c.part_key, c.supp_key, c.ext_price,
                     c.discount, c.n_rows, a, (const uint32_t*)pbits, (const uint32_t*)(exact ? pbits : hfilt), fwords,
                     exact, (const uint32_t*)okbm, (const uint8_t*)omap, (const uint8_t*)smap,
                     call.result<long long>());
      }
      return (int)GPUDB_OK;
    });
    if (rc) return rc;
  }
  const int32_t fy = Y.first_year, ny = Y.n;
  return call.finish(bytes, [out, fy, ny](const uint8_t* h) {
    std::memset(out, 0, sizeof *out);
    out->first_year = fy;
    out->n_years = ny;
    std::memcpy(out->volume, h, kYears * 8);
    std::memcpy(out->nation_volume, h + kYears * 8, kYears * 8);
    return GPUDB_OK;
  });
}
