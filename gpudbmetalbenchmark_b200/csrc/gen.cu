// Synthetic table generation on the device (one kernel per column) and on the host
// cores (same functions compiled for the host, split across threads). Replaces the
// reference's .tbl loading step (src/infra.h:262-361) for the synthetic workloads.
#include <algorithm>
#include <thread>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "gen.h"
#include "scan.cuh"

namespace gpudb {
namespace {

struct GenArgs {
  uint64_t seed, off, n;
  int64_t n_orders, n_cust, n_parts, n_supp;
  int32_t column, order_mode;
};

// Value of `column` at absolute row r (every column except clustered lineitem order keys).
__host__ __device__ __forceinline__ void gen_value(const GenArgs& a, uint64_t r, void* dst, uint64_t i) {
  int32_t* i32 = static_cast<int32_t*>(dst);
  int64_t* i64 = static_cast<int64_t*>(dst);
  uint8_t* u8 = static_cast<uint8_t*>(dst);
  switch (a.column) {
    case GPUDB_COL_LI_SHIP_DATE: i32[i] = gd_li_ship_date(a.seed, r); break;
    case GPUDB_COL_LI_QUANTITY: i32[i] = gd_li_quantity(a.seed, r); break;
    case GPUDB_COL_LI_EXT_PRICE: i64[i] = gd_li_ext_price(a.seed, r); break;
    case GPUDB_COL_LI_DISCOUNT: i32[i] = gd_li_discount(a.seed, r); break;
    case GPUDB_COL_LI_TAX: i32[i] = gd_li_tax(a.seed, r); break;
    case GPUDB_COL_LI_FLAG: u8[i] = gd_li_flag(a.seed, r); break;
    case GPUDB_COL_LI_STATUS: u8[i] = gd_li_status(a.seed, r); break;
    case GPUDB_COL_LI_ORDER_KEY: i32[i] = gd_li_order_uniform(a.seed, r, a.n_orders); break;
    case GPUDB_COL_LI_PART_KEY: i32[i] = gd_li_part(a.seed, r, a.n_parts); break;
    case GPUDB_COL_LI_SUPP_KEY: i32[i] = gd_li_supp(a.seed, r, a.n_parts, a.n_supp); break;
    case GPUDB_COL_LI_COMMIT_DATE: i32[i] = gd_li_commit_date(a.seed, r); break;
    case GPUDB_COL_LI_RECEIPT_DATE: i32[i] = gd_li_receipt_date(a.seed, r); break;
    case GPUDB_COL_LI_SHIP_MODE: u8[i] = gd_li_ship_mode(a.seed, r); break;
    case GPUDB_COL_CU_CUST_KEY: i32[i] = (int32_t)r; break;
    case GPUDB_COL_CU_SEGMENT: u8[i] = gd_cu_segment(a.seed, r); break;
    case GPUDB_COL_CU_NATION: u8[i] = gd_cu_nation(a.seed, r); break;
    case GPUDB_COL_OR_ORDER_KEY: i32[i] = gd_order_key_of((int64_t)r); break;
    case GPUDB_COL_OR_CUST_KEY: i32[i] = gd_or_cust(a.seed, r, a.n_cust); break;
    case GPUDB_COL_OR_ORDER_DATE: i32[i] = gd_or_date(a.seed, r); break;
    case GPUDB_COL_OR_PRIORITY: u8[i] = gd_or_priority(a.seed, r); break;
    case GPUDB_COL_OR_COMMENT: gd_or_comment(a.seed, r, reinterpret_cast<char*>(u8) + i * GD_COMMENT_WIDTH); break;
    case GPUDB_COL_PA_PART_KEY: i32[i] = (int32_t)r; break;
    case GPUDB_COL_PA_FLAG: u8[i] = gd_pa_flag(a.seed, r); break;
    case GPUDB_COL_PA_TYPE: u8[i] = gd_pa_type(a.seed, r); break;
    case GPUDB_COL_SU_SUPP_KEY: i32[i] = (int32_t)r; break;
    case GPUDB_COL_SU_NATION: u8[i] = gd_su_nation(a.seed, r); break;
    case GPUDB_COL_PS_PART_KEY: i32[i] = (int32_t)(r / 4); break;
    case GPUDB_COL_PS_SUPP_KEY: i32[i] = gd_partsupp_supp((int64_t)(r / 4), (int64_t)(r % 4), a.n_supp); break;
    case GPUDB_COL_PS_SUPPLY_COST: i64[i] = gd_ps_cost(a.seed, r); break;
    default: break;
  }
}

__global__ void gen_column_kernel(GenArgs a, void* dst) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride)
    gen_value(a, a.off + i, dst, i);
}

__global__ void run_lengths_kernel(uint64_t seed, uint64_t runs, uint8_t* len) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < runs; s += stride)
    len[s] = (uint8_t)gd_li_run_length(seed, s);
}

// Run s covers rows [start[s], start[s] + len[s]) and carries order (s mod n_orders).
__global__ void run_fill_kernel(const uint8_t* len, const uint64_t* start, uint64_t runs, uint64_t off,
                                uint64_t n, int64_t n_orders, int32_t* dst) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < runs; s += stride) {
    const uint64_t b = start[s];
    const int32_t key = gd_order_key_of((int64_t)(s % (uint64_t)n_orders));
    for (uint32_t j = 0; j < len[s]; j++) {
      uint64_t row = b + j;
      if (row >= off && row < off + n) dst[row - off] = key;
    }
  }
}

int column_width(int32_t c) {
  switch (c) {
    case GPUDB_COL_LI_EXT_PRICE: case GPUDB_COL_PS_SUPPLY_COST: return 8;
    case GPUDB_COL_LI_FLAG: case GPUDB_COL_LI_STATUS: case GPUDB_COL_CU_SEGMENT:
    case GPUDB_COL_PA_FLAG: case GPUDB_COL_SU_NATION: case GPUDB_COL_LI_SHIP_MODE: case GPUDB_COL_OR_PRIORITY:
    case GPUDB_COL_CU_NATION: case GPUDB_COL_PA_TYPE:
      return 1;
    case GPUDB_COL_LI_COMMIT_DATE: case GPUDB_COL_LI_RECEIPT_DATE: return 4;
    case GPUDB_COL_OR_COMMENT: return GD_COMMENT_WIDTH;
    case GPUDB_COL_LI_SHIP_DATE: case GPUDB_COL_LI_QUANTITY: case GPUDB_COL_LI_DISCOUNT:
    case GPUDB_COL_LI_TAX: case GPUDB_COL_LI_ORDER_KEY: case GPUDB_COL_LI_PART_KEY:
    case GPUDB_COL_LI_SUPP_KEY: case GPUDB_COL_CU_CUST_KEY: case GPUDB_COL_OR_ORDER_KEY:
    case GPUDB_COL_OR_CUST_KEY: case GPUDB_COL_OR_ORDER_DATE: case GPUDB_COL_PA_PART_KEY:
    case GPUDB_COL_SU_SUPP_KEY: case GPUDB_COL_PS_PART_KEY: case GPUDB_COL_PS_SUPP_KEY: return 4;
    default: return 0;
  }
}

void host_clustered(const GenArgs& a, int32_t* dst) {
  uint64_t row = 0, s = 0, end = a.off + a.n;
  while (row < end) {
    int32_t len = gd_li_run_length(a.seed, s);
    int32_t key = gd_order_key_of((int64_t)(s % (uint64_t)a.n_orders));
    for (int32_t j = 0; j < len && row < end; j++, row++)
      if (row >= a.off) dst[row - a.off] = key;
    s++;
  }
}

void host_generate(const GenArgs& a, void* dst) {
  const uint64_t min_rows_per_thread = 1u << 16;
  unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  unsigned T = (unsigned)std::min<uint64_t>(hw, std::max<uint64_t>(1, a.n / min_rows_per_thread));
  const int w = column_width(a.column);
  auto work = [&](uint64_t b, uint64_t e) {
    GenArgs sub = a;
    sub.off = a.off + b;
    sub.n = e - b;
    uint8_t* d = static_cast<uint8_t*>(dst) + b * w;
    for (uint64_t i = 0; i < sub.n; i++) gen_value(sub, sub.off + i, d, i);
  };
  if (T <= 1) { work(0, a.n); return; }
  std::vector<std::thread> th;
  for (unsigned t = 0; t < T; t++) th.emplace_back(work, a.n * t / T, a.n * (t + 1) / T);
  for (auto& x : th) x.join();
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_column_width(int32_t column) { return column_width(column); }

extern "C" int gpudb_generate(gpudb_ctx* ctx, const gpudb_gen_spec* spec, int32_t column, void* dst,
                              int32_t location) {
  // host generation needs no context (and no GPU)
  if (!spec || (!ctx && location != GPUDB_MEM_HOST)) return GPUDB_E_INVALID;
  const int w = column_width(column);
  if (w == 0) return fail(ctx, GPUDB_E_INVALID, "unknown column id %d", column);
  if (spec->n_rows == 0) return GPUDB_OK;
  if (!dst) return fail(ctx, GPUDB_E_INVALID, "dst is NULL");
  GenArgs a{spec->seed, spec->row_offset, spec->n_rows, spec->n_orders, spec->n_cust,
            spec->n_parts, spec->n_supp, column, spec->order_mode};
  const bool li_order = column == GPUDB_COL_LI_ORDER_KEY;
  if (li_order && (a.n_orders <= 0 || (a.order_mode != GPUDB_ORDERS_CLUSTERED && a.order_mode != GPUDB_ORDERS_UNIFORM)))
    return fail(ctx, GPUDB_E_INVALID, "lineitem order keys need n_orders > 0 and an order_mode");
  if ((column == GPUDB_COL_LI_PART_KEY || column == GPUDB_COL_LI_SUPP_KEY) && a.n_parts <= 0)
    return fail(ctx, GPUDB_E_INVALID, "lineitem part/supp keys need n_parts > 0");
  if ((column == GPUDB_COL_LI_SUPP_KEY || column == GPUDB_COL_PS_SUPP_KEY) && a.n_supp < 4)
    return fail(ctx, GPUDB_E_INVALID, "supplier keys need n_supp >= 4");
  if (column == GPUDB_COL_OR_CUST_KEY && a.n_cust <= 0)
    return fail(ctx, GPUDB_E_INVALID, "orders cust keys need n_cust > 0");
  const bool clustered = li_order && a.order_mode == GPUDB_ORDERS_CLUSTERED;

  if (location == GPUDB_MEM_HOST) {
    if (clustered) host_clustered(a, static_cast<int32_t*>(dst));
    else host_generate(a, dst);
    return GPUDB_OK;
  }
  if (location != GPUDB_MEM_DEVICE) return fail(ctx, GPUDB_E_INVALID, "bad location");

  Call call(ctx, nullptr, nullptr);
  const unsigned grid = (unsigned)std::min<uint64_t>((a.n + 255) / 256, (uint64_t)ctx->sm_count * 16);
  if (!clustered) {
    GPUDB_LAUNCH(call, gen_column_kernel, grid, 256, 0, a, dst);
  } else {
    // every run ends at or after its first row, so runs 0..off+n-1 cover rows [0, off+n)
    const uint64_t runs = a.off + a.n;
    const uint64_t tiles = scan_tiles_count(runs);
    void *len = nullptr, *start = nullptr, *tmp = nullptr;
    int rc = scratch(ctx, "gen.len", runs, &len);
    if (!rc) rc = scratch(ctx, "gen.start", runs * sizeof(uint64_t), &start);
    if (!rc) rc = scratch(ctx, "gen.tmp", (tiles + 1) * sizeof(uint64_t), &tmp);
    if (rc) return rc;
    const unsigned rg = (unsigned)std::min<uint64_t>((runs + 255) / 256, (uint64_t)ctx->sm_count * 16);
    GPUDB_LAUNCH(call, run_lengths_kernel, rg, 256, 0, a.seed, runs, (uint8_t*)len);
    rc = exclusive_scan<uint8_t, uint64_t>(call, (const uint8_t*)len, runs, (uint64_t*)start,
                                           (uint64_t*)tmp, nullptr);
    if (rc) return rc;
    GPUDB_LAUNCH(call, run_fill_kernel, rg, 256, 0, (const uint8_t*)len, (const uint64_t*)start, runs,
                 a.off, a.n, a.n_orders, (int32_t*)dst);
  }
  GPUDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GPUDB_OK;
}
