// One host driver per operator pipeline, in the shape of the reference's runQnBenchmark
// functions (src/q1.cpp, src/q3.cpp, src/q6.cpp, src/q9.cpp, src/microbenchmarks.cpp):
// load (here: generate) the tables, run the pipeline three times and keep the third
// timing, print the exact result and the reference's timing lines. All device work goes
// through the C ABI (include/gpudb_capi.h).
#include <algorithm>
#include <cinttypes>
#include <cstring>

#include "infra.hpp"

namespace gpudb_host {
namespace {

// Fixed-point integer -> decimal text with `digits` fraction digits.
std::string fixed(__int128 v, int digits) {
  gpudb_i128 x{(uint64_t)(unsigned __int128)v, (int64_t)(v >> 64)};
  std::string s = i128_str(x);
  bool neg = !s.empty() && s[0] == '-';
  if (neg) s.erase(0, 1);
  while ((int)s.size() <= digits) s.insert(s.begin(), '0');
  s.insert(s.end() - digits, '.');
  return neg ? "-" + s : s;
}

__int128 as128(const gpudb_i128& v) { return ((__int128)v.hi << 64) | (__int128)v.lo; }

struct Lineitem {
  std::vector<Buffer> cols;
  gpudb_lineitem li{};
};

// The fact columns a pipeline needs; device-resident, or pinned host memory when streamed.
Lineitem make_lineitem(gpudb_ctx* ctx, const RunOptions& o, std::initializer_list<int32_t> ids, int32_t order_mode,
                       int64_t n_orders, int64_t n_parts, int64_t n_supp) {
  Lineitem L;
  gpudb_gen_spec spec{};
  spec.seed = o.seed;
  spec.n_rows = o.scale.lineitem;
  spec.n_orders = n_orders;
  spec.n_parts = n_parts;
  spec.n_supp = n_supp;
  spec.order_mode = order_mode;
  const int loc = o.scale.streamed ? GPUDB_MEM_HOST : GPUDB_MEM_DEVICE;
  L.li.n_rows = spec.n_rows;
  L.li.location = loc;
  L.li.order_key_max = n_orders > 0 ? (int32_t)(4 * (n_orders - 1) + 1) : -1;
  for (int32_t id : ids) {
    L.cols.push_back(generate(ctx, spec, id, loc));
    void* p = L.cols.back().as<void>();
    switch (id) {
      case GPUDB_COL_LI_SHIP_DATE: L.li.ship_date = (const int32_t*)p; break;
      case GPUDB_COL_LI_QUANTITY: L.li.quantity = (const int32_t*)p; break;
      case GPUDB_COL_LI_EXT_PRICE: L.li.ext_price = (const int64_t*)p; break;
      case GPUDB_COL_LI_DISCOUNT: L.li.discount = (const int32_t*)p; break;
      case GPUDB_COL_LI_TAX: L.li.tax = (const int32_t*)p; break;
      case GPUDB_COL_LI_FLAG: L.li.flag = (const uint8_t*)p; break;
      case GPUDB_COL_LI_STATUS: L.li.status = (const uint8_t*)p; break;
      case GPUDB_COL_LI_ORDER_KEY: L.li.order_key = (const int32_t*)p; break;
      case GPUDB_COL_LI_PART_KEY: L.li.part_key = (const int32_t*)p; break;
      case GPUDB_COL_LI_SUPP_KEY: L.li.supp_key = (const int32_t*)p; break;
    }
  }
  return L;
}

void header(const RunOptions& o, const char* q, uint64_t rows, const gpudb_timing& t, const char* suffix = "") {
  if (o.scale.streamed)
    std::printf("\nSF100 %s | %u chunks | %" PRIu64 " rows%s\n", q, t.chunks, rows, suffix);
  else
    std::printf("\n%s | %" PRIu64 " rows%s\n", q, rows, suffix);
}

}  // namespace

void runQ1Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("--- Running TPC-H Query 1 Benchmark ---\n");
  double t0 = now_ms();
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_SHIP_DATE, GPUDB_COL_LI_QUANTITY, GPUDB_COL_LI_EXT_PRICE,
                                      GPUDB_COL_LI_DISCOUNT, GPUDB_COL_LI_TAX, GPUDB_COL_LI_FLAG, GPUDB_COL_LI_STATUS},
                             GPUDB_ORDERS_NONE, 0, 0, 0);
  const double gen_ms = now_ms() - t0;
  gpudb_q1_params p{2436, 0};
  gpudb_q1_result r{};
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++) check(ctx, gpudb_q1_group6(ctx, &L.li, &p, &r, &t, nullptr), "gpudb_q1_group6");
  const double p0 = now_ms();
  std::printf("\n+----------+----------+------------+------------------+----------------------+---------------------------+------------+------------+----------+----------+\n");
  std::printf("| l_return | l_linest |    sum_qty |   sum_base_price |       sum_disc_price |                sum_charge |    avg_qty |  avg_price | avg_disc | count    |\n");
  std::printf("+----------+----------+------------+------------------+----------------------+---------------------------+------------+------------+----------+----------+\n");
  for (uint32_t i = 0; i < r.n_groups; i++) {
    const gpudb_q1_group& g = r.groups[i];
    const __int128 c = (__int128)g.count;
    // averages rounded half up to the printed digits, from the exact sums
    const __int128 avg_qty = (as128(g.sum_qty) * 100 + c / 2) / c;                 // 2 decimals
    const __int128 avg_price = (as128(g.sum_base_price) * 100 + c / 2) / c;        // hundredths -> 4 dec
    const __int128 avg_disc = (as128(g.sum_discount) * 100 + c / 2) / c;           // hundredths -> 4 dec
    std::printf("| %8c | %8c | %10s | %16s | %20s | %25s | %10s | %10s | %8s | %8" PRIu64 " |\n", "ANR"[g.flag],
                "FO"[g.status], i128_str(g.sum_qty).c_str(), fixed(as128(g.sum_base_price), 2).c_str(),
                fixed(as128(g.sum_disc_price), 4).c_str(), fixed(as128(g.sum_charge), 6).c_str(),
                fixed(avg_qty, 2).c_str(), fixed(avg_price, 4).c_str(), fixed(avg_disc, 4).c_str(), g.count);
  }
  std::printf("+----------+----------+------------+------------------+----------------------+---------------------------+------------+------------+----------+----------+\n");
  header(o, "Q1", L.li.n_rows, t);
  printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
  std::printf("  Bandwidth:          %10.2f GB/s\n", 26.0 * (double)L.li.n_rows / (t.gpu_ms * 1e6));
}

void runQ6Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("--- Running TPC-H Query 6 Benchmark ---\n");
  double t0 = now_ms();
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_SHIP_DATE, GPUDB_COL_LI_DISCOUNT, GPUDB_COL_LI_QUANTITY,
                                      GPUDB_COL_LI_EXT_PRICE}, GPUDB_ORDERS_NONE, 0, 0, 0);
  const double gen_ms = now_ms() - t0;
  gpudb_q6_params p{365, 730, 5, 7, 24};
  gpudb_q6_result r{};
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++) check(ctx, gpudb_q6_sum(ctx, &L.li, &p, &r, &t, nullptr), "gpudb_q6_sum");
  const double p0 = now_ms();
  std::printf("TPC-H Query 6 Result:\n");
  std::printf("Total Revenue: $%s\n", fixed(r.revenue, 4).c_str());
  std::printf("Rows matched: %" PRIu64 "\n", r.rows_matched);
  header(o, "Q6", L.li.n_rows, t);
  printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
  std::printf("  Bandwidth:          %10.2f GB/s\n", 20.0 * (double)L.li.n_rows / (t.gpu_ms * 1e6));
}

void runQ3Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("\n--- Running TPC-H Query 3 Benchmark ---\n");
  const Scale& s = o.scale;
  double t0 = now_ms();
  gpudb_gen_spec cs{};
  cs.seed = o.seed;
  cs.n_rows = s.customer;
  Buffer ck = generate(ctx, cs, GPUDB_COL_CU_CUST_KEY, GPUDB_MEM_DEVICE);
  Buffer cg = generate(ctx, cs, GPUDB_COL_CU_SEGMENT, GPUDB_MEM_DEVICE);
  gpudb_gen_spec os = cs;
  os.n_rows = s.orders;
  os.n_cust = (int64_t)s.customer;
  Buffer ok = generate(ctx, os, GPUDB_COL_OR_ORDER_KEY, GPUDB_MEM_DEVICE);
  Buffer oc = generate(ctx, os, GPUDB_COL_OR_CUST_KEY, GPUDB_MEM_DEVICE);
  Buffer od = generate(ctx, os, GPUDB_COL_OR_ORDER_DATE, GPUDB_MEM_DEVICE);
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_ORDER_KEY, GPUDB_COL_LI_SHIP_DATE, GPUDB_COL_LI_EXT_PRICE,
                                      GPUDB_COL_LI_DISCOUNT}, GPUDB_ORDERS_CLUSTERED, (int64_t)s.orders, 0, 0);
  const double gen_ms = now_ms() - t0;
  std::printf("Loaded %" PRIu64 " customers, %" PRIu64 " orders, %" PRIu64 " lineitem rows.\n", s.customer, s.orders,
              s.lineitem);
  gpudb_customer cu{s.customer, (int32_t)s.customer - 1, 0, ck.as<int32_t>(), cg.as<uint8_t>()};
  gpudb_orders orr{s.orders, (int32_t)(4 * (s.orders - 1) + 1), (int32_t)s.customer - 1, ok.as<int32_t>(),
                   oc.as<int32_t>(), od.as<int32_t>()};
  for (int mode : {GPUDB_JOIN_GLOBAL, GPUDB_JOIN_RADIX}) {
    gpudb_q3_params p{1, 1170, 1170, 10, mode, 0};
    gpudb_q3_result r{};
    gpudb_timing t{};
    for (int i = 0; i < o.reps; i++) check(ctx, gpudb_q3_join_topk(ctx, &cu, &orr, &L.li, &p, &r, &t, nullptr), "gpudb_q3");
    const double p0 = now_ms();
    std::printf("\nTPC-H Q3 Results (Top 10, %s join):\n", mode == GPUDB_JOIN_GLOBAL ? "global hash table" : "radix partitioned");
    std::printf("+----------+------------------+------------+--------------+\n");
    std::printf("| orderkey |          revenue | orderdate  | shippriority |\n");
    std::printf("+----------+------------------+------------+--------------+\n");
    for (uint32_t i = 0; i < r.n_rows; i++)
      std::printf("| %8d | $%15s | %10d | %12d |\n", r.rows[i].order_key, fixed(r.rows[i].revenue, 4).c_str(),
                  r.rows[i].order_date, 0);
    std::printf("+----------+------------------+------------+--------------+\n");
    std::printf("Total results found: %" PRIu64 "\n", r.n_groups);
    header(o, "Q3", L.li.n_rows, t, mode == GPUDB_JOIN_GLOBAL ? " (lineitem)" : " (lineitem, radix)");
    printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
  }
}

void runQ9Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("\n--- Running TPC-H Query 9 Benchmark ---\n");
  const Scale& s = o.scale;
  double t0 = now_ms();
  gpudb_gen_spec ps{};
  ps.seed = o.seed;
  ps.n_rows = s.part;
  Buffer pk = generate(ctx, ps, GPUDB_COL_PA_PART_KEY, GPUDB_MEM_DEVICE);
  Buffer pf = generate(ctx, ps, GPUDB_COL_PA_FLAG, GPUDB_MEM_DEVICE);
  gpudb_gen_spec ss = ps;
  ss.n_rows = s.supplier;
  Buffer sk = generate(ctx, ss, GPUDB_COL_SU_SUPP_KEY, GPUDB_MEM_DEVICE);
  Buffer sn = generate(ctx, ss, GPUDB_COL_SU_NATION, GPUDB_MEM_DEVICE);
  gpudb_gen_spec pss = ps;
  pss.n_rows = 4 * s.part;
  pss.n_supp = (int64_t)s.supplier;
  Buffer psp = generate(ctx, pss, GPUDB_COL_PS_PART_KEY, GPUDB_MEM_DEVICE);
  Buffer pssk = generate(ctx, pss, GPUDB_COL_PS_SUPP_KEY, GPUDB_MEM_DEVICE);
  Buffer psc = generate(ctx, pss, GPUDB_COL_PS_SUPPLY_COST, GPUDB_MEM_DEVICE);
  gpudb_gen_spec os = ps;
  os.n_rows = s.orders;
  Buffer ok = generate(ctx, os, GPUDB_COL_OR_ORDER_KEY, GPUDB_MEM_DEVICE);
  Buffer od = generate(ctx, os, GPUDB_COL_OR_ORDER_DATE, GPUDB_MEM_DEVICE);
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_PART_KEY, GPUDB_COL_LI_SUPP_KEY, GPUDB_COL_LI_ORDER_KEY,
                                      GPUDB_COL_LI_EXT_PRICE, GPUDB_COL_LI_DISCOUNT, GPUDB_COL_LI_QUANTITY},
                             GPUDB_ORDERS_UNIFORM, (int64_t)s.orders, (int64_t)s.part, (int64_t)s.supplier);
  const double gen_ms = now_ms() - t0;
  gpudb_part pa{s.part, (int32_t)s.part - 1, 0, pk.as<int32_t>(), pf.as<uint8_t>()};
  gpudb_supplier su{s.supplier, (int32_t)s.supplier - 1, 0, sk.as<int32_t>(), sn.as<uint8_t>()};
  gpudb_partsupp pt{4 * s.part, psp.as<int32_t>(), pssk.as<int32_t>(), psc.as<int64_t>()};
  gpudb_orders orr{s.orders, (int32_t)(4 * (s.orders - 1) + 1), 0, ok.as<int32_t>(), nullptr, od.as<int32_t>()};
  std::vector<gpudb_q9_group> groups(4096);
  uint32_t n = 0;
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++)
    check(ctx, gpudb_q9_star(ctx, &pa, &su, &pt, &orr, &L.li, nullptr, groups.data(), 4096, &n, &t, nullptr), "gpudb_q9");
  const double p0 = now_ms();
  std::printf("\nTPC-H Query 9 Results (Top 15):\n");
  std::printf("+--------+------+------------------------+\n");
  std::printf("| Nation | Year |                 Profit |\n");
  std::printf("+--------+------+------------------------+\n");
  for (uint32_t i = 0; i < n && i < 15; i++)
    std::printf("| %6d | %4d | $%21s |\n", groups[i].nation, groups[i].year, fixed(groups[i].profit, 4).c_str());
  std::printf("+--------+------+------------------------+\n");
  std::printf("Total results found: %u\n", n);
  header(o, "Q9", L.li.n_rows, t);
  printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
}

void runSelectionBenchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("--- Running Selection Benchmark ---\n");
  gpudb_gen_spec spec{};
  spec.seed = o.seed;
  spec.n_rows = o.scale.lineitem;
  Buffer col = generate(ctx, spec, GPUDB_COL_LI_SHIP_DATE, GPUDB_MEM_DEVICE);
  Buffer bits(ctx, ((spec.n_rows + 31) / 32) * 4, GPUDB_MEM_DEVICE);
  std::printf("Loaded %" PRIu64 " rows for selection.\n", spec.n_rows);
  for (int32_t v : {100, 1000, 2000}) {
    uint64_t c = 0;
    gpudb_timing t{};
    for (int i = 0; i < o.reps; i++)
      check(ctx, gpudb_select_lt(ctx, col.as<int32_t>(), spec.n_rows, v, bits.as<uint32_t>(), nullptr, &c, &t, nullptr),
            "gpudb_select_lt");
    std::printf("--- Filter Value: < %d ---\n", v);
    std::printf("Selectivity: %.4f%% (%" PRIu64 " rows matched)\n", 100.0 * (double)c / (double)spec.n_rows, c);
    std::printf("GPU execution time: %.4f ms\n", t.gpu_ms);
    std::printf("Effective Bandwidth: %.2f GB/s\n\n", 4.125 * (double)spec.n_rows / (t.gpu_ms * 1e6));
  }
}

void runAggregationBenchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("--- Running Aggregation Benchmark ---\n");
  gpudb_gen_spec spec{};
  spec.seed = o.seed;
  spec.n_rows = o.scale.lineitem;
  Buffer col = generate(ctx, spec, GPUDB_COL_LI_QUANTITY, GPUDB_MEM_DEVICE);
  std::printf("Loaded %" PRIu64 " rows for aggregation.\n", spec.n_rows);
  int64_t sum = 0;
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++) check(ctx, gpudb_sum_i32(ctx, col.as<int32_t>(), spec.n_rows, &sum, &t, nullptr), "gpudb_sum_i32");
  std::printf("Final SUM(l_quantity): %" PRId64 "\n", sum);
  std::printf("GPU execution time: %.4f ms\n", t.gpu_ms);
  std::printf("Effective Bandwidth: %.2f GB/s\n\n", 4.0 * (double)spec.n_rows / (t.gpu_ms * 1e6));
}

void runJoinBenchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("--- Running Join Benchmark ---\n");
  gpudb_gen_spec bs{};
  bs.seed = o.seed;
  bs.n_rows = o.scale.orders;
  Buffer build = generate(ctx, bs, GPUDB_COL_OR_ORDER_KEY, GPUDB_MEM_DEVICE);
  gpudb_gen_spec ps = bs;
  ps.n_rows = o.scale.lineitem;
  ps.n_orders = (int64_t)o.scale.orders;
  ps.order_mode = GPUDB_ORDERS_CLUSTERED;
  Buffer probe = generate(ctx, ps, GPUDB_COL_LI_ORDER_KEY, GPUDB_MEM_DEVICE);
  std::printf("Loaded %" PRIu64 " rows for build phase, %" PRIu64 " rows for probe phase.\n", bs.n_rows, ps.n_rows);
  for (int mode : {GPUDB_JOIN_GLOBAL, GPUDB_JOIN_RADIX}) {
    uint64_t m = 0;
    gpudb_timing t{};
    for (int i = 0; i < o.reps; i++)
      check(ctx, gpudb_hash_join_count(ctx, build.as<int32_t>(), bs.n_rows, probe.as<int32_t>(), ps.n_rows, mode, &m, &t, nullptr),
            "gpudb_hash_join_count");
    std::printf("Join (%s) complete. Found %" PRIu64 " total matches.\n", mode == GPUDB_JOIN_GLOBAL ? "global table" : "radix partitioned", m);
    std::printf("Total Join GPU time: %.4f ms\n\n", t.gpu_ms);
  }
}

}  // namespace gpudb_host
