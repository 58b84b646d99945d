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

// Column id -> (position in gpudb_tbl_parse's lineitem columns, width).
std::pair<int, int> li_tbl_column(int32_t id) {
  switch (id) {
    case GPUDB_COL_LI_ORDER_KEY: return {0, 4};
    case GPUDB_COL_LI_PART_KEY: return {1, 4};
    case GPUDB_COL_LI_SUPP_KEY: return {2, 4};
    case GPUDB_COL_LI_QUANTITY: return {3, 4};
    case GPUDB_COL_LI_EXT_PRICE: return {4, 8};
    case GPUDB_COL_LI_DISCOUNT: return {5, 4};
    case GPUDB_COL_LI_TAX: return {6, 4};
    case GPUDB_COL_LI_FLAG: return {7, 1};
    case GPUDB_COL_LI_STATUS: return {8, 1};
    case GPUDB_COL_LI_COMMIT_DATE: return {10, 4};
    case GPUDB_COL_LI_RECEIPT_DATE: return {11, 4};
    case GPUDB_COL_LI_SHIP_MODE: return {12, 1};
    default: return {9, 4};   // ship date
  }
}

void set_li_column(gpudb_lineitem& li, int32_t id, void* p) {
  switch (id) {
    case GPUDB_COL_LI_SHIP_DATE: li.ship_date = (const int32_t*)p; break;
    case GPUDB_COL_LI_QUANTITY: li.quantity = (const int32_t*)p; break;
    case GPUDB_COL_LI_EXT_PRICE: li.ext_price = (const int64_t*)p; break;
    case GPUDB_COL_LI_DISCOUNT: li.discount = (const int32_t*)p; break;
    case GPUDB_COL_LI_TAX: li.tax = (const int32_t*)p; break;
    case GPUDB_COL_LI_FLAG: li.flag = (const uint8_t*)p; break;
    case GPUDB_COL_LI_STATUS: li.status = (const uint8_t*)p; break;
    case GPUDB_COL_LI_ORDER_KEY: li.order_key = (const int32_t*)p; break;
    case GPUDB_COL_LI_PART_KEY: li.part_key = (const int32_t*)p; break;
    case GPUDB_COL_LI_SUPP_KEY: li.supp_key = (const int32_t*)p; break;
    case GPUDB_COL_LI_COMMIT_DATE: li.commit_date = (const int32_t*)p; break;
    case GPUDB_COL_LI_RECEIPT_DATE: li.receipt_date = (const int32_t*)p; break;
    case GPUDB_COL_LI_SHIP_MODE: li.ship_mode = (const uint8_t*)p; break;
  }
}

// Orders with key, date and priority (Q4, Q12): generated, or parsed from orders.tbl.
struct OrdersKDP {
  gpudb_orders od{};
  TblTable t;
  Buffer key, date, prio;
};

void make_orders_kdp(gpudb_ctx* ctx, const RunOptions& o, OrdersKDP& O) {
  if (!o.data_dir.empty()) {
    O.t = load_tbl(ctx, o.data_dir, "orders", GPUDB_TBL_ORDERS, {0, 2, 3}, {4, 4, 1}, o.tbl_piece);
    O.od = {O.t.rows, O.t.col_max[0], 0, O.t.col<int32_t>(0), nullptr, O.t.col<int32_t>(2), O.t.col<uint8_t>(3)};
    return;
  }
  gpudb_gen_spec os{};
  os.seed = o.seed;
  os.n_rows = o.scale.orders;
  O.key = generate(ctx, os, GPUDB_COL_OR_ORDER_KEY, GPUDB_MEM_DEVICE);
  O.date = generate(ctx, os, GPUDB_COL_OR_ORDER_DATE, GPUDB_MEM_DEVICE);
  O.prio = generate(ctx, os, GPUDB_COL_OR_PRIORITY, GPUDB_MEM_DEVICE);
  O.od = {o.scale.orders, (int32_t)(4 * (o.scale.orders - 1) + 1), 0, O.key.as<int32_t>(), nullptr,
          O.date.as<int32_t>(), O.prio.as<uint8_t>()};
}

// The fact columns a pipeline needs: generated (device-resident, or pinned host memory when
// streamed), or parsed from <data_dir>/lineitem.tbl into device memory.
Lineitem make_lineitem(gpudb_ctx* ctx, const RunOptions& o, std::initializer_list<int32_t> ids, int32_t order_mode,
                       int64_t n_orders, int64_t n_parts, int64_t n_supp) {
  Lineitem L;
  if (!o.data_dir.empty()) {
    std::vector<int> keep, widths;
    for (int32_t id : ids) {
      keep.push_back(li_tbl_column(id).first);
      widths.push_back(li_tbl_column(id).second);
    }
    TblTable t = load_tbl(ctx, o.data_dir, "lineitem", GPUDB_TBL_LINEITEM, keep, widths, o.tbl_piece);
    L.li.n_rows = t.rows;
    L.li.location = GPUDB_MEM_DEVICE;
    L.li.order_key_max = t.col_max[0];
    for (int32_t id : ids) set_li_column(L.li, id, t.cols[li_tbl_column(id).first].as<void>());
    for (auto& b : t.cols)
      if (b.bytes()) L.cols.push_back(std::move(b));
    return L;
  }
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
    set_li_column(L.li, id, L.cols.back().as<void>());
  }
  return L;
}

void q9_report(gpudb_ctx* ctx, const RunOptions& o, const gpudb_part& pa, const gpudb_supplier& su,
               const gpudb_partsupp& pt, const gpudb_orders& orr, const Lineitem& L, double gen_ms);

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
  gpudb_customer cu{};
  gpudb_orders orr{};
  TblTable ct, ot;
  Buffer ck, cg, ok, oc, od;
  if (!o.data_dir.empty()) {
    ct = load_tbl(ctx, o.data_dir, "customer", GPUDB_TBL_CUSTOMER, {0, 2}, {4, 1}, o.tbl_piece);
    ot = load_tbl(ctx, o.data_dir, "orders", GPUDB_TBL_ORDERS, {0, 1, 2}, {4, 4, 4}, o.tbl_piece);
    cu = {ct.rows, ct.col_max[0], 0, ct.col<int32_t>(0), ct.col<uint8_t>(2)};
    orr = {ot.rows, ot.col_max[0], ot.col_max[1], ot.col<int32_t>(0), ot.col<int32_t>(1), ot.col<int32_t>(2)};
  } else {
    gpudb_gen_spec cs{};
    cs.seed = o.seed;
    cs.n_rows = s.customer;
    ck = generate(ctx, cs, GPUDB_COL_CU_CUST_KEY, GPUDB_MEM_DEVICE);
    cg = generate(ctx, cs, GPUDB_COL_CU_SEGMENT, GPUDB_MEM_DEVICE);
    gpudb_gen_spec os = cs;
    os.n_rows = s.orders;
    os.n_cust = (int64_t)s.customer;
    ok = generate(ctx, os, GPUDB_COL_OR_ORDER_KEY, GPUDB_MEM_DEVICE);
    oc = generate(ctx, os, GPUDB_COL_OR_CUST_KEY, GPUDB_MEM_DEVICE);
    od = generate(ctx, os, GPUDB_COL_OR_ORDER_DATE, GPUDB_MEM_DEVICE);
    cu = {s.customer, (int32_t)s.customer - 1, 0, ck.as<int32_t>(), cg.as<uint8_t>()};
    orr = {s.orders, (int32_t)(4 * (s.orders - 1) + 1), (int32_t)s.customer - 1, ok.as<int32_t>(), oc.as<int32_t>(),
           od.as<int32_t>()};
  }
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_ORDER_KEY, GPUDB_COL_LI_SHIP_DATE, GPUDB_COL_LI_EXT_PRICE,
                                      GPUDB_COL_LI_DISCOUNT}, GPUDB_ORDERS_CLUSTERED, (int64_t)s.orders, 0, 0);
  const double gen_ms = now_ms() - t0;
  std::printf("Loaded %" PRIu64 " customers, %" PRIu64 " orders, %" PRIu64 " lineitem rows.\n", cu.n_rows, orr.n_rows,
              L.li.n_rows);
  // AUTO first: the direct map when the orders' key range fits 30% of device memory (the
  // reference's choice, src/q3.cpp:246), else the hash table; then the other two modes
  for (int mode : {GPUDB_JOIN_AUTO, GPUDB_JOIN_GLOBAL, GPUDB_JOIN_RADIX}) {
    gpudb_q3_params p{1, 1170, 1170, 10, mode, 0};
    gpudb_q3_result r{};
    gpudb_timing t{};
    for (int i = 0; i < o.reps; i++) check(ctx, gpudb_q3_join_topk(ctx, &cu, &orr, &L.li, &p, &r, &t, nullptr), "gpudb_q3");
    const double p0 = now_ms();
    const char* name = r.join_mode == GPUDB_JOIN_DIRECT ? "direct map" : r.join_mode == GPUDB_JOIN_RADIX
                                                                            ? "radix partitioned" : "global hash table";
    if (mode == GPUDB_JOIN_AUTO)
      std::printf("Orders map: %d entries (%.1f MB): using the %s join\n", orr.key_max + 1,
                  (orr.key_max + 1) * 4.0 / (1024.0 * 1024.0), name);
    std::printf("\nTPC-H Q3 Results (Top 10, %s join):\n", name);
    std::printf("+----------+------------------+------------+--------------+\n");
    std::printf("| orderkey |          revenue | orderdate  | shippriority |\n");
    std::printf("+----------+------------------+------------+--------------+\n");
    for (uint32_t i = 0; i < r.n_rows; i++)
      std::printf("| %8d | $%15s | %10d | %12d |\n", r.rows[i].order_key, fixed(r.rows[i].revenue, 4).c_str(),
                  r.rows[i].order_date, 0);
    std::printf("+----------+------------------+------------+--------------+\n");
    std::printf("Total results found: %" PRIu64 "\n", r.n_groups);
    header(o, "Q3", L.li.n_rows, t, r.join_mode == GPUDB_JOIN_GLOBAL ? " (lineitem)"
                                    : r.join_mode == GPUDB_JOIN_DIRECT ? " (lineitem, direct)" : " (lineitem, radix)");
    printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
  }
}

void runQ4Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("\n--- Running TPC-H Query 4 Benchmark ---\n");
  const double t0 = now_ms();
  OrdersKDP O;
  make_orders_kdp(ctx, o, O);
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_ORDER_KEY, GPUDB_COL_LI_COMMIT_DATE, GPUDB_COL_LI_RECEIPT_DATE},
                             GPUDB_ORDERS_CLUSTERED, (int64_t)O.od.n_rows, 0, 0);
  const double gen_ms = now_ms() - t0;
  std::printf("Loaded %" PRIu64 " lineitem, %" PRIu64 " orders rows for Q4.\n", L.li.n_rows, O.od.n_rows);
  const gpudb_q4_params p{547, 639};   // 1993-07-01 <= o_orderdate < 1993-10-01
  gpudb_q4_result r{};
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++) check(ctx, gpudb_q4_priority(ctx, &O.od, &L.li, &p, &r, &t, nullptr), "gpudb_q4");
  const double p0 = now_ms();
  static const char* names[5] = {"1-URGENT", "2-HIGH", "3-MEDIUM", "4-NOT SPECIFIED", "5-LOW"};
  std::printf("\nTPC-H Q4 Results:\n");
  std::printf("+------------------+-------------+\n");
  std::printf("| o_orderpriority  | order_count |\n");
  std::printf("+------------------+-------------+\n");
  for (int i = 0; i < 5; i++) std::printf("| %-16s | %11" PRIu64 " |\n", names[i], r.count[i]);
  std::printf("+------------------+-------------+\n");
  if (o.scale.streamed) header(o, "Q4", L.li.n_rows, t);
  else std::printf("\nQ4 | %" PRIu64 " lineitem, %" PRIu64 " orders\n", L.li.n_rows, O.od.n_rows);
  printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
}

void runQ12Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("\n--- Running TPC-H Query 12 Benchmark ---\n");
  const double t0 = now_ms();
  OrdersKDP O;
  make_orders_kdp(ctx, o, O);
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_ORDER_KEY, GPUDB_COL_LI_SHIP_DATE, GPUDB_COL_LI_COMMIT_DATE,
                                      GPUDB_COL_LI_RECEIPT_DATE, GPUDB_COL_LI_SHIP_MODE},
                             GPUDB_ORDERS_CLUSTERED, (int64_t)O.od.n_rows, 0, 0);
  const double gen_ms = now_ms() - t0;
  std::printf("Loaded %" PRIu64 " orders, %" PRIu64 " lineitem rows for Q12.\n", O.od.n_rows, L.li.n_rows);
  // 1994-01-01 <= l_receiptdate < 1995-01-01, MAIL and SHIP, priorities 1-URGENT and 2-HIGH
  const gpudb_q12_params p{731, 1096, {GPUDB_MODE_MAIL, GPUDB_MODE_SHIP}, 2, 0};
  gpudb_q12_result r{};
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++) check(ctx, gpudb_q12_shipmode(ctx, &O.od, &L.li, &p, &r, &t, nullptr), "gpudb_q12");
  const double p0 = now_ms();
  std::printf("\nTPC-H Q12 Results:\n");
  std::printf("+----------+------------------+-----------------+\n");
  std::printf("| shipmode | high_line_count  | low_line_count  |\n");
  std::printf("+----------+------------------+-----------------+\n");
  std::printf("| MAIL     | %16" PRIu64 " | %15" PRIu64 " |\n", r.high[0], r.low[0]);
  std::printf("| SHIP     | %16" PRIu64 " | %15" PRIu64 " |\n", r.high[1], r.low[1]);
  std::printf("+----------+------------------+-----------------+\n");
  header(o, "Q12", L.li.n_rows, t);
  printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
}

namespace {
// TPC-H nation table names by nation key (Q5, Q7 output).
const char* const kNationNames[GPUDB_NATIONS] = {
    "ALGERIA", "ARGENTINA", "BRAZIL", "CANADA", "EGYPT", "ETHIOPIA", "FRANCE", "GERMANY", "INDIA",
    "INDONESIA", "IRAN", "IRAQ", "JAPAN", "JORDAN", "KENYA", "MOROCCO", "MOZAMBIQUE", "PERU", "CHINA",
    "ROMANIA", "SAUDI ARABIA", "VIETNAM", "RUSSIA", "UNITED KINGDOM", "UNITED STATES"};
}  // namespace

void runQ5Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("\n--- Running TPC-H Query 5 Benchmark ---\n");
  const Scale& s = o.scale;
  const double t0 = now_ms();
  gpudb_customer cu{};
  gpudb_supplier su{};
  gpudb_orders orr{};
  TblTable ct, st, ot;
  Buffer ck, cn, sk, sn, ok, oc, od;
  if (!o.data_dir.empty()) {
    ct = load_tbl(ctx, o.data_dir, "customer", GPUDB_TBL_CUSTOMER, {0, 1}, {4, 1}, o.tbl_piece);
    st = load_tbl(ctx, o.data_dir, "supplier", GPUDB_TBL_SUPPLIER, {0, 1}, {4, 1}, o.tbl_piece);
    ot = load_tbl(ctx, o.data_dir, "orders", GPUDB_TBL_ORDERS, {0, 1, 2}, {4, 4, 4}, o.tbl_piece);
    cu = {ct.rows, ct.col_max[0], 0, ct.col<int32_t>(0), nullptr, ct.col<uint8_t>(1)};
    su = {st.rows, st.col_max[0], 0, st.col<int32_t>(0), st.col<uint8_t>(1)};
    orr = {ot.rows, ot.col_max[0], ot.col_max[1], ot.col<int32_t>(0), ot.col<int32_t>(1), ot.col<int32_t>(2)};
  } else {
    gpudb_gen_spec cs{};
    cs.seed = o.seed;
    cs.n_rows = s.customer;
    ck = generate(ctx, cs, GPUDB_COL_CU_CUST_KEY, GPUDB_MEM_DEVICE);
    cn = generate(ctx, cs, GPUDB_COL_CU_NATION, GPUDB_MEM_DEVICE);
    gpudb_gen_spec ss = cs;
    ss.n_rows = s.supplier;
    sk = generate(ctx, ss, GPUDB_COL_SU_SUPP_KEY, GPUDB_MEM_DEVICE);
    sn = generate(ctx, ss, GPUDB_COL_SU_NATION, GPUDB_MEM_DEVICE);
    gpudb_gen_spec os = cs;
    os.n_rows = s.orders;
    os.n_cust = (int64_t)s.customer;
    ok = generate(ctx, os, GPUDB_COL_OR_ORDER_KEY, GPUDB_MEM_DEVICE);
    oc = generate(ctx, os, GPUDB_COL_OR_CUST_KEY, GPUDB_MEM_DEVICE);
    od = generate(ctx, os, GPUDB_COL_OR_ORDER_DATE, GPUDB_MEM_DEVICE);
    cu = {s.customer, (int32_t)s.customer - 1, 0, ck.as<int32_t>(), nullptr, cn.as<uint8_t>()};
    su = {s.supplier, (int32_t)s.supplier - 1, 0, sk.as<int32_t>(), sn.as<uint8_t>()};
    orr = {s.orders, (int32_t)(4 * (s.orders - 1) + 1), (int32_t)s.customer - 1, ok.as<int32_t>(), oc.as<int32_t>(),
           od.as<int32_t>()};
  }
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_ORDER_KEY, GPUDB_COL_LI_SUPP_KEY, GPUDB_COL_LI_EXT_PRICE,
                                      GPUDB_COL_LI_DISCOUNT}, GPUDB_ORDERS_CLUSTERED, (int64_t)orr.n_rows,
                             (int64_t)s.part, (int64_t)su.n_rows);
  const double gen_ms = now_ms() - t0;
  std::printf("Loaded %" PRIu64 " customers, %" PRIu64 " suppliers, %" PRIu64 " orders, %" PRIu64 " lineitem rows.\n",
              cu.n_rows, su.n_rows, orr.n_rows, L.li.n_rows);
  // ASIA (TPC-H nation table: INDIA, INDONESIA, JAPAN, CHINA, VIETNAM), orders of 1994
  const gpudb_q5_params p{731, 1096, (1u << 8) | (1u << 9) | (1u << 12) | (1u << 18) | (1u << 21), 0};
  gpudb_q5_result r{};
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++) check(ctx, gpudb_q5_local_supplier(ctx, &cu, &su, &orr, &L.li, &p, &r, &t, nullptr), "gpudb_q5");
  const double p0 = now_ms();
  std::vector<int> order;
  for (int n = 0; n < GPUDB_NATIONS; n++)
    if (r.revenue[n]) order.push_back(n);
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    return r.revenue[a] != r.revenue[b] ? r.revenue[a] > r.revenue[b] : a < b;
  });
  std::printf("\nTPC-H Q5 Results:\n");
  std::printf("+----------------+---------------------+\n");
  std::printf("| n_name         |             revenue |\n");
  std::printf("+----------------+---------------------+\n");
  for (int n : order) std::printf("| %-14s | $%18s |\n", kNationNames[n], fixed(r.revenue[n], 4).c_str());
  std::printf("+----------------+---------------------+\n");
  std::printf("\nQ5 | %" PRIu64 " rows (lineitem)\n", L.li.n_rows);
  printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
}

namespace {
// Customer (key, nation), supplier (key, nation) and orders (key, customer, date): generated,
// or parsed from the .tbl files (Q7, Q8).
struct Dims {
  gpudb_customer cu{};
  gpudb_supplier su{};
  gpudb_orders od{};
  TblTable ct, st, ot;
  Buffer ck, cn, sk, sn, ok, oc, odt;
};

void make_dims(gpudb_ctx* ctx, const RunOptions& o, Dims& D) {
  const Scale& s = o.scale;
  if (!o.data_dir.empty()) {
    D.ct = load_tbl(ctx, o.data_dir, "customer", GPUDB_TBL_CUSTOMER, {0, 1}, {4, 1}, o.tbl_piece);
    D.st = load_tbl(ctx, o.data_dir, "supplier", GPUDB_TBL_SUPPLIER, {0, 1}, {4, 1}, o.tbl_piece);
    D.ot = load_tbl(ctx, o.data_dir, "orders", GPUDB_TBL_ORDERS, {0, 1, 2}, {4, 4, 4}, o.tbl_piece);
    D.cu = {D.ct.rows, D.ct.col_max[0], 0, D.ct.col<int32_t>(0), nullptr, D.ct.col<uint8_t>(1)};
    D.su = {D.st.rows, D.st.col_max[0], 0, D.st.col<int32_t>(0), D.st.col<uint8_t>(1)};
    D.od = {D.ot.rows, D.ot.col_max[0], D.ot.col_max[1], D.ot.col<int32_t>(0), D.ot.col<int32_t>(1),
            D.ot.col<int32_t>(2)};
    return;
  }
  gpudb_gen_spec cs{};
  cs.seed = o.seed;
  cs.n_rows = s.customer;
  D.ck = generate(ctx, cs, GPUDB_COL_CU_CUST_KEY, GPUDB_MEM_DEVICE);
  D.cn = generate(ctx, cs, GPUDB_COL_CU_NATION, GPUDB_MEM_DEVICE);
  gpudb_gen_spec ss = cs;
  ss.n_rows = s.supplier;
  D.sk = generate(ctx, ss, GPUDB_COL_SU_SUPP_KEY, GPUDB_MEM_DEVICE);
  D.sn = generate(ctx, ss, GPUDB_COL_SU_NATION, GPUDB_MEM_DEVICE);
  gpudb_gen_spec os = cs;
  os.n_rows = s.orders;
  os.n_cust = (int64_t)s.customer;
  D.ok = generate(ctx, os, GPUDB_COL_OR_ORDER_KEY, GPUDB_MEM_DEVICE);
  D.oc = generate(ctx, os, GPUDB_COL_OR_CUST_KEY, GPUDB_MEM_DEVICE);
  D.odt = generate(ctx, os, GPUDB_COL_OR_ORDER_DATE, GPUDB_MEM_DEVICE);
  D.cu = {s.customer, (int32_t)s.customer - 1, 0, D.ck.as<int32_t>(), nullptr, D.cn.as<uint8_t>()};
  D.su = {s.supplier, (int32_t)s.supplier - 1, 0, D.sk.as<int32_t>(), D.sn.as<uint8_t>()};
  D.od = {s.orders, (int32_t)(4 * (s.orders - 1) + 1), (int32_t)s.customer - 1, D.ok.as<int32_t>(),
          D.oc.as<int32_t>(), D.odt.as<int32_t>()};
}
}  // namespace

void runQ7Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("\n--- Running TPC-H Query 7 Benchmark ---\n");
  const double t0 = now_ms();
  Dims D;
  make_dims(ctx, o, D);
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_ORDER_KEY, GPUDB_COL_LI_SUPP_KEY, GPUDB_COL_LI_SHIP_DATE,
                                      GPUDB_COL_LI_EXT_PRICE, GPUDB_COL_LI_DISCOUNT}, GPUDB_ORDERS_CLUSTERED,
                             (int64_t)D.od.n_rows, (int64_t)o.scale.part, (int64_t)D.su.n_rows);
  const double gen_ms = now_ms() - t0;
  const gpudb_q7_params p{6, 7, 1096, 1826};   // FRANCE and GERMANY, shipped 1995-01-01 .. 1996-12-31
  gpudb_q7_result r{};
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++) check(ctx, gpudb_q7_volume_shipping(ctx, &D.cu, &D.su, &D.od, &L.li, &p, &r, &t, nullptr), "gpudb_q7");
  const double p0 = now_ms();
  std::printf("\nTPC-H Q7 Results:\n");
  std::printf("+-------------+-------------+--------+---------------------+\n");
  std::printf("| supp_nation | cust_nation | l_year |             revenue |\n");
  std::printf("+-------------+-------------+--------+---------------------+\n");
  const int pairs[2][2] = {{p.nation_a, p.nation_b}, {p.nation_b, p.nation_a}};
  const int first = std::strcmp(kNationNames[p.nation_a], kNationNames[p.nation_b]) <= 0 ? 0 : 1;
  for (int q = 0; q < 2; q++) {
    const int pair = q == 0 ? first : 1 - first;
    for (int y = 0; y < r.n_years; y++)
      if (r.revenue[pair][y])
        std::printf("| %-11s | %-11s | %6d | $%18s |\n", kNationNames[pairs[pair][0]], kNationNames[pairs[pair][1]],
                    r.first_year + y, fixed(r.revenue[pair][y], 4).c_str());
  }
  std::printf("+-------------+-------------+--------+---------------------+\n");
  header(o, "Q7", L.li.n_rows, t);
  printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
}

void runQ8Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("\n--- Running TPC-H Query 8 Benchmark ---\n");
  const double t0 = now_ms();
  Dims D;
  make_dims(ctx, o, D);
  gpudb_part pa{};
  TblTable pt;
  Buffer pk, ptype;
  if (!o.data_dir.empty()) {
    pt = load_tbl(ctx, o.data_dir, "part", GPUDB_TBL_PART, {0, 2}, {4, 1}, o.tbl_piece);
    pa = {pt.rows, pt.col_max[0], 0, pt.col<int32_t>(0), nullptr, pt.col<uint8_t>(2)};
  } else {
    gpudb_gen_spec ps{};
    ps.seed = o.seed;
    ps.n_rows = o.scale.part;
    pk = generate(ctx, ps, GPUDB_COL_PA_PART_KEY, GPUDB_MEM_DEVICE);
    ptype = generate(ctx, ps, GPUDB_COL_PA_TYPE, GPUDB_MEM_DEVICE);
    pa = {o.scale.part, (int32_t)o.scale.part - 1, 0, pk.as<int32_t>(), nullptr, ptype.as<uint8_t>()};
  }
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_ORDER_KEY, GPUDB_COL_LI_PART_KEY, GPUDB_COL_LI_SUPP_KEY,
                                      GPUDB_COL_LI_EXT_PRICE, GPUDB_COL_LI_DISCOUNT}, GPUDB_ORDERS_CLUSTERED,
                             (int64_t)D.od.n_rows, (int64_t)pa.n_rows, (int64_t)D.su.n_rows);
  const double gen_ms = now_ms() - t0;
  // BRAZIL in AMERICA, ECONOMY ANODIZED STEEL, orders of 1995-01-01 .. 1996-12-31
  const uint32_t america = (1u << 1) | (1u << 2) | (1u << 3) | (1u << 17) | (1u << 24);
  const gpudb_q8_params p{1096, 1826, america, 2, GPUDB_PART_TYPE(4, 0, 3), 0};
  gpudb_q8_result r{};
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++) check(ctx, gpudb_q8_market_share(ctx, &D.cu, &D.su, &pa, &D.od, &L.li, &p, &r, &t, nullptr), "gpudb_q8");
  const double p0 = now_ms();
  std::printf("\nTPC-H Q8 Results:\n");
  std::printf("+--------+------------+\n");
  std::printf("| o_year |  mkt_share |\n");
  std::printf("+--------+------------+\n");
  for (int y = 0; y < r.n_years; y++) {
    const long double share = r.volume[y] ? (long double)r.nation_volume[y] / (long double)r.volume[y] : 0.0L;
    std::printf("| %6d | %10.6Lf |\n", r.first_year + y, share);
  }
  std::printf("+--------+------------+\n");
  for (int y = 0; y < r.n_years; y++)
    std::printf("volume %d: %" PRId64 " of %" PRId64 "\n", r.first_year + y, r.nation_volume[y], r.volume[y]);
  std::printf("\nQ8 | %" PRIu64 " lineitem\n", L.li.n_rows);
  printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
}

void runQ10Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("\n--- Running TPC-H Query 10 Benchmark ---\n");
  const Scale& s = o.scale;
  const double t0 = now_ms();
  gpudb_customer cu{};
  gpudb_orders orr{};
  TblTable ct, ot;
  Buffer ck, ok, oc, od;
  if (!o.data_dir.empty()) {
    ct = load_tbl(ctx, o.data_dir, "customer", GPUDB_TBL_CUSTOMER, {0}, {4}, o.tbl_piece);
    ot = load_tbl(ctx, o.data_dir, "orders", GPUDB_TBL_ORDERS, {0, 1, 2}, {4, 4, 4}, o.tbl_piece);
    cu = {ct.rows, ct.col_max[0], 0, ct.col<int32_t>(0), nullptr};
    orr = {ot.rows, ot.col_max[0], ot.col_max[1], ot.col<int32_t>(0), ot.col<int32_t>(1), ot.col<int32_t>(2)};
  } else {
    gpudb_gen_spec cs{};
    cs.seed = o.seed;
    cs.n_rows = s.customer;
    ck = generate(ctx, cs, GPUDB_COL_CU_CUST_KEY, GPUDB_MEM_DEVICE);
    gpudb_gen_spec os = cs;
    os.n_rows = s.orders;
    os.n_cust = (int64_t)s.customer;
    ok = generate(ctx, os, GPUDB_COL_OR_ORDER_KEY, GPUDB_MEM_DEVICE);
    oc = generate(ctx, os, GPUDB_COL_OR_CUST_KEY, GPUDB_MEM_DEVICE);
    od = generate(ctx, os, GPUDB_COL_OR_ORDER_DATE, GPUDB_MEM_DEVICE);
    cu = {s.customer, (int32_t)s.customer - 1, 0, ck.as<int32_t>(), nullptr};
    orr = {s.orders, (int32_t)(4 * (s.orders - 1) + 1), (int32_t)s.customer - 1, ok.as<int32_t>(), oc.as<int32_t>(),
           od.as<int32_t>()};
  }
  Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_ORDER_KEY, GPUDB_COL_LI_FLAG, GPUDB_COL_LI_EXT_PRICE,
                                      GPUDB_COL_LI_DISCOUNT}, GPUDB_ORDERS_CLUSTERED, (int64_t)orr.n_rows, 0, 0);
  const double gen_ms = now_ms() - t0;
  std::printf("Loaded %" PRIu64 " customers, %" PRIu64 " orders, %" PRIu64 " lineitem rows for Q10.\n", cu.n_rows,
              orr.n_rows, L.li.n_rows);
  const gpudb_q10_params p{639, 731, 20, 0};   // 1993-10-01 <= o_orderdate < 1994-01-01, top 20
  gpudb_q10_result r{};
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++) check(ctx, gpudb_q10_returned(ctx, &cu, &orr, &L.li, &p, &r, &t, nullptr), "gpudb_q10");
  const double p0 = now_ms();
  std::printf("\nTPC-H Q10 Results (Top 20):\n");
  std::printf("+---------+--------------------+--------------------+\n");
  std::printf("| custkey |             c_name |            revenue |\n");
  std::printf("+---------+--------------------+--------------------+\n");
  for (uint32_t i = 0; i < r.n_rows; i++) {
    char name[32];
    std::snprintf(name, sizeof name, "Customer#%09d", r.rows[i].cust_key);
    std::printf("| %7d | %18s | $%17s |\n", r.rows[i].cust_key, name, fixed(r.rows[i].revenue, 4).c_str());
  }
  std::printf("+---------+--------------------+--------------------+\n");
  std::printf("Customers with returned revenue: %" PRIu64 "\n", r.n_customers);
  header(o, "Q10", L.li.n_rows, t);
  printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
}

void runQ13Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("\n--- Running TPC-H Query 13 Benchmark ---\n");
  const double t0 = now_ms();
  gpudb_customer cu{};
  gpudb_orders orr{};
  TblTable ct, ot;
  Buffer ck, oc, om;
  if (!o.data_dir.empty()) {
    ct = load_tbl(ctx, o.data_dir, "customer", GPUDB_TBL_CUSTOMER, {0}, {4}, o.tbl_piece);
    ot = load_tbl(ctx, o.data_dir, "orders", GPUDB_TBL_ORDERS, {1, 4}, {4, GPUDB_COMMENT_WIDTH}, o.tbl_piece);
    cu = {ct.rows, ct.col_max[0], 0, ct.col<int32_t>(0), nullptr};
    orr.n_rows = ot.rows;
    orr.cust_key = ot.col<int32_t>(1);
    orr.comment = ot.col<char>(4);
  } else {
    gpudb_gen_spec cs{};
    cs.seed = o.seed;
    cs.n_rows = o.scale.customer;
    ck = generate(ctx, cs, GPUDB_COL_CU_CUST_KEY, GPUDB_MEM_DEVICE);
    gpudb_gen_spec os = cs;
    os.n_rows = o.scale.orders;
    os.n_cust = (int64_t)o.scale.customer;
    oc = generate(ctx, os, GPUDB_COL_OR_CUST_KEY, GPUDB_MEM_DEVICE);
    om = generate(ctx, os, GPUDB_COL_OR_COMMENT, GPUDB_MEM_DEVICE);
    cu = {o.scale.customer, (int32_t)o.scale.customer - 1, 0, ck.as<int32_t>(), nullptr};
    orr.n_rows = o.scale.orders;
    orr.cust_key = oc.as<int32_t>();
    orr.comment = om.as<char>();
  }
  const double gen_ms = now_ms() - t0;
  gpudb_q13_params p{};
  std::strcpy(p.word1, "special");
  std::strcpy(p.word2, "requests");
  std::vector<gpudb_q13_row> rows(GPUDB_Q13_MAX_COUNT + 1);
  uint32_t n = 0;
  gpudb_timing t{};
  for (int i = 0; i < o.reps; i++)
    check(ctx, gpudb_q13_distribution(ctx, &cu, &orr, &p, rows.data(), (uint32_t)rows.size(), &n, &t, nullptr),
          "gpudb_q13");
  const double p0 = now_ms();
  std::printf("\nTPC-H Query 13 Results (Comparable histogram):\n");
  std::printf("+---------+----------+\n");
  std::printf("| c_count | custdist |\n");
  std::printf("+---------+----------+\n");
  for (uint32_t i = 0; i < n && i < rows.size(); i++) std::printf("| %7u | %8u |\n", rows[i].c_count, rows[i].custdist);
  std::printf("+---------+----------+\n");
  std::printf("\nQ13 | %" PRIu64 " orders | %" PRIu64 " customers\n", orr.n_rows, cu.n_rows);
  printTimingSummary(gen_ms, t.gpu_ms, now_ms() - p0);
}

void runQ9Benchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("\n--- Running TPC-H Query 9 Benchmark ---\n");
  const Scale& s = o.scale;
  if (!o.data_dir.empty()) {
    double t0 = now_ms();
    TblTable pt = load_tbl(ctx, o.data_dir, "part", GPUDB_TBL_PART, {0, 1}, {4, 1}, o.tbl_piece);
    TblTable st = load_tbl(ctx, o.data_dir, "supplier", GPUDB_TBL_SUPPLIER, {0, 1}, {4, 1}, o.tbl_piece);
    TblTable pst = load_tbl(ctx, o.data_dir, "partsupp", GPUDB_TBL_PARTSUPP, {0, 1, 2}, {4, 4, 8}, o.tbl_piece);
    TblTable ot = load_tbl(ctx, o.data_dir, "orders", GPUDB_TBL_ORDERS, {0, 2}, {4, 4}, o.tbl_piece);
    Lineitem L = make_lineitem(ctx, o, {GPUDB_COL_LI_PART_KEY, GPUDB_COL_LI_SUPP_KEY, GPUDB_COL_LI_ORDER_KEY,
                                        GPUDB_COL_LI_EXT_PRICE, GPUDB_COL_LI_DISCOUNT, GPUDB_COL_LI_QUANTITY},
                               GPUDB_ORDERS_UNIFORM, 0, 0, 0);
    gpudb_part pa{pt.rows, pt.col_max[0], 0, pt.col<int32_t>(0), pt.col<uint8_t>(1)};
    gpudb_supplier su{st.rows, st.col_max[0], 0, st.col<int32_t>(0), st.col<uint8_t>(1)};
    gpudb_partsupp pp{pst.rows, pst.col<int32_t>(0), pst.col<int32_t>(1), pst.col<int64_t>(2)};
    gpudb_orders orr{ot.rows, ot.col_max[0], 0, ot.col<int32_t>(0), nullptr, ot.col<int32_t>(2)};
    q9_report(ctx, o, pa, su, pp, orr, L, now_ms() - t0);
    return;
  }
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
  q9_report(ctx, o, pa, su, pt, orr, L, gen_ms);
}

namespace {

void q9_report(gpudb_ctx* ctx, const RunOptions& o, const gpudb_part& pa, const gpudb_supplier& su,
               const gpudb_partsupp& pt, const gpudb_orders& orr, const Lineitem& L, double gen_ms) {
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

}  // namespace

void runSelectionBenchmark(gpudb_ctx* ctx, const RunOptions& o) {
  std::printf("--- Running Selection Benchmark ---\n");
  RunOptions od = o;
  od.scale.streamed = false;   // a device column
  Lineitem L = make_lineitem(ctx, od, {GPUDB_COL_LI_SHIP_DATE}, GPUDB_ORDERS_NONE, 0, 0, 0);
  gpudb_gen_spec spec{};
  spec.n_rows = L.li.n_rows;
  const Buffer& col = L.cols[0];
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
  RunOptions od = o;
  od.scale.streamed = false;   // a device column
  Lineitem L = make_lineitem(ctx, od, {GPUDB_COL_LI_QUANTITY}, GPUDB_ORDERS_NONE, 0, 0, 0);
  gpudb_gen_spec spec{};
  spec.n_rows = L.li.n_rows;
  const Buffer& col = L.cols[0];
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
  gpudb_gen_spec ps = bs;
  Buffer build, probe;
  if (!o.data_dir.empty()) {
    TblTable ot = load_tbl(ctx, o.data_dir, "orders", GPUDB_TBL_ORDERS, {0}, {4}, o.tbl_piece);
    TblTable lt = load_tbl(ctx, o.data_dir, "lineitem", GPUDB_TBL_LINEITEM, {0}, {4}, o.tbl_piece);
    bs.n_rows = ot.rows;
    ps.n_rows = lt.rows;
    build = std::move(ot.cols[0]);
    probe = std::move(lt.cols[0]);
  } else {
    build = generate(ctx, bs, GPUDB_COL_OR_ORDER_KEY, GPUDB_MEM_DEVICE);
    ps.n_rows = o.scale.lineitem;
    ps.n_orders = (int64_t)o.scale.orders;
    ps.order_mode = GPUDB_ORDERS_CLUSTERED;
    probe = generate(ctx, ps, GPUDB_COL_LI_ORDER_KEY, GPUDB_MEM_DEVICE);
  }
  std::printf("Loaded %" PRIu64 " rows for build phase, %" PRIu64 " rows for probe phase.\n", bs.n_rows, ps.n_rows);
  for (int mode : {GPUDB_JOIN_GLOBAL, GPUDB_JOIN_RADIX, GPUDB_JOIN_DIRECT}) {
    uint64_t m = 0;
    gpudb_timing t{};
    for (int i = 0; i < o.reps; i++)
      check(ctx, gpudb_hash_join_count(ctx, build.as<int32_t>(), bs.n_rows, probe.as<int32_t>(), ps.n_rows, mode, &m, &t, nullptr),
            "gpudb_hash_join_count");
    const char* name = mode == GPUDB_JOIN_GLOBAL ? "global table" : mode == GPUDB_JOIN_RADIX ? "radix partitioned"
                                                                                          : "direct bitmap";
    std::printf("Join (%s) complete. Found %" PRIu64 " total matches.\n", name, m);
    std::printf("Total Join GPU time: %.4f ms\n\n", t.gpu_ms);
  }
}

}  // namespace gpudb_host
