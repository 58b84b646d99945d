// Counter-based synthetic table generator, shared by host C++ and CUDA device code.
//
// Every value is a pure function of (seed, column id, row index), so any row range
// (a streamed chunk, one rank's shard) is generated independently of the rest and the
// host and the device produce identical bytes.
//
//   draw(seed, col, row) = fin(key(seed, col) + (row + 1) * GOLDEN)
//   key(seed, col)       = fin(seed * GOLDEN + (col + 1) * 0xD1B54A32D192ED03)
//   fin                  = the 64-bit SplitMix finaliser (Steele, Lea, Flood:
//                          "Fast splittable pseudorandom number generators", OOPSLA 2014)
//   uniform(lo, hi)      = lo + mulhi64(draw, hi - lo + 1)   (Lemire's multiply-shift range map)
//
// The tables stand in for the TPC-H tables the reference reads from dbgen `.tbl` files
// (src/infra.h:262-361 loads them); no dbgen data is used. Column distributions:
//   lineitem: ship_date U[0,2526], quantity U[1,50], ext_price = quantity * U[90000,209900]
//             (int64 hundredths), discount U[0,10], tax U[0,8], flag U{0,1,2}, status U{0,1},
//             order_key clustered (runs of 1..7 rows per order, orders in sequence) or
//             uniform (4*U[0,n_orders)+1), part_key U[0,n_parts), supp_key one of the
//             part's 4 partsupp suppliers.
//   customer: cust_key = i, segment U{0..4}
//   orders:   order_key = 4*i+1, cust_key U[0,n_cust), order_date U[0,2405]
//   part:     part_key = i, flag = (U[0,999] < 55)  (Bernoulli 0.055)
//   supplier: supp_key = i, nation U[0,24]
//   partsupp: part_key = r/4, supp_key = gd_partsupp_supp(r/4, r%4), supply_cost U[100,100000]
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define GD_HD __host__ __device__ __forceinline__
#else
#define GD_HD static inline
#endif

#define GD_GOLDEN 0x9E3779B97F4A7C15ull

// Column identifiers: table * 16 + column.
enum gd_column {
  GD_LI_SHIP_DATE = 16, GD_LI_QUANTITY, GD_LI_UNIT_PRICE, GD_LI_DISCOUNT, GD_LI_TAX,
  GD_LI_FLAG, GD_LI_STATUS, GD_LI_ORDER_PICK, GD_LI_PART, GD_LI_SUPP_SLOT, GD_LI_ORDER_RUN,
  GD_LI_COMMIT, GD_LI_RECEIPT, GD_LI_MODE,
  GD_CU_SEGMENT = 32, GD_CU_NATION,
  GD_OR_CUST = 48, GD_OR_DATE, GD_OR_PRIORITY, GD_OR_COMMENT,
  GD_PA_FLAG = 64, GD_PA_TYPE,
  GD_SU_NATION = 80,
  GD_PS_COST = 96
};

GD_HD uint64_t gd_fin(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

GD_HD uint64_t gd_mulhi(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64);
#endif
}

GD_HD uint64_t gd_stream_key(uint64_t seed, uint32_t col) {
  return gd_fin(seed * GD_GOLDEN + (uint64_t)(col + 1) * 0xD1B54A32D192ED03ull);
}

GD_HD uint64_t gd_draw_k(uint64_t key, uint64_t row) { return gd_fin(key + (row + 1) * GD_GOLDEN); }

GD_HD int64_t gd_uniform_k(uint64_t key, uint64_t row, int64_t lo, int64_t hi) {
  return lo + (int64_t)gd_mulhi(gd_draw_k(key, row), (uint64_t)(hi - lo + 1));
}

GD_HD int64_t gd_uniform(uint64_t seed, uint32_t col, uint64_t row, int64_t lo, int64_t hi) {
  return gd_uniform_k(gd_stream_key(seed, col), row, lo, hi);
}

// Domain constants of the synthetic schema.
#define GD_SHIP_DATE_MAX 2526
#define GD_ORDER_DATE_MAX 2405
#define GD_BASE_YEAR 1992
#define GD_RUN_MAX 7           /* 1..7 lineitem rows per order in the clustered layout */

// Lineitem order-key layouts.
enum gd_order_mode { GD_ORDERS_NONE = 0, GD_ORDERS_CLUSTERED = 1, GD_ORDERS_UNIFORM = 2 };

GD_HD int32_t gd_li_ship_date(uint64_t seed, uint64_t r) { return (int32_t)gd_uniform(seed, GD_LI_SHIP_DATE, r, 0, GD_SHIP_DATE_MAX); }
GD_HD int32_t gd_li_quantity(uint64_t seed, uint64_t r) { return (int32_t)gd_uniform(seed, GD_LI_QUANTITY, r, 1, 50); }
GD_HD int64_t gd_li_ext_price(uint64_t seed, uint64_t r) {
  return (int64_t)gd_li_quantity(seed, r) * gd_uniform(seed, GD_LI_UNIT_PRICE, r, 90000, 209900);
}
GD_HD int32_t gd_li_discount(uint64_t seed, uint64_t r) { return (int32_t)gd_uniform(seed, GD_LI_DISCOUNT, r, 0, 10); }
GD_HD int32_t gd_li_tax(uint64_t seed, uint64_t r) { return (int32_t)gd_uniform(seed, GD_LI_TAX, r, 0, 8); }
GD_HD uint8_t gd_li_flag(uint64_t seed, uint64_t r) { return (uint8_t)gd_uniform(seed, GD_LI_FLAG, r, 0, 2); }
GD_HD uint8_t gd_li_status(uint64_t seed, uint64_t r) { return (uint8_t)gd_uniform(seed, GD_LI_STATUS, r, 0, 1); }
GD_HD int32_t gd_li_order_uniform(uint64_t seed, uint64_t r, int64_t n_orders) {
  return (int32_t)(4 * gd_uniform(seed, GD_LI_ORDER_PICK, r, 0, n_orders - 1) + 1);
}
// Rows of clustered run s (order index s mod n_orders): 1..7.
GD_HD int32_t gd_li_run_length(uint64_t seed, uint64_t s) { return (int32_t)gd_uniform(seed, GD_LI_ORDER_RUN, s, 1, GD_RUN_MAX); }
GD_HD int32_t gd_order_key_of(int64_t order_index) { return (int32_t)(4 * order_index + 1); }
GD_HD int32_t gd_li_part(uint64_t seed, uint64_t r, int64_t n_parts) { return (int32_t)gd_uniform(seed, GD_LI_PART, r, 0, n_parts - 1); }
// The j-th (0..3) supplier of a part; shared by lineitem and partsupp so that every lineitem
// (part, supp) pair exists in partsupp.
GD_HD int32_t gd_partsupp_supp(int64_t part, int64_t j, int64_t n_supp) {
  return (int32_t)((part + j * (n_supp / 4)) % n_supp);
}
GD_HD int32_t gd_li_supp(uint64_t seed, uint64_t r, int64_t n_parts, int64_t n_supp) {
  return gd_partsupp_supp(gd_li_part(seed, r, n_parts), gd_uniform(seed, GD_LI_SUPP_SLOT, r, 0, 3), n_supp);
}

// Commit and receipt dates follow TPC-H's offsets: commit = order date + [30, 90] and ship =
// order date + [1, 121] give commit - ship in [-91, 89]; receipt = ship + [1, 30].
GD_HD int32_t gd_li_commit_date(uint64_t seed, uint64_t r) {
  return gd_li_ship_date(seed, r) + (int32_t)gd_uniform(seed, GD_LI_COMMIT, r, -91, 89);
}
GD_HD int32_t gd_li_receipt_date(uint64_t seed, uint64_t r) {
  return gd_li_ship_date(seed, r) + (int32_t)gd_uniform(seed, GD_LI_RECEIPT, r, 1, 30);
}
GD_HD uint8_t gd_li_ship_mode(uint64_t seed, uint64_t r) { return (uint8_t)gd_uniform(seed, GD_LI_MODE, r, 0, 6); }
GD_HD uint8_t gd_or_priority(uint64_t seed, uint64_t r) { return (uint8_t)gd_uniform(seed, GD_OR_PRIORITY, r, 1, 5); }
// Order comments: 2..9 words drawn from a 24-word vocabulary (draw 0 of row r's sub-stream
// r*16 is the word count, draws 1.. the words), separated by one space; a word that would
// pass 79 characters ends the comment; the rest of the 80 bytes is 0.
#define GD_COMMENT_WIDTH 80
#define GD_VOCAB "specialrequestspackagesdepositsaccountsinstructionsfoxesideastheodolitespintobeans" \
                 "plateletsfuriouslycarefullyquicklyslylyblithelyregularfinalpendingironicexpressboldeven"
GD_HD void gd_or_comment(uint64_t seed, uint64_t r, char* out) {
  const uint8_t len[24] = {7, 8, 8, 8, 8, 12, 5, 5, 11, 5, 5, 9, 9, 9, 7, 5, 8, 7, 5, 7, 6, 7, 4, 4};
  const uint8_t off[24] = {0, 7, 15, 23, 31, 39, 51, 56, 61, 72, 77, 82, 91, 100, 109, 116, 121, 129, 136, 141, 148,
                           154, 161, 165};
  const char* vocab = GD_VOCAB;
  const uint64_t key = gd_stream_key(seed, GD_OR_COMMENT);
  const int words = (int)gd_uniform_k(key, r * 16, 2, 9);
  int n = 0;
  for (int i = 0; i < words; i++) {
    const int w = (int)gd_uniform_k(key, r * 16 + 1 + i, 0, 23);
    if (n + (n ? 1 : 0) + len[w] > GD_COMMENT_WIDTH - 1) break;
    if (n) out[n++] = ' ';
    for (int c = 0; c < len[w]; c++) out[n++] = vocab[off[w] + c];
  }
  for (; n < GD_COMMENT_WIDTH; n++) out[n] = 0;
}
GD_HD uint8_t gd_cu_nation(uint64_t seed, uint64_t r) { return (uint8_t)gd_uniform(seed, GD_CU_NATION, r, 0, 24); }
GD_HD uint8_t gd_cu_segment(uint64_t seed, uint64_t r) { return (uint8_t)gd_uniform(seed, GD_CU_SEGMENT, r, 0, 4); }
GD_HD int32_t gd_or_cust(uint64_t seed, uint64_t r, int64_t n_cust) { return (int32_t)gd_uniform(seed, GD_OR_CUST, r, 0, n_cust - 1); }
GD_HD int32_t gd_or_date(uint64_t seed, uint64_t r) { return (int32_t)gd_uniform(seed, GD_OR_DATE, r, 0, GD_ORDER_DATE_MAX); }
GD_HD uint8_t gd_pa_type(uint64_t seed, uint64_t r) { return (uint8_t)gd_uniform(seed, GD_PA_TYPE, r, 0, 149); }
GD_HD uint8_t gd_pa_flag(uint64_t seed, uint64_t r) { return (uint8_t)(gd_uniform(seed, GD_PA_FLAG, r, 0, 999) < 55); }
GD_HD uint8_t gd_su_nation(uint64_t seed, uint64_t r) { return (uint8_t)gd_uniform(seed, GD_SU_NATION, r, 0, 24); }
GD_HD int64_t gd_ps_cost(uint64_t seed, uint64_t r) { return gd_uniform(seed, GD_PS_COST, r, 100, 100000); }

// Order year of the star-join grouping: 1992 + order_date / 365 (integer division).
GD_HD int32_t gd_order_year(int32_t order_date) { return GD_BASE_YEAR + order_date / 365; }
