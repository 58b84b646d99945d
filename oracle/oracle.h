/*
 * oracle.h -- CPU oracle of the query engine's hot path. TEST INFRASTRUCTURE ONLY:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library,
 * and only to check or time against it. The engine never links or calls it.
 *
 * Single-threaded C (gcc, __int128), exact integer arithmetic. Each function cites the
 * reference code whose query logic it restates. The reference computes in float32 and
 * rounds per row in places (kernels/q1.metal:84-89); the oracle instead follows the
 * exact fixed-point semantics of the synthetic workloads (money in int64 hundredths,
 * products exact, group totals in int128). The reference's own kernels are compiled for
 * the CPU separately (oracle/ref_harness.cpp) to pin this restatement's query logic.
 */
#ifndef GPUDB_ORACLE_H
#define GPUDB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_spec {
  uint64_t seed, row_offset, n_rows;
  int64_t n_orders, n_cust, n_parts, n_supp;
  int32_t order_mode, reserved;
} or_spec;

/* Column ids: the same numbering as include/gpudb_capi.h (GPUDB_COL_*). */
int or_gen_column(const or_spec* spec, int32_t column, void* dst);

/* Q6-like: sum(ext*disc) where ship in [lo,hi), disc in [dlo,dhi], qty < qlt. */
void or_q6(uint64_t n, const int32_t* ship, const int32_t* disc, const int32_t* qty,
           const int64_t* ext, int32_t lo, int32_t hi, int32_t dlo, int32_t dhi, int32_t qlt,
           int64_t* revenue, uint64_t* matched);

/* Q1-like: 6 groups (flag*2+status). Per group out[g*11 + ...]:
 *   [0]=count, then lo/hi pairs of sum_qty, sum_base, sum_disc, sum_charge, sum_discount. */
void or_q1(uint64_t n, const int32_t* ship, const int32_t* qty, const int64_t* ext,
           const int32_t* disc, const int32_t* tax, const uint8_t* flag, const uint8_t* status,
           int32_t ship_le, uint64_t* out);

/* Multi-threaded Q1/Q6 (pthreads), used only as the timed CPU baseline. */
void or_q6_mt(int threads, uint64_t n, const int32_t* ship, const int32_t* disc,
              const int32_t* qty, const int64_t* ext, int32_t lo, int32_t hi, int32_t dlo,
              int32_t dhi, int32_t qlt, int64_t* revenue, uint64_t* matched);
void or_q1_mt(int threads, uint64_t n, const int32_t* ship, const int32_t* qty,
              const int64_t* ext, const int32_t* disc, const int32_t* tax,
              const uint8_t* flag, const uint8_t* status, int32_t ship_le, uint64_t* out);

/* Q3-like: top-k rows (order_key, order_date, revenue) ordered by revenue desc,
 * order_date asc, order_key asc. Returns the number of groups (orders with >= 1 joined
 * lineitem row); writes min(k, groups) rows. */
uint64_t or_q3(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_seg, int32_t cu_key_max,
               uint64_t n_or, const int32_t* or_key, const int32_t* or_cust,
               const int32_t* or_date, int32_t or_key_max,
               uint64_t n_li, const int32_t* li_order, const int32_t* li_ship,
               const int64_t* li_ext, const int32_t* li_disc,
               int32_t segment, int32_t date_lt, int32_t ship_gt, int32_t k,
               int32_t* top_key, int32_t* top_date, int64_t* top_rev);

/* Q9-like: groups (nation, year, profit) ordered by nation asc, year desc. Returns the
 * number of groups; writes at most cap. */
uint32_t or_q9(uint64_t n_pa, const int32_t* pa_key, const uint8_t* pa_flag, int32_t pa_key_max,
               uint64_t n_su, const int32_t* su_key, const uint8_t* su_nation, int32_t su_key_max,
               uint64_t n_ps, const int32_t* ps_part, const int32_t* ps_supp, const int64_t* ps_cost,
               uint64_t n_or, const int32_t* or_key, const int32_t* or_date, int32_t or_key_max,
               uint64_t n_li, const int32_t* li_part, const int32_t* li_supp, const int32_t* li_order,
               const int64_t* li_ext, const int32_t* li_disc, const int32_t* li_qty,
               uint32_t cap, int32_t* g_nation, int32_t* g_year, int64_t* g_profit);

/* Microbenchmarks. */
/* Q4: the late-delivery bitmap of kernels/q4.metal:21-37 (order keys of lineitem rows with
 * commit < receipt; keys outside 0..or_key_max match no order) and the count of
 * kernels/q4.metal:40-72 (orders in [date_lo, date_hi) whose key is in it, by priority 1..5). */
void or_q4(uint64_t n_or, const int32_t* o_key, const int32_t* o_date, const uint8_t* o_prio, int32_t or_key_max,
           uint64_t n_li, const int32_t* l_key, const int32_t* l_commit, const int32_t* l_receipt, int32_t date_lo,
           int32_t date_hi, uint64_t* count5);
/* Q12: the priority bitmap of kernels/q12.metal:87-99 (orders with priority 1..high_max) and the
 * filter + 4-bin count of kernels/q12.metal:22-66. out = {high[mode0], high[mode1], low[mode0],
 * low[mode1]}; a row whose key is outside 0..or_key_max is low. */
void or_q12(uint64_t n_or, const int32_t* o_key, const uint8_t* o_prio, int32_t or_key_max, uint64_t n_li,
            const int32_t* l_key, const int32_t* l_ship, const int32_t* l_commit, const int32_t* l_receipt,
            const uint8_t* l_mode, int32_t receipt_lo, int32_t receipt_hi, int32_t mode0, int32_t mode1,
            int32_t high_max, uint64_t* out4);

/* Q5: revenue25[n] = exact sum of ext*(100-disc) over lineitem rows whose order is in
 * [date_lo, date_hi) and whose customer and supplier are both of nation n, n in nation_mask
 * (kernels/q5.metal:19-125). */
void or_q5(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_nation, int32_t cu_key_max, uint64_t n_su,
           const int32_t* su_key, const uint8_t* su_nation, int32_t su_key_max, uint64_t n_or, const int32_t* o_key,
           const int32_t* o_cust, const int32_t* o_date, int32_t or_key_max, uint64_t n_li, const int32_t* l_key,
           const int32_t* l_supp, const int64_t* l_ext, const int32_t* l_disc, int32_t date_lo, int32_t date_hi,
           uint32_t nation_mask, int64_t* revenue25);
/* Q7: rev16[pair * 8 + y], pair 0 = supplier of a / customer of b, 1 = the reverse, y = calendar
 * year of the ship date (in [ship_lo, ship_hi], both included) - first_year
 * (kernels/q7.metal:12-109). Returns -1 when the window spans more than 8 years. */
int or_q7(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_nation, int32_t cu_key_max, uint64_t n_su,
          const int32_t* su_key, const uint8_t* su_nation, int32_t su_key_max, uint64_t n_or, const int32_t* o_key,
          const int32_t* o_cust, int32_t or_key_max, uint64_t n_li, const int32_t* l_key, const int32_t* l_supp,
          const int32_t* l_ship, const int64_t* l_ext, const int32_t* l_disc, int32_t a, int32_t b, int32_t ship_lo,
          int32_t ship_hi, int64_t* rev16, int32_t* first_year, int32_t* n_years);
/* Q8: vol8[y] / nvol8[y] = revenue of the part type's lineitems whose order is in [date_lo,
 * date_hi] (both included) with a customer of region_mask, all suppliers / suppliers of
 * `nation`; y = calendar year of the order date - first_year (kernels/q8.metal:9-76). */
int or_q8(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_nation, int32_t cu_key_max, uint64_t n_su,
          const int32_t* su_key, const uint8_t* su_nation, int32_t su_key_max, uint64_t n_pa, const int32_t* pa_key,
          const uint8_t* pa_type, int32_t pa_key_max, uint64_t n_or, const int32_t* o_key, const int32_t* o_cust,
          const int32_t* o_date, int32_t or_key_max, uint64_t n_li, const int32_t* l_key, const int32_t* l_part,
          const int32_t* l_supp, const int64_t* l_ext, const int32_t* l_disc, int32_t date_lo, int32_t date_hi,
          uint32_t region_mask, int32_t nation, int32_t part_type, int64_t* vol8, int64_t* nvol8, int32_t* first_year,
          int32_t* n_years);
/* Q10: exact revenue sum ext*(100-disc) of returned lineitems (flag 2) per customer of cu, over
 * orders with date_lo <= date < date_hi (kernels/q10.metal:8-54); the top k by revenue desc,
 * cust_key asc among customers with revenue > 0 (src/q10.cpp:102-121). rev_out (cu_key_max+1
 * entries, may be NULL) gets every customer's revenue. Returns the number of customers with
 * revenue > 0. */
uint64_t or_q10(uint64_t n_cu, const int32_t* cu_key, int32_t cu_key_max, uint64_t n_or, const int32_t* o_key,
                const int32_t* o_cust, const int32_t* o_date, int32_t or_key_max, uint64_t n_li, const int32_t* l_key,
                const uint8_t* l_flag, const int64_t* l_ext, const int32_t* l_disc, int32_t date_lo, int32_t date_hi,
                int32_t k, int32_t* top_key, int64_t* top_rev, int64_t* rev_out);

/* Q13: per-customer counts of orders whose 80-byte NUL-padded comment is NOT LIKE
 * '%w1%w2%' (kernels/q13.metal:33-127), the histogram of those counts over the customer rows
 * (kernels/q13.metal:133-168) ordered by custdist desc, c_count desc (postProcessQ13
 * src/infra.h:783-800). Writes up to cap rows, returns the number of distinct counts. */
uint32_t or_q13(uint64_t n_cu, const int32_t* cu_key, int32_t cu_key_max, uint64_t n_or, const int32_t* o_cust,
                const char* o_comment, const char* w1, const char* w2, uint32_t* c_count, uint32_t* custdist,
                uint32_t cap);

uint64_t or_select_lt(uint64_t n, const int32_t* col, int32_t value, uint32_t* bits, uint32_t* rows);
int64_t or_sum_i32(uint64_t n, const int32_t* col);
uint64_t or_join_count(uint64_t nb, const int32_t* bkeys, uint64_t np, const int32_t* pkeys);
/* The reference's 1024-way partition hash (kernels/common.h:81-87, microbenchmarks.metal:10-12). */
uint32_t or_key_hash(int32_t key);
void or_radix_histogram(uint64_t n, const int32_t* keys, int32_t bits, uint32_t* hist);
/* Stable partition: keys_out/payload_out grouped by partition, input order inside one. */
void or_radix_partition(uint64_t n, const int32_t* keys, const int32_t* payload, int32_t bits,
                        int32_t* keys_out, int32_t* payload_out, uint32_t* offsets);
/* Equi-join pairs in (probe row, build row) order; returns the total, writes <= cap. */
uint64_t or_join_pairs(uint64_t nb, const int32_t* bkeys, uint64_t np, const int32_t* pkeys,
                       uint64_t cap, int32_t* out_b, int32_t* out_p);

#ifdef __cplusplus
}
#endif
#endif
