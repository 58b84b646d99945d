// ref_harness.cpp -- runs the reference's own Metal kernels (kernels/q1.metal, q3.metal,
// q4.metal, q5.metal, q6.metal, q7.metal, q8.metal, q9.metal, q10.metal, q12.metal, q13.metal, microbenchmarks.metal, compiled in place from the reference tree
// through the CPU shim in oracle/refshim) on the synthetic tables. TEST INFRASTRUCTURE
// ONLY: it pins the oracle's query logic to the reference's code, and it is the timed
// reference arm of bench.py. It is never linked into the engine.
//
// The synthetic columns are converted to the reference's storage types the way its
// loaders would hold them (src/infra.h:262-361): money and fractions as float32 dollars,
// dates as YYYYMMDD integers, flags as the TPC-H characters.
#include <algorithm>
#include <thread>
#include <vector>

#include <metal_stdlib>
using namespace metal;

#include "common.h"
#include "microbenchmarks.metal"
#include "q1.metal"
#include "q10.metal"
#include "q12.metal"
#include "q13.metal"
#include "q3.metal"
#include "q4.metal"
#include "q5.metal"
#include "q6.metal"
#include "q7.metal"
#include "q8.metal"
#include "q9.metal"

namespace {

// Day number (0 = 1992-01-01, negative before it) -> YYYYMMDD, proleptic Gregorian calendar.
int yyyymmdd(int day) {
  static const int mdays[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
  auto year_len = [](int y) { return ((y % 4 == 0 && y % 100 != 0) || y % 400 == 0) ? 366 : 365; };
  int y = 1992;
  while (day < 0) day += year_len(--y);
  for (;;) {
    bool leap = (y % 4 == 0 && y % 100 != 0) || y % 400 == 0;
    int len = leap ? 366 : 365;
    if (day < len) {
      for (int m = 0; m < 12; m++) {
        int ml = mdays[m] + (m == 1 && leap ? 1 : 0);
        if (day < ml) return y * 10000 + (m + 1) * 100 + day + 1;
        day -= ml;
      }
    }
    day -= len;
    y++;
  }
}

std::vector<int> dates(uint64_t n, const int32_t* d) {
  int lo = 0, hi = 0;
  for (uint64_t i = 0; i < n; i++) { lo = std::min(lo, d[i]); hi = std::max(hi, d[i]); }
  std::vector<int> table(hi - lo + 2);
  for (int i = lo; i <= hi + 1; i++) table[i - lo] = yyyymmdd(i);
  std::vector<int> out(n);
  for (uint64_t i = 0; i < n; i++) out[i] = table[d[i] - lo];
  return out;
}

template <class T> std::vector<float> hundredths(uint64_t n, const T* v) {
  std::vector<float> out(n);
  for (uint64_t i = 0; i < n; i++) out[i] = (float)v[i] / 100.0f;
  return out;
}
template <class T> std::vector<float> as_float(uint64_t n, const T* v) {
  std::vector<float> out(n);
  for (uint64_t i = 0; i < n; i++) out[i] = (float)v[i];
  return out;
}

// Runs fn(group) for groups 0..G-1 on up to `threads` host threads.
template <class F> void run_groups(uint G, int threads, F fn) {
  if (threads <= 1 || G <= 1) { for (uint g = 0; g < G; g++) fn(g); return; }
  std::vector<std::thread> th;
  uint T = std::min<uint>((uint)threads, G);
  for (uint t = 0; t < T; t++)
    th.emplace_back([=] { for (uint g = t; g < G; g += T) fn(g); });
  for (auto& x : th) x.join();
}

uint next_pow2_u(uint v) { uint p = 1; while (p < v) p <<= 1; return p; }

template <class K> int max_of(uint64_t n, const K* v) {
  int m = 0;
  for (uint64_t i = 0; i < n; i++) m = std::max(m, (int)v[i]);
  return m;
}

}  // namespace

extern "C" {

// Q6 through q6_filter_and_sum_stage1 + q6_final_sum_stage2 (kernels/q6.metal:12-70).
// `groups` threadgroups run on `threads` host threads. Returns revenue in dollars.
float ref_q6(uint64_t n, const int32_t* ship, const int32_t* disc, const int32_t* qty,
             const int64_t* ext, int32_t lo, int32_t hi, int32_t dlo, int32_t dhi, int32_t qlt,
             int groups, int threads) {
  std::vector<int> sd = dates(n, ship);
  std::vector<float> d = hundredths(n, disc), q = as_float(n, qty), e = hundredths(n, ext);
  std::vector<float> partial(groups);
  uint size = (uint)n;
  int start = yyyymmdd(lo), end = yyyymmdd(hi);
  float mind = (float)dlo / 100.0f, maxd = (float)dhi / 100.0f, maxq = (float)qlt;
  run_groups((uint)groups, threads, [&](uint g) {
    q6_filter_and_sum_stage1(sd.data(), d.data(), q.data(), e.data(), partial.data(), size,
                             start, end, mind, maxd, maxq, g, 0, 1, (uint)groups);
  });
  float result = 0;
  uint ng = (uint)groups;
  q6_final_sum_stage2(partial.data(), &result, ng, 0);
  return result;
}

// Q1 through q1_fused_kernel (kernels/q1.metal:39-121). Per bin (A/F, A/O, N/F, N/O, R/F,
// R/O) out[b*6 + ...] = qty cents, base cents, disc cents, charge cents, discount bp, count.
void ref_q1(uint64_t n, const int32_t* ship, const int32_t* qty, const int64_t* ext,
            const int32_t* disc, const int32_t* tax, const uint8_t* flag, const uint8_t* status,
            int32_t ship_le, int groups, int threads, int64_t* out) {
  std::vector<int> sd = dates(n, ship);
  std::vector<float> q = as_float(n, qty), e = hundredths(n, ext), d = hundredths(n, disc), t = hundredths(n, tax);
  std::vector<char> rf(n), ls(n);
  for (uint64_t i = 0; i < n; i++) { rf[i] = "ANR"[flag[i] % 3]; ls[i] = "FO"[status[i] % 2]; }
  std::vector<atomic_uint> acc(60);
  for (auto& a : acc) a.v = 0;
  atomic_uint* A = acc.data();
  uint size = (uint)n;
  int cutoff = yyyymmdd(ship_le);
  run_groups((uint)groups, threads, [&](uint g) {
    q1_fused_kernel(sd.data(), rf.data(), ls.data(), q.data(), e.data(), d.data(), t.data(),
                    A + 0, A + 6, A + 12, A + 18, A + 24, A + 30, A + 36, A + 42, A + 48, A + 54,
                    size, cutoff, g, 0, 1, (uint)groups);
  });
  for (int b = 0; b < 6; b++) {
    for (int m = 0; m < 4; m++) {
      uint64_t lo = acc[12 * m + b].v, hi = acc[12 * m + 6 + b].v;
      out[b * 6 + m] = (int64_t)((hi << 32) | lo);
    }
    out[b * 6 + 4] = acc[48 + b].v;
    out[b * 6 + 5] = acc[54 + b].v;
  }
}

// Q3 through q3_build_customer_bitmap_kernel, q3_build_orders_map_kernel,
// q3_probe_and_aggregate_direct_kernel and q3_compact_results_kernel (kernels/q3.metal).
// Writes all groups (order key, revenue in dollars, order date) and returns their count.
uint32_t ref_q3(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_seg,
                uint64_t n_or, const int32_t* or_key, const int32_t* or_cust, const int32_t* or_date,
                uint64_t n_li, const int32_t* li_order, const int32_t* li_ship,
                const int64_t* li_ext, const int32_t* li_disc,
                int32_t segment, int32_t date_lt, int32_t ship_gt, int groups, int threads,
                int32_t* g_key, float* g_rev, int32_t* g_date, uint32_t cap) {
  std::vector<char> seg(n_cu);
  int max_cust = 0;
  for (uint64_t i = 0; i < n_cu; i++) { seg[i] = cu_seg[i] == segment ? 'B' : 'M'; max_cust = std::max(max_cust, cu_key[i]); }
  std::vector<atomic_uint> bitmap((max_cust + 31) / 32 + 1);
  for (auto& w : bitmap) w.v = 0;
  uint ncu = (uint)n_cu, nor = (uint)n_or, nli = (uint)n_li;
  for (uint i = 0; i < ncu; i++) q3_build_customer_bitmap_kernel(cu_key, seg.data(), bitmap.data(), ncu, i);

  int max_order = 0;
  for (uint64_t i = 0; i < n_or; i++) max_order = std::max(max_order, or_key[i]);
  std::vector<int> omap((size_t)max_order + 1, -1);
  std::vector<int> odate = dates(n_or, or_date), prio(n_or, 0);
  int cut = yyyymmdd(date_lt);
  const uint* bm = reinterpret_cast<const uint*>(bitmap.data());
  for (uint i = 0; i < nor; i++) q3_build_orders_map_kernel(or_key, odate.data(), omap.data(), nor, cut, or_cust, bm, i);

  std::vector<int> lship = dates(n_li, li_ship);
  std::vector<float> ext = hundredths(n_li, li_ext), dsc = hundredths(n_li, li_disc);
  uint ht_size = next_pow2_u(nor * 2);
  std::vector<Q3CompactResult> ht(ht_size), dense(ht_size);
  std::memset(ht.data(), 0, ht.size() * sizeof(Q3CompactResult));
  int ship_cut = yyyymmdd(ship_gt);
  auto* fht = reinterpret_cast<Q3Aggregates*>(ht.data());
  run_groups((uint)groups, threads, [&](uint g) {
    q3_probe_and_aggregate_direct_kernel(li_order, lship.data(), ext.data(), dsc.data(), omap.data(),
                                         or_cust, odate.data(), prio.data(), fht, nli, ship_cut, ht_size,
                                         g, 0, 1, (uint)groups);
  });
  atomic_uint count; count.v = 0;
  for (uint i = 0; i < ht_size; i++) q3_compact_results_kernel(ht.data(), dense.data(), count, ht_size, i);
  // orders map back from YYYYMMDD to the day number of the input
  for (uint i = 0; i < count.v && i < cap; i++) {
    g_key[i] = dense[i].key;
    g_rev[i] = dense[i].revenue;
    g_date[i] = -1;
  }
  // recover each group's order date as a day number via the orders map
  for (uint i = 0; i < count.v && i < cap; i++) {
    int row = omap[g_key[i]];
    g_date[i] = row >= 0 ? or_date[row] : -1;
  }
  return count.v;
}

// Q4 through q4_build_late_bitmap, q4_count_by_priority_stage1 and q4_final_count_stage2
// (kernels/q4.metal:21-94); priorities 1..5 are the characters '1'..'5'. out5 = counts.
void ref_q4(uint64_t n_or, const int32_t* or_key, const int32_t* or_date, const uint8_t* or_prio,
            uint64_t n_li, const int32_t* li_key, const int32_t* li_commit, const int32_t* li_receipt,
            int32_t date_lo, int32_t date_hi, int groups, int threads, uint32_t* out5) {
  int max_key = 0;
  for (uint64_t i = 0; i < n_or; i++) max_key = std::max(max_key, or_key[i]);
  for (uint64_t i = 0; i < n_li; i++) max_key = std::max(max_key, li_key[i]);
  std::vector<atomic_uint> late((size_t)(max_key + 31) / 32 + 1);
  for (auto& w : late) w.v = 0;
  std::vector<int> lc = dates(n_li, li_commit), lr = dates(n_li, li_receipt), od = dates(n_or, or_date);
  uint nli = (uint)n_li, nor = (uint)n_or;
  for (uint i = 0; i < nli; i++) q4_build_late_bitmap(li_key, lc.data(), lr.data(), late.data(), nli, i);
  std::vector<char> pr(n_or);
  for (uint64_t i = 0; i < n_or; i++) pr[i] = (char)('0' + or_prio[i]);
  std::vector<uint> partial((size_t)groups * 5);
  int ds = yyyymmdd(date_lo), de = yyyymmdd(date_hi);
  const uint* bm = reinterpret_cast<const uint*>(late.data());
  run_groups((uint)groups, threads, [&](uint g) {
    q4_count_by_priority_stage1(or_key, od.data(), pr.data(), bm, partial.data(), nor, ds, de, g, 0, 1, (uint)groups);
  });
  uint ng = (uint)groups;
  q4_final_count_stage2(partial.data(), out5, ng, 0);
}

// Q12 through q12_build_priority_bitmap, q12_filter_and_count_stage1 and
// q12_final_count_stage2 (kernels/q12.metal:22-99): ship modes as the first character of
// their names ('M' MAIL, 'S' SHIP are counted), high priority = '1' or '2'.
// out4 = MAIL high, MAIL low, SHIP high, SHIP low.
void ref_q12(uint64_t n_or, const int32_t* or_key, const uint8_t* or_prio, uint64_t n_li,
             const int32_t* li_key, const int32_t* li_ship, const int32_t* li_commit,
             const int32_t* li_receipt, const uint8_t* li_mode, int32_t receipt_lo, int32_t receipt_hi,
             int groups, int threads, uint32_t* out4) {
  int max_key = 0;
  for (uint64_t i = 0; i < n_or; i++) max_key = std::max(max_key, or_key[i]);
  for (uint64_t i = 0; i < n_li; i++) max_key = std::max(max_key, li_key[i]);
  std::vector<atomic_uint> bitmap((size_t)(max_key + 31) / 32 + 1);
  for (auto& w : bitmap) w.v = 0;
  std::vector<char> pr(n_or);
  for (uint64_t i = 0; i < n_or; i++) pr[i] = (char)('0' + or_prio[i]);
  uint nor = (uint)n_or, nli = (uint)n_li;
  for (uint i = 0; i < nor; i++) q12_build_priority_bitmap(or_key, pr.data(), bitmap.data(), nor, i);
  std::vector<char> sm(n_li);
  for (uint64_t i = 0; i < n_li; i++) sm[i] = "AFMRRST"[li_mode[i] % 7];   // AIR FOB MAIL RAIL REG AIR SHIP TRUCK
  std::vector<int> ls = dates(n_li, li_ship), lc = dates(n_li, li_commit), lr = dates(n_li, li_receipt);
  std::vector<uint> partial((size_t)groups * 4);
  int rs = yyyymmdd(receipt_lo), re = yyyymmdd(receipt_hi);
  const uint* bm = reinterpret_cast<const uint*>(bitmap.data());
  run_groups((uint)groups, threads, [&](uint g) {
    q12_filter_and_count_stage1(li_key, sm.data(), ls.data(), lc.data(), lr.data(), bm, partial.data(), nli, rs, re,
                                g, 0, 1, (uint)groups);
  });
  uint ng = (uint)groups;
  q12_final_count_stage2(partial.data(), out4, ng, 0);
}

// Q5 through q5_build_customer_nation_map_kernel, q5_build_supplier_nation_map_kernel,
// q5_build_orders_map_kernel and q5_probe_and_aggregate_kernel (kernels/q5.metal:19-125),
// with the host's -1-filled direct maps (src/q5.cpp) and the region's nation bitmap.
void ref_q5(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_nation, uint64_t n_su, const int32_t* su_key,
            const uint8_t* su_nation, uint64_t n_or, const int32_t* or_key, const int32_t* or_cust,
            const int32_t* or_date, uint64_t n_li, const int32_t* li_key, const int32_t* li_supp,
            const int64_t* li_ext, const int32_t* li_disc, int32_t date_lo, int32_t date_hi, uint32_t nation_mask,
            int groups, int threads, float* revenue25) {
  int max_c = 0, max_s = 0, max_o = 0;
  for (uint64_t i = 0; i < n_cu; i++) max_c = std::max(max_c, cu_key[i]);
  for (uint64_t i = 0; i < n_su; i++) max_s = std::max(max_s, su_key[i]);
  for (uint64_t i = 0; i < n_or; i++) max_o = std::max(max_o, or_key[i]);
  for (uint64_t i = 0; i < n_li; i++) max_o = std::max(max_o, li_key[i]);
  std::vector<int> cmap((size_t)max_c + 1, -1), smap((size_t)max_s + 1, -1), omap((size_t)max_o + 1, -1);
  std::vector<int> cn(cu_nation, cu_nation + n_cu), sn(su_nation, su_nation + n_su);
  uint ncu = (uint)n_cu, nsu = (uint)n_su, nor = (uint)n_or, nli = (uint)n_li, map_size = (uint)max_o + 1;
  for (uint i = 0; i < ncu; i++) q5_build_customer_nation_map_kernel(cu_key, cn.data(), cmap.data(), &nation_mask, ncu, i);
  for (uint i = 0; i < nsu; i++) q5_build_supplier_nation_map_kernel(su_key, sn.data(), smap.data(), &nation_mask, nsu, i);
  std::vector<int> od = dates(n_or, or_date);
  int ds = yyyymmdd(date_lo), de = yyyymmdd(date_hi);
  for (uint i = 0; i < nor; i++)
    q5_build_orders_map_kernel(or_key, or_cust, od.data(), omap.data(), nor, ds, de, map_size, cmap.data(), i);
  std::vector<float> ext = hundredths(n_li, li_ext), dsc = hundredths(n_li, li_disc);
  std::vector<atomic_float> rev(25);
  for (auto& r : rev) r.v = 0.0f;
  run_groups((uint)groups, threads, [&](uint g) {
    q5_probe_and_aggregate_kernel(li_key, li_supp, ext.data(), dsc.data(), omap.data(), smap.data(), rev.data(), nli,
                                  map_size, g, 0, 1, (uint)groups);
  });
  for (int n = 0; n < 25; n++) revenue25[n] = rev[n].v;
}

// Q7 through q7_build_supplier_map_kernel, q7_build_customer_map_kernel,
// q7_build_orders_map_kernel and q7_probe_and_aggregate_kernel (kernels/q7.metal:12-109), with
// -1-filled maps; the kernel bins the years 1995 and 1996. bins4 = pair * 2 + year.
void ref_q7(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_nation, uint64_t n_su, const int32_t* su_key,
            const uint8_t* su_nation, uint64_t n_or, const int32_t* or_key, const int32_t* or_cust, uint64_t n_li,
            const int32_t* li_key, const int32_t* li_supp, const int32_t* li_ship, const int64_t* li_ext,
            const int32_t* li_disc, int32_t a, int32_t b, int32_t ship_lo, int32_t ship_hi, int groups, int threads,
            float* bins4) {
  const int max_o = std::max(max_of(n_or, or_key), max_of(n_li, li_key));
  std::vector<int> smap((size_t)max_of(n_su, su_key) + 1, -1), cmap((size_t)max_of(n_cu, cu_key) + 1, -1);
  std::vector<int> omap((size_t)max_o + 1, -1);
  std::vector<int> sn(su_nation, su_nation + n_su), cn(cu_nation, cu_nation + n_cu);
  uint nsu = (uint)n_su, ncu = (uint)n_cu, nor = (uint)n_or, nli = (uint)n_li, map_size = (uint)max_o + 1;
  for (uint i = 0; i < nsu; i++) q7_build_supplier_map_kernel(su_key, sn.data(), smap.data(), a, b, nsu, i);
  for (uint i = 0; i < ncu; i++) q7_build_customer_map_kernel(cu_key, cn.data(), cmap.data(), a, b, ncu, i);
  for (uint i = 0; i < nor; i++) q7_build_orders_map_kernel(or_key, or_cust, omap.data(), nor, i);
  std::vector<int> ls = dates(n_li, li_ship);
  std::vector<float> ext = hundredths(n_li, li_ext), dsc = hundredths(n_li, li_disc);
  std::vector<atomic_float> bins(4);
  for (auto& x : bins) x.v = 0.0f;
  int ds = yyyymmdd(ship_lo), de = yyyymmdd(ship_hi);
  run_groups((uint)groups, threads, [&](uint g) {
    q7_probe_and_aggregate_kernel(li_key, li_supp, ls.data(), ext.data(), dsc.data(), omap.data(), cmap.data(),
                                  smap.data(), bins.data(), nli, map_size, a, b, ds, de, g, 0, 1, (uint)groups);
  });
  for (int i = 0; i < 4; i++) bins4[i] = bins[i].v;
}

// Q8 through q8_build_orders_map_kernel and q8_probe_and_aggregate_kernel
// (kernels/q8.metal:9-76), with the host-side part bitmap (p_type == part_type), customer map
// of the region's nations and supplier map that the reference's driver builds; the kernel bins
// the years 1995 and 1996. bins4 = nation 1995, nation 1996, total 1995, total 1996.
void ref_q8(uint64_t n_cu, const int32_t* cu_key, const uint8_t* cu_nation, uint64_t n_su, const int32_t* su_key,
            const uint8_t* su_nation, uint64_t n_pa, const int32_t* pa_key, const uint8_t* pa_type, uint64_t n_or,
            const int32_t* or_key, const int32_t* or_cust, const int32_t* or_date, uint64_t n_li,
            const int32_t* li_key, const int32_t* li_part, const int32_t* li_supp, const int64_t* li_ext,
            const int32_t* li_disc, int32_t date_lo, int32_t date_hi, uint32_t region_mask, int32_t nation,
            int32_t part_type, int groups, int threads, float* bins4) {
  std::vector<uint> pbits((size_t)max_of(n_pa, pa_key) / 32 + 2, 0u);
  for (uint64_t i = 0; i < n_pa; i++)
    if (pa_type[i] == part_type) pbits[(uint)pa_key[i] >> 5] |= 1u << ((uint)pa_key[i] & 31u);
  std::vector<int> cmap((size_t)max_of(n_cu, cu_key) + 1, -1), smap((size_t)max_of(n_su, su_key) + 1, -1);
  for (uint64_t i = 0; i < n_cu; i++) if ((region_mask >> cu_nation[i]) & 1u) cmap[cu_key[i]] = cu_nation[i];
  for (uint64_t i = 0; i < n_su; i++) smap[su_key[i]] = su_nation[i];
  const int max_o = std::max(max_of(n_or, or_key), max_of(n_li, li_key));
  std::vector<int> ocust((size_t)max_o + 1, -1), oyear((size_t)max_o + 1, -1), od = dates(n_or, or_date);
  uint nor = (uint)n_or, nli = (uint)n_li, map_size = (uint)max_o + 1;
  int ds = yyyymmdd(date_lo), de = yyyymmdd(date_hi);
  for (uint i = 0; i < nor; i++)
    q8_build_orders_map_kernel(or_key, or_cust, od.data(), ocust.data(), oyear.data(), cmap.data(), nor, ds, de, i);
  std::vector<float> ext = hundredths(n_li, li_ext), dsc = hundredths(n_li, li_disc);
  std::vector<atomic_float> bins(4);
  for (auto& x : bins) x.v = 0.0f;
  run_groups((uint)groups, threads, [&](uint g) {
    q8_probe_and_aggregate_kernel(li_key, li_part, li_supp, ext.data(), dsc.data(), pbits.data(), ocust.data(),
                                  oyear.data(), smap.data(), bins.data(), nli, map_size, nation, g, 0, 1, (uint)groups);
  });
  for (int i = 0; i < 4; i++) bins4[i] = bins[i].v;
}

// Q10 through q10_build_orders_map_kernel and q10_probe_and_aggregate_kernel
// (kernels/q10.metal:8-54): float revenue per customer key (its customers are indexed by
// key: cust_rev has max key + 1 entries). Return flags are the characters A/N/R.
void ref_q10(uint64_t n_or, const int32_t* or_key, const int32_t* or_cust, const int32_t* or_date, uint64_t n_li,
             const int32_t* li_key, const uint8_t* li_flag, const int64_t* li_ext, const int32_t* li_disc,
             int32_t date_lo, int32_t date_hi, int groups, int threads, float* cust_rev, uint32_t n_cust) {
  int max_key = 0;
  for (uint64_t i = 0; i < n_or; i++) max_key = std::max(max_key, or_key[i]);
  for (uint64_t i = 0; i < n_li; i++) max_key = std::max(max_key, li_key[i]);
  uint map_size = (uint)max_key + 1, nor = (uint)n_or, nli = (uint)n_li;
  std::vector<int> omap(map_size, -1), od = dates(n_or, or_date);
  int ds = yyyymmdd(date_lo), de = yyyymmdd(date_hi);
  for (uint i = 0; i < nor; i++) q10_build_orders_map_kernel(or_key, or_cust, od.data(), omap.data(), nor, ds, de, i);
  std::vector<char> rf(n_li);
  for (uint64_t i = 0; i < n_li; i++) rf[i] = "ANR"[li_flag[i] % 3];
  std::vector<float> ext = hundredths(n_li, li_ext), dsc = hundredths(n_li, li_disc);
  std::vector<atomic_float> rev(n_cust);
  for (auto& r : rev) r.v = 0.0f;
  run_groups((uint)groups, threads, [&](uint g) {
    q10_probe_and_aggregate_kernel(li_key, rf.data(), ext.data(), dsc.data(), omap.data(), rev.data(), nli, map_size,
                                   g, 0, 1, (uint)groups);
  });
  for (uint32_t c = 0; c < n_cust; c++) cust_rev[c] = rev[c].v;
}

// Q13 through q13_pattern_match_kernel, q13_count_prefiltered_kernel and
// q13_build_histogram_kernel (kernels/q13.metal:33-168), with the reference's 80-byte comment
// stride and 256 bins. Its customer keys are 1-based (counts[ck - 1]): the synthetic keys
// 0..n_cu-1 go in as 1..n_cu. hist256[c] = customers with c qualifying orders.
void ref_q13(uint64_t n_cu, uint64_t n_or, const int32_t* or_cust, const char* or_comment, int groups, int threads,
             uint32_t* hist256) {
  uint nor = (uint)n_or, ncu = (uint)n_cu, stride = 80, bins = 256;
  std::vector<uchar> q(n_or);
  for (uint i = 0; i < nor; i++) q13_pattern_match_kernel(or_comment, q.data(), nor, stride, i);
  std::vector<int> ck(n_or);
  for (uint64_t i = 0; i < n_or; i++) ck[i] = or_cust[i] + 1;
  std::vector<atomic_uint> counts(n_cu);
  for (auto& c : counts) c.v = 0;
  run_groups((uint)groups, threads, [&](uint g) {
    q13_count_prefiltered_kernel(ck.data(), q.data(), counts.data(), nor, ncu, g, 0, 1, (uint)groups);
  });
  std::vector<atomic_uint> hist(bins);
  for (auto& h : hist) h.v = 0;
  const uint* cc = reinterpret_cast<const uint*>(counts.data());
  run_groups((uint)groups, threads, [&](uint g) {
    q13_build_histogram_kernel(cc, hist.data(), ncu, bins, g, 0, 1, (uint)groups);
  });
  for (uint b = 0; b < bins; b++) hist256[b] = hist[b].v;
}

// Q9 through q9_build_part_ht_kernel, q9_build_supplier_ht_kernel,
// q9_build_partsupp_ht_kernel, q9_build_orders_ht_kernel and q9_probe_and_global_agg_kernel
// (kernels/q9.metal:44-289). Part names carry "green" exactly for flagged parts; order
// dates are encoded so that date / 10000 is the synthetic order year. Writes groups
// (nation, year, profit in dollars) and returns their count.
uint32_t ref_q9(uint64_t n_pa, const int32_t* pa_key, const uint8_t* pa_flag,
                uint64_t n_su, const int32_t* su_key, const uint8_t* su_nation,
                uint64_t n_ps, const int32_t* ps_part, const int32_t* ps_supp, const int64_t* ps_cost,
                uint64_t n_or, const int32_t* or_key, const int32_t* or_date,
                uint64_t n_li, const int32_t* li_part, const int32_t* li_supp, const int32_t* li_order,
                const int64_t* li_ext, const int32_t* li_disc, const int32_t* li_qty,
                int groups, int threads, int32_t* g_nation, int32_t* g_year, float* g_profit, uint32_t cap) {
  uint npa = (uint)n_pa, nsu = (uint)n_su, nps = (uint)n_ps, nor = (uint)n_or, nli = (uint)n_li;
  std::vector<char> names((size_t)npa * 55, 'x');
  int max_part = 0;
  for (uint i = 0; i < npa; i++) {
    char* nm = &names[(size_t)i * 55];
    std::memcpy(nm, "forest blue lace", 16);
    if (pa_flag[i]) std::memcpy(nm + 20, "green", 5);
    nm[54] = '\0';
    max_part = std::max(max_part, pa_key[i]);
  }
  std::vector<atomic_uint> pbits((max_part + 31) / 32 + 1);
  for (auto& w : pbits) w.v = 0;
  for (uint i = 0; i < npa; i++) q9_build_part_ht_kernel(pa_key, names.data(), pbits.data(), npa, i, 0, 1);
  const uint* pbm = reinterpret_cast<const uint*>(pbits.data());

  int max_supp = 0;
  for (uint i = 0; i < nsu; i++) max_supp = std::max(max_supp, su_key[i]);
  std::vector<int> nation_of(n_su), smap((size_t)max_supp + 1, -1);
  for (uint i = 0; i < nsu; i++) nation_of[i] = su_nation[i];
  for (uint i = 0; i < nsu; i++) q9_build_supplier_ht_kernel(su_key, nation_of.data(), smap.data(), nsu, i, 0, 1);

  uint ps_size = next_pow2_u(nps);
  std::vector<PartSuppEntry> psht(ps_size);
  std::memset(psht.data(), 0xFF, psht.size() * sizeof(PartSuppEntry));
  for (uint i = 0; i < nps; i++) q9_build_partsupp_ht_kernel(ps_part, ps_supp, psht.data(), nps, ps_size, pbm, i, 0, 1);

  std::vector<int> oyear(n_or);
  for (uint i = 0; i < nor; i++) oyear[i] = (1992 + or_date[i] / 365) * 10000 + 101;
  uint or_size = next_pow2_u(nor * 2);
  std::vector<HashTableEntry> orht(or_size);
  std::memset(orht.data(), 0xFF, orht.size() * sizeof(HashTableEntry));
  for (uint i = 0; i < nor; i++) q9_build_orders_ht_kernel(or_key, oyear.data(), orht.data(), nor, or_size, i, 0, 1);

  std::vector<float> ext = hundredths(n_li, li_ext), dsc = hundredths(n_li, li_disc), qty = as_float(n_li, li_qty);
  std::vector<float> cost = hundredths(n_ps, ps_cost);
  uint agg_size = 256;
  std::vector<Q9Aggregates_Local> agg(agg_size);
  std::memset(agg.data(), 0, agg.size() * sizeof(Q9Aggregates_Local));
  auto* gagg = reinterpret_cast<Q9Aggregates*>(agg.data());
  uint zero = 0;
  run_groups((uint)groups, threads, [&](uint g) {
    q9_probe_and_global_agg_kernel(li_supp, li_part, li_order, ext.data(), dsc.data(), qty.data(), cost.data(),
                                   pbm, smap.data(), psht.data(), orht.data(), gagg, nli, zero, zero,
                                   ps_size, or_size, agg_size, g, 0, 1, (uint)groups);
  });
  uint32_t m = 0;
  for (uint i = 0; i < agg_size; i++) {
    if (agg[i].key == 0) continue;
    if (m < cap) { g_nation[m] = (int32_t)(agg[i].key >> 16); g_year[m] = (int32_t)(agg[i].key & 0xFFFF); g_profit[m] = agg[i].profit; }
    m++;
  }
  return m;
}

// ---- timed form of the two scans: the columns are converted once (the reference's load
// step, excluded from its GPU time), then the kernels run over them as often as asked ----
struct RefScan {
  uint64_t n;
  std::vector<int> ship;
  std::vector<float> qty, ext, disc, tax;
  std::vector<char> rf, ls;
};

void* ref_scan_prepare(uint64_t n, const int32_t* ship, const int32_t* qty, const int64_t* ext,
                       const int32_t* disc, const int32_t* tax, const uint8_t* flag, const uint8_t* status) {
  RefScan* s = new RefScan();
  s->n = n;
  s->ship = dates(n, ship);
  s->qty = as_float(n, qty);
  s->ext = hundredths(n, ext);
  s->disc = hundredths(n, disc);
  s->tax = hundredths(n, tax);
  s->rf.resize(n);
  s->ls.resize(n);
  for (uint64_t i = 0; i < n; i++) { s->rf[i] = "ANR"[flag[i] % 3]; s->ls[i] = "FO"[status[i] % 2]; }
  return s;
}

void ref_scan_free(void* h) { delete static_cast<RefScan*>(h); }

float ref_q6_run(void* h, int32_t lo, int32_t hi, int32_t dlo, int32_t dhi, int32_t qlt, int groups, int threads) {
  RefScan* s = static_cast<RefScan*>(h);
  std::vector<float> partial(groups);
  uint size = (uint)s->n;
  int start = yyyymmdd(lo), end = yyyymmdd(hi);
  float mind = (float)dlo / 100.0f, maxd = (float)dhi / 100.0f, maxq = (float)qlt;
  run_groups((uint)groups, threads, [&](uint g) {
    q6_filter_and_sum_stage1(s->ship.data(), s->disc.data(), s->qty.data(), s->ext.data(), partial.data(), size,
                             start, end, mind, maxd, maxq, g, 0, 1, (uint)groups);
  });
  float result = 0;
  uint ng = (uint)groups;
  q6_final_sum_stage2(partial.data(), &result, ng, 0);
  return result;
}

uint32_t ref_q1_run(void* h, int32_t ship_le, int groups, int threads) {
  RefScan* s = static_cast<RefScan*>(h);
  std::vector<atomic_uint> acc(60);
  for (auto& a : acc) a.v = 0;
  atomic_uint* A = acc.data();
  uint size = (uint)s->n;
  int cutoff = yyyymmdd(ship_le);
  run_groups((uint)groups, threads, [&](uint g) {
    q1_fused_kernel(s->ship.data(), s->rf.data(), s->ls.data(), s->qty.data(), s->ext.data(), s->disc.data(),
                    s->tax.data(), A + 0, A + 6, A + 12, A + 18, A + 24, A + 30, A + 36, A + 42, A + 48, A + 54,
                    size, cutoff, g, 0, 1, (uint)groups);
  });
  uint32_t rows = 0;
  for (int b = 0; b < 6; b++) rows += acc[54 + b].v;
  return rows;
}

// selection_kernel (kernels/microbenchmarks.metal:160-171): one 0/1 word per row.
void ref_select_lt(uint64_t n, const int32_t* col, int32_t value, uint32_t* out) {
  for (uint i = 0; i < (uint)n; i++) selection_kernel(col, out, value, i);
}

// sum_kernel_stage1/2 (kernels/microbenchmarks.metal:178-220) over the column as float.
float ref_sum(uint64_t n, const int32_t* col, int groups, int threads) {
  std::vector<float> v = as_float(n, col), partial(groups);
  uint size = (uint)n;
  run_groups((uint)groups, threads, [&](uint g) { sum_kernel_stage1(v.data(), partial.data(), size, g, 0, 1, (uint)groups); });
  float r = 0; uint ng = (uint)groups;
  sum_kernel_stage2(partial.data(), &r, ng, 0);
  return r;
}

// hash_join_build + hash_join_probe (kernels/microbenchmarks.metal:225-294).
uint32_t ref_join_count(uint64_t nb, const int32_t* bkeys, uint64_t np, const int32_t* pkeys) {
  uint size = (uint)nb * 2;
  std::vector<HashTableEntry> ht(size ? size : 1);
  std::memset(ht.data(), 0xFF, ht.size() * sizeof(HashTableEntry));
  uint nbu = (uint)nb, npu = (uint)np;
  for (uint i = 0; i < nbu; i++) hash_join_build(bkeys, bkeys, ht.data(), nbu, size, i);
  atomic_uint matches; matches.v = 0;
  for (uint i = 0; i < npu; i++) hash_join_probe(pkeys, ht.data(), &matches, npu, size, i);
  return matches.v;
}

// sf100_radix_histogram + sf100_radix_prefix_sum + sf100_radix_scatter
// (kernels/microbenchmarks.metal:15-99), one thread: the scatter keeps input order.
void ref_radix_partition(uint64_t n, const int32_t* keys, const int32_t* payload,
                         uint32_t* hist, uint32_t* offsets, int32_t* keys_out, int32_t* payload_out) {
  std::vector<atomic_uint> h(1024);
  for (auto& x : h) x.v = 0;
  uint nu = (uint)n;
  sf100_radix_histogram(keys, h.data(), nu, 0, 1, 0, 1);
  std::vector<uint> off(1024), tot(1024);
  for (int i = 0; i < 1024; i++) { hist[i] = h[i].v; off[i] = h[i].v; }
  uint parts = 1024;
  sf100_radix_prefix_sum(off.data(), tot.data(), parts, 0, 1);
  for (int i = 0; i < 1024; i++) offsets[i] = off[i];
  std::vector<atomic_uint> cur(1024);
  for (int i = 0; i < 1024; i++) cur[i].v = off[i];
  sf100_radix_scatter(keys, payload, keys_out, payload_out, cur.data(), nu, 0, 1);
}

// sf100_partition_join (kernels/microbenchmarks.metal:104-156) on one partition
// (build_count <= 16384). Returns the number of pairs, writes <= cap.
uint32_t ref_partition_join(uint64_t nb, const int32_t* bkeys, uint64_t np, const int32_t* pkeys,
                            int32_t* out_b, int32_t* out_p, uint32_t cap) {
  std::vector<int> bp(nb), pp(np);
  for (uint64_t i = 0; i < nb; i++) bp[i] = (int)i;
  for (uint64_t i = 0; i < np; i++) pp[i] = (int)i;
  // the kernel appends pairs without a bound: size its output for the exact pair count
  std::vector<int32_t> sorted(bkeys, bkeys + nb);
  std::sort(sorted.begin(), sorted.end());
  size_t pairs = 0;
  for (uint64_t i = 0; i < np; i++) {
    auto r = std::equal_range(sorted.begin(), sorted.end(), pkeys[i]);
    pairs += (size_t)(r.second - r.first);
  }
  std::vector<int> ob(pairs + 1), op(pairs + 1);
  atomic_uint cnt; cnt.v = 0;
  uint nbu = (uint)nb, npu = (uint)np;
  sf100_partition_join(bkeys, bp.data(), nbu, pkeys, pp.data(), npu, ob.data(), op.data(), &cnt, 0, 1);
  for (uint i = 0; i < cnt.v && i < cap; i++) { out_b[i] = ob[i]; out_p[i] = op[i]; }
  return cnt.v;
}

}  // extern "C"
