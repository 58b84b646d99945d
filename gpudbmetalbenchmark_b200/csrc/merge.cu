// Exact merges of shard results on the host (multi-GPU row shards, or one table split over
// several calls): Q6/Q1 partial sums add, Q9 groups add per (nation, year), Q3 top-k lists
// of order-disjoint shards merge into the top k of their union. No device work.
#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include "../../include/gpudb_capi.h"

namespace {

typedef __int128 i128;

i128 get(const gpudb_i128& v) { return (i128)(((unsigned __int128)(uint64_t)v.hi << 64) | v.lo); }
void put(gpudb_i128& v, i128 x) {
  v.lo = (uint64_t)x;
  v.hi = (int64_t)(x >> 64);
}

}  // namespace

extern "C" int gpudb_q6_result_merge(const gpudb_q6_result* parts, uint32_t n, gpudb_q6_result* out) {
  if (!out || (n && !parts)) return GPUDB_E_INVALID;
  gpudb_q6_result r{0, 0};
  for (uint32_t i = 0; i < n; i++) {
    r.revenue += parts[i].revenue;
    r.rows_matched += parts[i].rows_matched;
  }
  *out = r;
  return GPUDB_OK;
}

extern "C" int gpudb_q1_result_merge(const gpudb_q1_result* parts, uint32_t n, gpudb_q1_result* out) {
  if (!out || (n && !parts)) return GPUDB_E_INVALID;
  struct Acc { uint64_t count = 0; i128 s[5] = {0, 0, 0, 0, 0}; };
  Acc acc[6];
  for (uint32_t i = 0; i < n; i++) {
    if (parts[i].n_groups > 6) return GPUDB_E_INVALID;
    for (uint32_t g = 0; g < parts[i].n_groups; g++) {
      const gpudb_q1_group& x = parts[i].groups[g];
      if (x.flag > 2 || x.status > 1) return GPUDB_E_INVALID;
      Acc& a = acc[x.flag * 2 + x.status];
      a.count += x.count;
      const gpudb_i128* f[5] = {&x.sum_qty, &x.sum_base_price, &x.sum_disc_price, &x.sum_charge, &x.sum_discount};
      for (int m = 0; m < 5; m++) a.s[m] += get(*f[m]);
    }
  }
  gpudb_q1_result r;
  std::memset(&r, 0, sizeof r);
  for (int g = 0; g < 6; g++) {
    if (!acc[g].count) continue;
    gpudb_q1_group& o = r.groups[r.n_groups++];
    o.flag = (uint8_t)(g / 2);
    o.status = (uint8_t)(g % 2);
    o.count = acc[g].count;
    gpudb_i128* f[5] = {&o.sum_qty, &o.sum_base_price, &o.sum_disc_price, &o.sum_charge, &o.sum_discount};
    for (int m = 0; m < 5; m++) put(*f[m], acc[g].s[m]);
  }
  *out = r;
  return GPUDB_OK;
}

extern "C" int gpudb_q9_result_merge(const gpudb_q9_group* groups, const uint32_t* counts, uint32_t n,
                                     gpudb_q9_group* out, uint32_t capacity, uint32_t* n_out) {
  if (!n_out || (n && !counts) || (capacity && !out)) return GPUDB_E_INVALID;
  // nation asc, year desc
  std::map<std::pair<int32_t, int32_t>, int64_t> m;
  size_t at = 0;
  for (uint32_t i = 0; i < n; i++) {
    if (counts[i] && !groups) return GPUDB_E_INVALID;
    for (uint32_t j = 0; j < counts[i]; j++, at++) {
      const gpudb_q9_group& g = groups[at];
      m[{g.nation, -g.year}] += g.profit;
    }
  }
  uint32_t k = 0;
  for (const auto& kv : m) {
    if (k < capacity) out[k] = gpudb_q9_group{kv.first.first, -kv.first.second, kv.second};
    k++;
  }
  *n_out = k;
  return GPUDB_OK;
}

extern "C" int gpudb_q3_result_merge(const gpudb_q3_result* parts, uint32_t n, int32_t k, gpudb_q3_result* out) {
  if (!out || (n && !parts) || k < 1 || k > GPUDB_Q3_MAX_K) return GPUDB_E_INVALID;
  std::vector<gpudb_q3_row> rows;
  uint64_t groups = 0;
  int32_t mode = n ? parts[0].join_mode : GPUDB_JOIN_GLOBAL;
  for (uint32_t i = 0; i < n; i++) {
    if (parts[i].n_rows > GPUDB_Q3_MAX_K) return GPUDB_E_INVALID;
    groups += parts[i].n_groups;
    rows.insert(rows.end(), parts[i].rows, parts[i].rows + parts[i].n_rows);
    if (parts[i].join_mode != mode) mode = GPUDB_JOIN_AUTO;   // shards ran in different modes
  }
  // revenue desc, order_date asc, order_key asc (the order of every Q3 result)
  std::sort(rows.begin(), rows.end(), [](const gpudb_q3_row& a, const gpudb_q3_row& b) {
    if (a.revenue != b.revenue) return a.revenue > b.revenue;
    if (a.order_date != b.order_date) return a.order_date < b.order_date;
    return a.order_key < b.order_key;
  });
  gpudb_q3_result r;
  std::memset(&r, 0, sizeof r);
  r.n_groups = groups;
  r.join_mode = mode;
  r.n_rows = (uint32_t)std::min<size_t>(rows.size(), (size_t)k);
  std::copy(rows.begin(), rows.begin() + r.n_rows, r.rows);
  *out = r;
  return GPUDB_OK;
}
