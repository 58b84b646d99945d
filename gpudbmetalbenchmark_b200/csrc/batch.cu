// Batched execution: many requests per call (gpudb_batch_run).
//
// Shared scans. Q6/Q1 requests over device-resident tables are grouped by (table, row
// range); each group is read from HBM once per pass, and every request of the group is
// evaluated on the rows while they are in registers:
//  - Q6 requests (up to kMaxQ6 per pass) keep per-thread register sums;
//  - Q1 requests (up to kMaxQ1 per pass) differ only in their ship_date cutoff, so the
//    cutoffs are sorted and a row falls in bucket j = number of cutoffs below its ship
//    date; it counts for every request whose sorted position is >= j. Rows are aggregated
//    per (bucket, group) with shared-memory atomics, and each request's totals are the
//    prefix sums over buckets 0..position. The per-row cost does not grow with the number
//    of Q1 requests.
// All groups' row tiles form one work list; a persistent grid pulls tiles from a device
// queue (one atomicAdd per tile), so a batch of many requests over several tables is one
// launch. Partial sums reach the requests' result words through integer atomics (exact and
// order-independent). Q3/Q9 requests are enqueued behind it on the same stream as ordinary
// async pipeline calls, so the whole batch needs one host synchronisation.
#include <algorithm>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace gpudb {
namespace {

constexpr int kBT = 256;
constexpr int kBW = kBT / 32;
constexpr uint64_t kTileRows = 8192;      // per warp per tile <= 1024 rows: packed Q1 fields cannot carry
constexpr int kMaxQ6 = 16;                // Q6 requests per pass (register sums)
constexpr int kMaxQ1 = 15;                // Q1 requests per pass (16 buckets incl. padding)
constexpr int kQ1Keys = (kMaxQ1 + 1) * 6; // (bucket, flag*2+status)
constexpr int kQ6Words = 2;               // revenue, rows matched
constexpr int kQ1Words = 72;              // 6 groups x 6 raw metrics x u128

struct ScanGroup {
  const int32_t *ship, *qty, *disc, *tax;
  const int64_t* ext;
  const uint8_t *flag, *stat;
  uint64_t begin, end;
  uint32_t n_q6, n_q1, vec, pad;
  int32_t q6p[kMaxQ6][5];                 // ship_lo, ship_hi, disc_lo, disc_hi, qty_lt
  uint32_t q6_res[kMaxQ6];                // first result word
  int32_t q1_cut[kMaxQ1 + 1];             // ascending; padded with INT32_MAX
  uint32_t q1_res[kMaxQ1];                // in cutoff order
  uint32_t q1_idx[kMaxQ1];                // status word of the request
};
struct ScanTile {
  uint32_t group, pad;
  uint64_t begin, end;
};

struct ScanSmem {
  ScanGroup g;
  unsigned long long wacc[kBW][kQ1Keys][4];   // per warp: packed (qty<<32|disc<<13|1), ext, ext*disc, (ext*100-ext*disc)*tax
  u128 bacc[kQ1Keys][6];                      // per block: count, qty, ext, ext*disc, ext*(100-disc)*tax, disc
  uint32_t bad[kMaxQ1 + 1];
  unsigned long long red[kBW][2];
  uint32_t tile;
};

__device__ __forceinline__ void atomic_add_u128(unsigned long long* p, u128 v) {
  const unsigned long long lo = (unsigned long long)v;
  unsigned long long hi = (unsigned long long)(v >> 64);
  const unsigned long long old = atomicAdd(p, lo);
  if (old + lo < old) hi++;
  if (hi) atomicAdd(p + 1, hi);
}

// Adds the block's sums for the current group to the requests' result words.
__device__ void flush_group(ScanSmem& S, const int64_t (&rev)[kMaxQ6], const uint32_t (&cnt)[kMaxQ6],
                            unsigned long long* res, uint32_t* req_status) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const ScanGroup& g = S.g;
#pragma unroll
  for (int r = 0; r < kMaxQ6; r++) {
    if (r >= (int)g.n_q6) break;
    const unsigned long long a = warp_sum_u64((unsigned long long)rev[r]), b = warp_sum_u64(cnt[r]);
    if (lane == 0) { S.red[warp][0] = a; S.red[warp][1] = b; }
    __syncthreads();
    if (t < 2) {
      unsigned long long v = 0;
      for (int w = 0; w < kBW; w++) v += S.red[w][t];
      if (v) atomicAdd(res + g.q6_res[r] + t, v);
    }
    __syncthreads();
  }
  // Q1: request at sorted position p = prefix over buckets 0..p
  for (uint32_t i = t; i < g.n_q1 * 36; i += kBT) {
    const uint32_t p = i / 36, gm = i % 36, grp = gm / 6, m = gm % 6;
    u128 v = 0;
    for (uint32_t j = 0; j <= p; j++) v += S.bacc[j * 6 + grp][m];
    if (v) atomic_add_u128(res + g.q1_res[p] + 2 * gm, v);
  }
  for (uint32_t p = t; p < g.n_q1; p += kBT) {
    uint32_t b = 0;
    for (uint32_t j = 0; j <= p; j++) b |= S.bad[j];
    if (b) atomicOr(req_status + g.q1_idx[p], ST_DOMAIN);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kBT) scan_batch_kernel(const ScanGroup* __restrict__ groups,
                                                         const ScanTile* __restrict__ tiles, uint32_t n_tiles,
                                                         unsigned* queue, unsigned long long* res, uint32_t* req_status) {
  extern __shared__ __align__(16) unsigned char scan_smem[];
  ScanSmem& S = *reinterpret_cast<ScanSmem*>(scan_smem);
  const int t = threadIdx.x, warp = t >> 5;
  int64_t rev[kMaxQ6];
  uint32_t cnt[kMaxQ6];
  uint32_t cur = 0xFFFFFFFFu;
  for (;;) {
    if (t == 0) S.tile = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t i = S.tile;
    const uint32_t gi = i < n_tiles ? tiles[i].group : 0xFFFFFFFFu;
    if (gi != cur) {   // block-uniform
      if (cur != 0xFFFFFFFFu) flush_group(S, rev, cnt, res, req_status);
      if (i >= n_tiles) break;
      for (uint32_t w = t; w < sizeof(ScanGroup) / 4; w += kBT)
        reinterpret_cast<uint32_t*>(&S.g)[w] = reinterpret_cast<const uint32_t*>(groups + gi)[w];
      for (uint32_t w = t; w < kQ1Keys * 6; w += kBT) (&S.bacc[0][0])[w] = 0;
      if (t <= kMaxQ1) S.bad[t] = 0;
#pragma unroll
      for (int r = 0; r < kMaxQ6; r++) { rev[r] = 0; cnt[r] = 0; }
      cur = gi;
      __syncthreads();   // the descriptor and cleared sums are visible to every thread
    }
    if (i >= n_tiles) break;   // a block that never got a tile
    const uint32_t nq6 = S.g.n_q6, nq1 = S.g.n_q1;
    if (nq1)
      for (uint32_t w = t; w < (uint32_t)kBW * (nq1 * 6) * 4; w += kBT) {
        const uint32_t wp = w / ((nq1 * 6) * 4), rest = w % ((nq1 * 6) * 4);
        S.wacc[wp][rest / 4][rest % 4] = 0;
      }
    __syncthreads();
    const ScanTile T = tiles[i];
    const bool vec = S.g.vec != 0;
    uint32_t bad = 0;
    for (uint64_t q = (T.begin >> 2) + t; q < ((T.end + 3) >> 2); q += kBT) {
      const uint64_t r0 = q << 2;
      int32_t sh[4], ds[4], qt[4], tx[4] = {0, 0, 0, 0};
      int64_t ex[4];
      uint32_t fl = 0xFFFFFFFFu, st = 0xFFFFFFFFu;
      bool ok[4];
      if (vec && r0 >= T.begin && r0 + 4 <= T.end) {
        const int4 a = ld_stream(reinterpret_cast<const int4*>(S.g.ship) + q);
        const int4 d = ld_stream(reinterpret_cast<const int4*>(S.g.disc) + q);
        const int4 b = ld_stream(reinterpret_cast<const int4*>(S.g.qty) + q);
        const longlong2 e0 = ld_stream(reinterpret_cast<const longlong2*>(S.g.ext) + 2 * q);
        const longlong2 e1 = ld_stream(reinterpret_cast<const longlong2*>(S.g.ext) + 2 * q + 1);
        sh[0] = a.x; sh[1] = a.y; sh[2] = a.z; sh[3] = a.w;
        ds[0] = d.x; ds[1] = d.y; ds[2] = d.z; ds[3] = d.w;
        qt[0] = b.x; qt[1] = b.y; qt[2] = b.z; qt[3] = b.w;
        ex[0] = e0.x; ex[1] = e0.y; ex[2] = e1.x; ex[3] = e1.y;
        if (nq1) {
          const int4 x = ld_stream(reinterpret_cast<const int4*>(S.g.tax) + q);
          tx[0] = x.x; tx[1] = x.y; tx[2] = x.z; tx[3] = x.w;
          fl = ld_stream(reinterpret_cast<const uint32_t*>(S.g.flag) + q);
          st = ld_stream(reinterpret_cast<const uint32_t*>(S.g.stat) + q);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) ok[k] = true;
      } else {
        fl = 0; st = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint64_t r = r0 + k;
          ok[k] = r >= T.begin && r < T.end;
          sh[k] = ok[k] ? S.g.ship[r] : 0;
          ds[k] = ok[k] ? S.g.disc[r] : 0;
          qt[k] = ok[k] ? S.g.qty[r] : 0;
          ex[k] = ok[k] ? S.g.ext[r] : 0;
          if (nq1) {
            tx[k] = ok[k] ? S.g.tax[r] : 0;
            fl |= (ok[k] ? (uint32_t)S.g.flag[r] : 0xFFu) << (8 * k);
            st |= (ok[k] ? (uint32_t)S.g.stat[r] : 0xFFu) << (8 * k);
          }
        }
      }
#pragma unroll
      for (int r = 0; r < kMaxQ6; r++) {
        if (r >= (int)nq6) break;
        const int32_t lo = S.g.q6p[r][0], hi = S.g.q6p[r][1], dlo = S.g.q6p[r][2], dhi = S.g.q6p[r][3], qlt = S.g.q6p[r][4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const bool m = ok[k] & (sh[k] >= lo) & (sh[k] < hi) & (ds[k] >= dlo) & (ds[k] <= dhi) & (qt[k] < qlt);
          rev[r] += m ? ex[k] * (int64_t)ds[k] : 0;
          cnt[r] += m;
        }
      }
      if (nq1) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint32_t f = (fl >> (8 * k)) & 0xFFu, s = (st >> (8 * k)) & 0xFFu;
          if (!ok[k] || f > 2u || s > 1u) continue;
          // bucket = number of cutoffs below the ship date (cutoffs padded with INT32_MAX)
          uint32_t j = 0;
#pragma unroll
          for (uint32_t step = 8; step > 0; step >>= 1)
            if (S.g.q1_cut[j + step - 1] < sh[k]) j += step;
          if (j >= nq1) continue;
          const int32_t qv = qt[k], dv = ds[k], tv = tx[k];
          const int64_t e = ex[k];
          const uint32_t viol = ((uint32_t)qv >= 65536u) | ((uint32_t)dv > 100u) | ((uint32_t)tv > 100u) |
                                ((uint64_t)e >= (1ull << 36));
          if (viol) { atomicOr(&S.bad[j], 1u); continue; }
          const uint64_t ed = (uint64_t)e * (uint32_t)dv;
          const uint64_t edt = ((uint64_t)e * 100u - ed) * (uint32_t)tv;
          unsigned long long* a = S.wacc[warp][j * 6 + f * 2 + s];
          atomicAdd(a + 0, ((uint64_t)(uint32_t)qv << 32) | ((uint64_t)(uint32_t)dv << 13) | 1u);
          atomicAdd(a + 1, (unsigned long long)e);
          atomicAdd(a + 2, (unsigned long long)ed);
          atomicAdd(a + 3, (unsigned long long)edt);
        }
      }
    }
    (void)bad;
    __syncthreads();
    if (nq1) {   // fold the warps' tile sums into the block's u128 sums
      for (uint32_t k = t; k < nq1 * 6; k += kBT) {
        u128 c = 0, qs = 0, ds = 0, e = 0, ed = 0, edt = 0;
        for (int w = 0; w < kBW; w++) {
          const unsigned long long P = S.wacc[w][k][0];
          c += P & 0x1FFFu;
          ds += (P >> 13) & 0x7FFFFu;
          qs += P >> 32;
          e += S.wacc[w][k][1];
          ed += S.wacc[w][k][2];
          edt += S.wacc[w][k][3];
        }
        S.bacc[k][0] += c; S.bacc[k][1] += qs; S.bacc[k][2] += e;
        S.bacc[k][3] += ed; S.bacc[k][4] += edt; S.bacc[k][5] += ds;
      }
      __syncthreads();
    }
  }
}

size_t scan_smem_bytes() { return (sizeof(ScanSmem) + 15) / 16 * 16; }

unsigned scan_grid(gpudb_ctx* ctx, uint32_t tiles) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scan_batch_kernel, kBT, scan_smem_bytes()) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return std::max<unsigned>(1, std::min<unsigned>(tiles, (unsigned)(ctx->sm_count * per_sm)));
}

bool scan_columns_ok(const gpudb_request& r) {
  const gpudb_lineitem* li = r.li;
  if (!li || li->location != GPUDB_MEM_DEVICE) return false;
  if (r.pipeline == GPUDB_PIPE_Q6) return li->ship_date && li->discount && li->quantity && li->ext_price;
  return li->ship_date && li->quantity && li->ext_price && li->discount && li->tax && li->flag && li->status;
}

bool aligned(const void* p, uintptr_t a) { return !p || (reinterpret_cast<uintptr_t>(p) % a) == 0; }

// Runs the scan requests `ids` of `reqs` as shared scans (fits one result slot).
int run_scan_batch(gpudb_ctx* ctx, gpudb_request* reqs, const std::vector<uint32_t>& ids, gpudb_timing* t,
                   const gpudb_exec* ex) {
  // group by (scan columns, row range); within a group, Q1 requests also share their
  // tax/flag/status columns, so they are sub-grouped by those
  using Key = std::tuple<const void*, const void*, const void*, const void*, uint64_t, uint64_t>;
  using Q1Cols = std::tuple<const void*, const void*, const void*>;
  struct Members {
    std::vector<uint32_t> q6;
    std::map<Q1Cols, std::vector<uint32_t>> q1;
  };
  std::map<Key, Members> by_table;   // -> positions in ids
  uint32_t words = 0;
  std::vector<uint32_t> offs(ids.size());
  for (uint32_t k = 0; k < ids.size(); k++) {
    const gpudb_request& q = reqs[ids[k]];
    const gpudb_lineitem* li = q.li;
    const uint64_t end = q.row_end ? std::min<uint64_t>(q.row_end, li->n_rows) : li->n_rows;
    const uint64_t begin = std::min<uint64_t>(q.row_begin, end);
    Members& m = by_table[Key(li->ship_date, li->quantity, li->discount, li->ext_price, begin, end)];
    if (q.pipeline == GPUDB_PIPE_Q6) m.q6.push_back(k);
    else m.q1[Q1Cols(li->tax, li->flag, li->status)].push_back(k);
    offs[k] = words;
    words += q.pipeline == GPUDB_PIPE_Q6 ? kQ6Words : kQ1Words;
  }
  std::vector<ScanGroup> groups;
  std::vector<ScanTile> tiles;
  for (auto& kv : by_table) {
    Members& mb = kv.second;
    for (auto& c : mb.q1)
      std::sort(c.second.begin(), c.second.end(),
                [&](uint32_t a, uint32_t b) { return reqs[ids[a]].q1.ship_le < reqs[ids[b]].q1.ship_le; });
    auto q1it = mb.q1.begin();
    size_t i6 = 0, i1 = 0;
    while (i6 < mb.q6.size() || q1it != mb.q1.end()) {
      ScanGroup g{};
      g.ship = static_cast<const int32_t*>(std::get<0>(kv.first));
      g.qty = static_cast<const int32_t*>(std::get<1>(kv.first));
      g.disc = static_cast<const int32_t*>(std::get<2>(kv.first));
      g.ext = static_cast<const int64_t*>(std::get<3>(kv.first));
      g.begin = std::get<4>(kv.first);
      g.end = std::get<5>(kv.first);
      for (; i6 < mb.q6.size() && g.n_q6 < (uint32_t)kMaxQ6; i6++, g.n_q6++) {
        const gpudb_q6_params& p = reqs[ids[mb.q6[i6]]].q6;
        const int32_t v[5] = {p.ship_lo, p.ship_hi, p.disc_lo, p.disc_hi, p.qty_lt};
        std::memcpy(g.q6p[g.n_q6], v, sizeof v);
        g.q6_res[g.n_q6] = offs[mb.q6[i6]];
      }
      if (q1it != mb.q1.end()) {
        g.tax = static_cast<const int32_t*>(std::get<0>(q1it->first));
        g.flag = static_cast<const uint8_t*>(std::get<1>(q1it->first));
        g.stat = static_cast<const uint8_t*>(std::get<2>(q1it->first));
        const std::vector<uint32_t>& l = q1it->second;
        for (; i1 < l.size() && g.n_q1 < (uint32_t)kMaxQ1; i1++, g.n_q1++) {
          g.q1_cut[g.n_q1] = reqs[ids[l[i1]]].q1.ship_le;
          g.q1_res[g.n_q1] = offs[l[i1]];
          g.q1_idx[g.n_q1] = l[i1];
        }
        if (i1 == l.size()) { ++q1it; i1 = 0; }
      }
      for (uint32_t j = g.n_q1; j <= (uint32_t)kMaxQ1; j++) g.q1_cut[j] = INT32_MAX;
      g.vec = aligned(g.ship, 16) && aligned(g.qty, 16) && aligned(g.disc, 16) && aligned(g.ext, 16) &&
              aligned(g.tax, 16) && aligned(g.flag, 4) && aligned(g.stat, 4);
      const uint32_t gi = (uint32_t)groups.size();
      groups.push_back(g);
      for (uint64_t b = g.begin; b < g.end;) {
        const uint64_t e = std::min<uint64_t>(g.end, (b / kTileRows + 1) * kTileRows);
        tiles.push_back(ScanTile{gi, 0, b, e});
        b = e;
      }
    }
  }
  const size_t status_bytes = ((ids.size() * 4 + 15) / 16) * 16;
  const size_t bytes = status_bytes + (size_t)words * 8;
  Call call(ctx, ex, t);
  int rc = call.begin(bytes);
  if (rc) return rc;
  uint8_t* dres = call.result<uint8_t>();
  if (!tiles.empty()) {
    void* desc = nullptr;
    const size_t qbytes = 256, gbytes = groups.size() * sizeof(ScanGroup), tbytes = tiles.size() * sizeof(ScanTile);
    rc = scratch(ctx, "batch.desc", qbytes + gbytes + tbytes + 256, &desc);
    if (rc) return rc;
    uint8_t* base = static_cast<uint8_t*>(desc);
    unsigned* queue = reinterpret_cast<unsigned*>(base);
    ScanGroup* dgrp = reinterpret_cast<ScanGroup*>(base + qbytes);
    ScanTile* dtile = reinterpret_cast<ScanTile*>(base + qbytes + ((gbytes + 15) / 16) * 16);
    // pageable sources: the copies stage the descriptors before returning
    GPUDB_CUDA(ctx, cudaMemsetAsync(queue, 0, 4, call.stream()));
    GPUDB_CUDA(ctx, cudaMemcpyAsync(dgrp, groups.data(), gbytes, cudaMemcpyHostToDevice, call.stream()));
    GPUDB_CUDA(ctx, cudaMemcpyAsync(dtile, tiles.data(), tbytes, cudaMemcpyHostToDevice, call.stream()));
    const size_t smem = scan_smem_bytes();
    GPUDB_CUDA(ctx, cudaFuncSetAttribute(scan_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned grid = scan_grid(ctx, (uint32_t)tiles.size());
    GPUDB_LAUNCH(call, scan_batch_kernel, grid, kBT, smem, (const ScanGroup*)dgrp, (const ScanTile*)dtile,
                 (uint32_t)tiles.size(), queue, reinterpret_cast<unsigned long long*>(dres + status_bytes),
                 reinterpret_cast<uint32_t*>(dres));
  }
  std::vector<uint32_t> ids_copy = ids;
  return call.finish(bytes, [reqs, ids_copy, offs, status_bytes, ctx](const uint8_t* h) {
    for (size_t k = 0; k < ids_copy.size(); k++) {
      gpudb_request& q = reqs[ids_copy[k]];
      uint32_t st;
      std::memcpy(&st, h + 4 * k, 4);
      q.status = status_to_error(ctx, st);
      const uint8_t* w = h + status_bytes + (size_t)offs[k] * 8;
      if (q.pipeline == GPUDB_PIPE_Q6) {
        if (q.q6_out) { std::memcpy(&q.q6_out->revenue, w, 8); std::memcpy(&q.q6_out->rows_matched, w + 8, 8); }
        continue;
      }
      if (!q.q1_out) continue;
      gpudb_q1_result& o = *q.q1_out;
      std::memset(&o, 0, sizeof o);
      for (int g = 0; g < 6; g++) {
        u128 m[6];
        std::memcpy(m, w + (size_t)g * 6 * 16, sizeof m);
        if (m[0] == 0) continue;
        const u128 disc_price = (u128)100 * m[2] - m[3];
        const u128 charge = (u128)100 * disc_price + m[4];
        gpudb_q1_group& G = o.groups[o.n_groups++];
        G.flag = (uint8_t)(g / 2);
        G.status = (uint8_t)(g % 2);
        G.count = (uint64_t)m[0];
        const u128 vals[5] = {m[1], m[2], disc_price, charge, m[5]};
        gpudb_i128* f[5] = {&G.sum_qty, &G.sum_base_price, &G.sum_disc_price, &G.sum_charge, &G.sum_discount};
        for (int j = 0; j < 5; j++) { f[j]->lo = (uint64_t)vals[j]; f[j]->hi = (int64_t)(uint64_t)(vals[j] >> 64); }
      }
    }
    return GPUDB_OK;
  });
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_batch_run(gpudb_ctx* ctx, gpudb_request* reqs, uint32_t n, gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (n && !reqs) return fail(ctx, GPUDB_E_INVALID, "batch: requests are NULL");
  gpudb_exec aex{1, 0, ex ? ex->stream : nullptr};
  std::vector<uint32_t> scans;
  size_t scan_bytes = 0;
  auto flush_scans = [&]() -> int {
    if (scans.empty()) return GPUDB_OK;
    int rc = run_scan_batch(ctx, reqs, scans, t, &aex);
    if (rc) for (uint32_t i : scans) reqs[i].status = rc;
    scans.clear();
    scan_bytes = 0;
    return GPUDB_OK;
  };
  for (uint32_t i = 0; i < n; i++) {
    gpudb_request& q = reqs[i];
    q.status = GPUDB_OK;
    int rc = GPUDB_OK;
    switch (q.pipeline) {
      case GPUDB_PIPE_Q6:
      case GPUDB_PIPE_Q1: {
        if ((q.pipeline == GPUDB_PIPE_Q6 && !q.q6_out) || (q.pipeline == GPUDB_PIPE_Q1 && !q.q1_out)) {
          rc = fail(ctx, GPUDB_E_INVALID, "batch: request %u has no result struct", i);
          break;
        }
        if (scan_columns_ok(q)) {
          const size_t b = (q.pipeline == GPUDB_PIPE_Q6 ? kQ6Words : kQ1Words) * 8 + 4;
          if (scan_bytes + b + 64 > kBigSlotBytes - kSlotHeader) flush_scans();
          scans.push_back(i);
          scan_bytes += b;
          break;
        }
        // host-resident or incomplete columns: the single-request path reports or streams it
        gpudb_lineitem view = q.li ? *q.li : gpudb_lineitem{};
        if (q.li && (q.row_begin || q.row_end)) {
          const uint64_t end = q.row_end ? std::min<uint64_t>(q.row_end, view.n_rows) : view.n_rows;
          const uint64_t b = std::min<uint64_t>(q.row_begin, end);
          view.n_rows = end - b;
          auto adv = [b](const void* p, size_t w) { return p ? (const void*)((const uint8_t*)p + b * w) : nullptr; };
          view.ship_date = (const int32_t*)adv(view.ship_date, 4); view.quantity = (const int32_t*)adv(view.quantity, 4);
          view.ext_price = (const int64_t*)adv(view.ext_price, 8); view.discount = (const int32_t*)adv(view.discount, 4);
          view.tax = (const int32_t*)adv(view.tax, 4); view.flag = (const uint8_t*)adv(view.flag, 1);
          view.status = (const uint8_t*)adv(view.status, 1);
        }
        ctx->status_sink = &q.status;
        rc = q.pipeline == GPUDB_PIPE_Q6 ? gpudb_q6_sum(ctx, q.li ? &view : nullptr, &q.q6, q.q6_out, nullptr, &aex)
                                         : gpudb_q1_group6(ctx, q.li ? &view : nullptr, &q.q1, q.q1_out, nullptr, &aex);
        ctx->status_sink = nullptr;
        break;
      }
      case GPUDB_PIPE_Q3:
        if (!q.q3 || !q.q3_out) { rc = fail(ctx, GPUDB_E_INVALID, "batch: Q3 request %u lacks tables/result", i); break; }
        ctx->status_sink = &q.status;
        rc = gpudb_q3_join_topk(ctx, &q.q3->cu, &q.q3->od, &q.q3->li, &q.q3p, q.q3_out, nullptr, &aex);
        ctx->status_sink = nullptr;
        break;
      case GPUDB_PIPE_Q9:
        if (!q.q9 || (!q.q9_out && q.q9_capacity)) { rc = fail(ctx, GPUDB_E_INVALID, "batch: Q9 request %u lacks tables", i); break; }
        ctx->status_sink = &q.status;
        rc = gpudb_q9_star(ctx, &q.q9->pa, &q.q9->su, &q.q9->ps, &q.q9->od, &q.q9->li, &q.q9p, q.q9_out, q.q9_capacity,
                           &q.q9_groups, nullptr, &aex);
        ctx->status_sink = nullptr;
        break;
      default:
        rc = fail(ctx, GPUDB_E_INVALID, "batch: request %u has unknown pipeline %d", i, q.pipeline);
    }
    if (rc != GPUDB_OK) q.status = rc;
  }
  flush_scans();
  if (ex && ex->async) return GPUDB_OK;
  gpudb_sync(ctx);   // per-request outcomes are in each status
  return GPUDB_OK;
}
