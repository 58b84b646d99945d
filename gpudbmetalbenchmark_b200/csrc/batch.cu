// Batched execution: many requests per call (gpudb_batch_run).
//
// Shared scans. Q6/Q1 requests over device-resident tables are grouped by (table, row
// range); each group is read from HBM once per pass, and every request of the group is
// evaluated on the rows while they are in registers:
//  - a quad of rows whose ship dates no request can accept skips its other columns;
//  - Q6 requests (up to kMaxQ6 per pass) keep per-thread register sums;
//  - Q1 requests (up to kMaxQ1 per pass) differ only in their ship_date cutoff, so the
//    cutoffs are sorted and a row falls in bucket j = number of cutoffs below its ship
//    date; it counts for every request whose sorted position is >= j. Each thread keeps
//    private shared-memory sums per (bucket, flag, status) (no atomics; shared memory
//    bounds the buckets of one pass), and each request's totals are the prefix sums over
//    buckets 0..position.
// All groups' row tiles form one work list; a persistent grid pulls tiles from a device
// queue (one atomicAdd per tile), so a batch of many requests over several tables is one
// launch. Partial sums reach the requests' result words through integer atomics (exact and
// order-independent). Q3 requests over the same tables run as batched Q3 launches (q3batch.cu),
// and the other joins are enqueued behind them on the same stream as ordinary async
// pipeline calls, so the whole batch needs one host synchronisation.
#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "q3.h"
#include "scans.h"

namespace gpudb {
namespace {

constexpr int kBT = 256;
constexpr int kBW = kBT / 32;
constexpr uint64_t kTileRows = 8192;      // 32 rows per thread per tile
constexpr int kFoldTiles = 16;            // per-thread Q1 sums fold into the block's every 16 tiles (<= 512
                                          // rows): the packed count/discount fields and u64 sums cannot carry
constexpr int kMaxQ6 = 8;                 // Q6 requests per Q6 pass (register sums)
constexpr int kMaxQ6WithQ1 = 4;           // Q6 requests riding along a Q1 pass
constexpr int kMaxQ1 = 2;                 // Q1 requests per pass (one bucket of per-thread sums each)
constexpr int kQ6Words = 2;               // revenue, rows matched
constexpr int kQ1Words = 72;              // 6 groups x 6 raw metrics x u128

struct ScanGroup {
  const int32_t *ship, *qty, *disc, *tax;
  const int64_t* ext;
  const uint8_t *flag, *stat;
  uint64_t begin, end;
  uint32_t n_q6, n_q1, vec, pad;
  int32_t ship_lo, ship_hi;               // union of the Q6 ship ranges, [lo, hi)
  int32_t q6p[kMaxQ6][5];                 // ship_lo, ship_hi, disc_lo, disc_hi, qty_lt
  uint32_t q6_res[kMaxQ6];                // first result word
  int32_t q1_cut[kMaxQ1];                 // ascending
  uint32_t q1_res[kMaxQ1];                // in cutoff order
  uint32_t q1_idx[kMaxQ1];                // status word of the request
};
struct ScanTile {
  uint32_t group, pad;
  uint64_t begin, end;
};

template <int NB>
struct ScanSmem {
  static constexpr int kKeys = NB > 0 ? NB * 6 : 1;   // (bucket, flag*2+status)
  // per-thread Q1 sums, [metric][key][thread]: packed (qty<<32|disc<<13|1), ext, ext*disc,
  // (ext*100-ext*disc)*tax
  unsigned long long acc[NB > 0 ? 4 : 1][kKeys][NB > 0 ? kBT : 1];
  u128 bacc[kKeys][6];                    // per block: count, qty, ext, ext*disc, ext*(100-disc)*tax, disc
  ScanGroup g;
  uint32_t bad[NB > 0 ? NB : 1];
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

// Folds the per-thread Q1 sums into the block's u128 sums and clears them.
template <int NB>
__device__ void fold_q1(ScanSmem<NB>& S, uint32_t nq1) {
  __syncthreads();
  const uint32_t keys = nq1 * 6;
  for (uint32_t k = threadIdx.x; k < keys * 4; k += kBT) {
    const uint32_t key = k / 4, m = k % 4;
    const unsigned long long* row = S.acc[m][key];
    if (m == 0) {
      u128 c = 0, qs = 0, ds = 0;
      for (int t = 0; t < kBT; t++) {
        const unsigned long long P = row[t];
        c += P & 0x1FFFu;
        ds += (P >> 13) & 0x7FFFFu;
        qs += P >> 32;
      }
      S.bacc[key][0] += c; S.bacc[key][1] += qs; S.bacc[key][5] += ds;
    } else {
      u128 v = 0;
      for (int t = 0; t < kBT; t++) v += row[t];
      S.bacc[key][1 + m] += v;   // ext -> 2, ext*disc -> 3, charge -> 4
    }
  }
  __syncthreads();
  for (uint32_t m = 0; m < 4; m++)
    for (uint32_t key = 0; key < keys; key++) S.acc[m][key][threadIdx.x] = 0;
}

// Adds the block's sums for the current group to the requests' result words.
template <int NB, int Q6>
__device__ void flush_group(ScanSmem<NB>& S, const int64_t (&rev)[Q6], const uint32_t (&cnt)[Q6],
                            unsigned long long* res, uint32_t* req_status) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const ScanGroup& g = S.g;
  if (NB > 0 && g.n_q1) fold_q1<NB>(S, g.n_q1);
#pragma unroll
  for (int r = 0; r < Q6; r++) {
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
  if (NB == 0) return;
  // Q1: bucket j holds the rows whose ship date is above cutoffs 0..j-1 and at most cutoff j,
  // so the request at sorted position p takes buckets 0..p
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

// One quad (4 consecutive rows) of the columns a pass needs.
struct Quad {
  int32_t sh[4], ds[4], qt[4], tx[4];
  int64_t ex[4];
  uint32_t fl, st;   // 4 packed bytes; 0xFF = no row
  bool ok[4];
  bool need;         // some row may pass some request
};

__device__ __forceinline__ bool full_quad(bool vec, uint64_t q, uint64_t b, uint64_t e) {
  return vec && (q << 2) >= b && (q << 2) + 4 <= e;
}

// Ship dates of quad q (rows 4q..4q+3 within [b, e)), and whether some row can pass a
// Q6 request of the group (only then are the other columns of a Q6 pass loaded).
__device__ __forceinline__ void load_ship(const ScanGroup& g, uint64_t q, uint64_t b, uint64_t e, bool vec, Quad& d) {
  if (full_quad(vec, q, b, e)) {
    const int4 a = ld_stream(reinterpret_cast<const int4*>(g.ship) + q);
    d.sh[0] = a.x; d.sh[1] = a.y; d.sh[2] = a.z; d.sh[3] = a.w;
#pragma unroll
    for (int k = 0; k < 4; k++) d.ok[k] = true;
  } else {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint64_t r = (q << 2) + k;
      d.ok[k] = r >= b && r < e;
      d.sh[k] = d.ok[k] ? g.ship[r] : 0;
    }
  }
  bool need = false;
#pragma unroll
  for (int k = 0; k < 4; k++) need |= d.ok[k] & (d.sh[k] >= g.ship_lo) & (d.sh[k] < g.ship_hi);
  d.need = need;
}

// The other columns of quad q (Q1 columns when Q1).
template <bool Q1>
__device__ __forceinline__ void load_rest(const ScanGroup& g, uint64_t q, bool vec, Quad& d) {
  if (vec && d.ok[0] && d.ok[3]) {
    const int4 dd = ld_stream(reinterpret_cast<const int4*>(g.disc) + q);
    const int4 b = ld_stream(reinterpret_cast<const int4*>(g.qty) + q);
    const longlong2 e0 = ld_stream(reinterpret_cast<const longlong2*>(g.ext) + 2 * q);
    const longlong2 e1 = ld_stream(reinterpret_cast<const longlong2*>(g.ext) + 2 * q + 1);
    d.ds[0] = dd.x; d.ds[1] = dd.y; d.ds[2] = dd.z; d.ds[3] = dd.w;
    d.qt[0] = b.x; d.qt[1] = b.y; d.qt[2] = b.z; d.qt[3] = b.w;
    d.ex[0] = e0.x; d.ex[1] = e0.y; d.ex[2] = e1.x; d.ex[3] = e1.y;
    if (Q1) {
      const int4 x = ld_stream(reinterpret_cast<const int4*>(g.tax) + q);
      d.tx[0] = x.x; d.tx[1] = x.y; d.tx[2] = x.z; d.tx[3] = x.w;
      d.fl = ld_stream(reinterpret_cast<const uint32_t*>(g.flag) + q);
      d.st = ld_stream(reinterpret_cast<const uint32_t*>(g.stat) + q);
    }
  } else {
    d.fl = 0;
    d.st = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint64_t r = (q << 2) + k;
      const bool ok = d.ok[k];
      d.ds[k] = ok ? g.disc[r] : 0;
      d.qt[k] = ok ? g.qty[r] : 0;
      d.ex[k] = ok ? g.ext[r] : 0;
      if (Q1) {
        d.tx[k] = ok ? g.tax[r] : 0;
        d.fl |= (ok ? (uint32_t)g.flag[r] : 0xFFu) << (8 * k);
        d.st |= (ok ? (uint32_t)g.stat[r] : 0xFFu) << (8 * k);
      }
    }
  }
}

template <int NB, int Q6>
__device__ __forceinline__ void eval_quad(ScanSmem<NB>& S, const Quad& d, int64_t (&rev)[Q6], uint32_t (&cnt)[Q6],
                                          uint32_t nq6, uint32_t nq1) {
#pragma unroll
  for (int r = 0; r < Q6; r++) {
    if (r >= (int)nq6) break;
    const int32_t lo = S.g.q6p[r][0], hi = S.g.q6p[r][1], dlo = S.g.q6p[r][2], dhi = S.g.q6p[r][3], qlt = S.g.q6p[r][4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const bool m = d.ok[k] & (d.sh[k] >= lo) & (d.sh[k] < hi) & (d.ds[k] >= dlo) & (d.ds[k] <= dhi) & (d.qt[k] < qlt);
      rev[r] += m ? d.ex[k] * (int64_t)d.ds[k] : 0;
      cnt[r] += m;
    }
  }
  if (NB == 0) return;
  const int t = threadIdx.x;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t f = (d.fl >> (8 * k)) & 0xFFu, s = (d.st >> (8 * k)) & 0xFFu;
    uint32_t j = 0;   // bucket = number of cutoffs below the ship date
#pragma unroll
    for (int c = 0; c < (NB > 0 ? NB : 1); c++) j += (uint32_t)(c < (int)nq1) & (uint32_t)(S.g.q1_cut[c] < d.sh[k]);
    if (!d.ok[k] || f > 2u || s > 1u || j >= nq1) continue;
    const int32_t qv = d.qt[k], dv = d.ds[k], tv = d.tx[k];
    const int64_t e = d.ex[k];
    const uint32_t viol = ((uint32_t)qv >= 65536u) | ((uint32_t)dv > 100u) | ((uint32_t)tv > 100u) |
                          ((uint64_t)e >= (1ull << 36));
    if (viol) { atomicOr(&S.bad[j], 1u); continue; }
    const uint64_t ed = (uint64_t)e * (uint32_t)dv;
    const uint64_t edt = ((uint64_t)e * 100u - ed) * (uint32_t)tv;
    const uint32_t key = j * 6 + f * 2 + s;
    S.acc[0][key][t] += ((uint64_t)(uint32_t)qv << 32) | ((uint64_t)(uint32_t)dv << 13) | 1u;
    S.acc[1][key][t] += (uint64_t)e;
    S.acc[2][key][t] += ed;
    S.acc[3][key][t] += edt;
  }
}

// Persistent pass over the tiles of a set of groups. NB = 0: Q6 groups (ship dates first,
// the other columns only where a request's date range can match); NB > 0: groups with up
// to NB Q1 requests (and Q6 requests riding along), every column loaded at once.
template <int NB, int Q6>
__global__ void __launch_bounds__(kBT) scan_pass_kernel(const ScanGroup* __restrict__ groups,
                                                        const ScanTile* __restrict__ tiles, uint32_t n_tiles,
                                                        unsigned* queue, unsigned long long* res, uint32_t* req_status) {
  extern __shared__ __align__(16) unsigned char scan_smem[];
  ScanSmem<NB>& S = *reinterpret_cast<ScanSmem<NB>*>(scan_smem);
  const int t = threadIdx.x;
  int64_t rev[Q6];
  uint32_t cnt[Q6];
  uint32_t cur = 0xFFFFFFFFu;
  int since_fold = 0;
  for (;;) {
    if (t == 0) S.tile = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t i = S.tile;
    const uint32_t gi = i < n_tiles ? tiles[i].group : 0xFFFFFFFFu;
    if (gi != cur) {   // block-uniform
      if (cur != 0xFFFFFFFFu) flush_group<NB, Q6>(S, rev, cnt, res, req_status);
      if (i >= n_tiles) break;
      for (uint32_t w = t; w < sizeof(ScanGroup) / 4; w += kBT)
        reinterpret_cast<uint32_t*>(&S.g)[w] = reinterpret_cast<const uint32_t*>(groups + gi)[w];
      if (NB > 0) {
        for (uint32_t w = t; w < ScanSmem<NB>::kKeys * 6; w += kBT) (&S.bacc[0][0])[w] = 0;
        if (t < NB) S.bad[t] = 0;
        for (int m = 0; m < 4; m++)
          for (int key = 0; key < ScanSmem<NB>::kKeys; key++) S.acc[m][key][t] = 0;
      }
#pragma unroll
      for (int r = 0; r < Q6; r++) { rev[r] = 0; cnt[r] = 0; }
      cur = gi;
      since_fold = 0;
      __syncthreads();   // the descriptor and cleared sums are visible to every thread
    }
    if (i >= n_tiles) break;   // a block that never got a tile
    const uint32_t nq6 = S.g.n_q6, nq1 = S.g.n_q1;
    if (NB > 0) {
      if (since_fold == kFoldTiles) { fold_q1<NB>(S, nq1); since_fold = 0; }
      since_fold++;
    }
    const ScanTile T = tiles[i];
    const bool vec = S.g.vec != 0;
    const uint64_t q_end = (T.end + 3) >> 2;
    for (uint64_t q = (T.begin >> 2) + t; q < q_end; q += 2 * kBT) {   // two quads in flight per thread
      Quad a, b;
      const bool has_b = q + kBT < q_end;
      load_ship(S.g, q, T.begin, T.end, vec, a);
      if (has_b) load_ship(S.g, q + kBT, T.begin, T.end, vec, b);
      if (NB > 0) {
        a.need = true;
        b.need = has_b;
      } else if (!has_b) {
        b.need = false;
      }
      if (a.need) load_rest<(NB > 0)>(S.g, q, vec, a);
      if (b.need) load_rest<(NB > 0)>(S.g, q + kBT, vec, b);
      if (a.need) eval_quad<NB, Q6>(S, a, rev, cnt, nq6, nq1);
      if (b.need) eval_quad<NB, Q6>(S, b, rev, cnt, nq6, nq1);
    }
    __syncthreads();
  }
}

template <int NB, int Q6>
size_t pass_smem() { return (sizeof(ScanSmem<NB>) + 15) / 16 * 16; }

template <int NB, int Q6>
int launch_pass(gpudb_ctx* ctx, Call& call, const ScanGroup* dgrp, const std::vector<ScanTile>& tiles, ScanTile* dtile,
                unsigned* queue, unsigned long long* res, uint32_t* status) {
  if (tiles.empty()) return GPUDB_OK;
  auto kern = scan_pass_kernel<NB, Q6>;
  const size_t smem = pass_smem<NB, Q6>();
  GPUDB_CUDA(ctx, kernel_smem(ctx, (const void*)kern, smem));
  const int per_sm = kernel_occupancy(ctx, (const void*)kern, kBT, smem);
  const unsigned grid = std::max<unsigned>(1, std::min<unsigned>((unsigned)tiles.size(), (unsigned)(ctx->sm_count * per_sm)));
  GPUDB_CUDA(ctx, cudaMemcpyAsync(dtile, tiles.data(), tiles.size() * sizeof(ScanTile), cudaMemcpyHostToDevice, call.stream()));
  GPUDB_LAUNCH(call, kern, grid, kBT, smem, dgrp, (const ScanTile*)dtile, (uint32_t)tiles.size(), queue, res, status);
  return GPUDB_OK;
}

bool scan_columns_ok(const gpudb_request& r) {
  const gpudb_lineitem* li = r.li;
  if (!li || li->location != GPUDB_MEM_DEVICE) return false;
  if (r.pipeline == GPUDB_PIPE_Q6) return li->ship_date && li->discount && li->quantity && li->ext_price;
  return li->ship_date && li->quantity && li->ext_price && li->discount && li->tax && li->flag && li->status;
}

bool aligned(const void* p, uintptr_t a) { return !p || (reinterpret_cast<uintptr_t>(p) % a) == 0; }

// Q1 result from the raw words of one request: 6 groups x {count, qty, ext, ext*disc,
// ext*(100-disc)*tax, disc} as u128.
void q1_from_words(const uint8_t* w, gpudb_q1_result& o) {
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

// Runs the scan requests `ids` of `reqs` as shared scans (fits one result slot).
gpudb_lineitem row_view(const gpudb_lineitem& li, uint64_t begin, uint64_t end);

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
  std::vector<ScanTile> tiles6, tiles1, tiles11;   // Q6 passes, Q1 passes of two / of one Q1 request
  // Few requests on one table run the single-request kernels (both at the copy peak)
  // instead of shared passes, whose per-row work for several requests makes them
  // instruction-bound: over 60M rows a Q1 pass takes about 0.45 ms (two Q1 requests, Q6
  // requests riding along) and a Q6 pass about 0.3 ms, against 0.23 ms for the Q1 kernel and
  // 0.14 ms for the Q6 kernel. So up to kSoloQ1 Q1 requests on the same columns, and up to
  // kSoloQ6 Q6 requests of a table without a Q1 pass, run alone.
  // One Q1 request with up to kRideQ6 Q6 requests on its table runs the Q1 kernel with the
  // Q6 requests riding along (one read of the rows for all of them, at the Q1 kernel's speed).
  constexpr size_t kSoloQ1 = 2, kSoloQ6 = 3, kRideQ6 = 4;
  struct Riding {
    uint32_t q1;
    std::vector<uint32_t> q6;
    gpudb_lineitem view;
  };
  std::vector<Riding> riding;
  std::vector<std::pair<uint32_t, gpudb_lineitem>> solo_scans;   // (position in ids, row range view)
  std::vector<char> solo(ids.size(), 0);
  for (auto& kv : by_table) {
    Members& mb = kv.second;
    auto take_solo = [&](uint32_t k) {
      solo_scans.emplace_back(k, row_view(*reqs[ids[k]].li, std::get<4>(kv.first), std::get<5>(kv.first)));
      solo[k] = 1;
    };
    if (mb.q1.size() == 1 && mb.q1.begin()->second.size() == 1 && !mb.q6.empty() && mb.q6.size() <= kRideQ6) {
      const uint32_t k = mb.q1.begin()->second[0];
      riding.push_back(Riding{k, mb.q6, row_view(*reqs[ids[k]].li, std::get<4>(kv.first), std::get<5>(kv.first))});
      solo[k] = 1;
      for (uint32_t j : mb.q6) solo[j] = 1;
      mb.q1.clear();
      mb.q6.clear();
    }
    for (auto it = mb.q1.begin(); it != mb.q1.end();) {
      if (it->second.size() <= kSoloQ1) {
        for (uint32_t k : it->second) take_solo(k);
        it = mb.q1.erase(it);
      } else {
        ++it;
      }
    }
    if (mb.q1.empty() && mb.q6.size() <= kSoloQ6) {
      for (uint32_t k : mb.q6) take_solo(k);
      mb.q6.clear();
    }
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
      const bool q1pass = q1it != mb.q1.end();
      if (q1pass) {   // up to kMaxQ1 Q1 requests of one column set, Q6 requests riding along
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
      g.ship_lo = INT32_MAX;
      g.ship_hi = INT32_MIN;
      const uint32_t max6 = q1pass ? kMaxQ6WithQ1 : kMaxQ6;
      for (; i6 < mb.q6.size() && g.n_q6 < max6; i6++, g.n_q6++) {
        const gpudb_q6_params& p = reqs[ids[mb.q6[i6]]].q6;
        if (p.ship_lo < p.ship_hi) {
          g.ship_lo = std::min(g.ship_lo, p.ship_lo);
          g.ship_hi = std::max(g.ship_hi, p.ship_hi);
        }
        const int32_t v[5] = {p.ship_lo, p.ship_hi, p.disc_lo, p.disc_hi, p.qty_lt};
        std::memcpy(g.q6p[g.n_q6], v, sizeof v);
        g.q6_res[g.n_q6] = offs[mb.q6[i6]];
      }
      g.vec = aligned(g.ship, 16) && aligned(g.qty, 16) && aligned(g.disc, 16) && aligned(g.ext, 16) &&
              aligned(g.tax, 16) && aligned(g.flag, 4) && aligned(g.stat, 4);
      const uint32_t gi = (uint32_t)groups.size();
      groups.push_back(g);
      // a pass with one Q1 request keeps half the per-thread sums (twice the blocks per SM)
      std::vector<ScanTile>& tl = q1pass ? (g.n_q1 == 1 ? tiles11 : tiles1) : tiles6;
      for (uint64_t b = g.begin; b < g.end;) {
        const uint64_t e = std::min<uint64_t>(g.end, (b / kTileRows + 1) * kTileRows);
        tl.push_back(ScanTile{gi, 0, b, e});
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
  if (!groups.empty()) {
    void* desc = nullptr;
    const size_t qbytes = 256, gbytes = ((groups.size() * sizeof(ScanGroup) + 15) / 16) * 16;
    const size_t t6 = ((tiles6.size() * sizeof(ScanTile) + 15) / 16) * 16;
    const size_t t1 = ((tiles1.size() * sizeof(ScanTile) + 15) / 16) * 16, t11 = tiles11.size() * sizeof(ScanTile);
    rc = scratch(ctx, "batch.desc", qbytes + gbytes + t6 + t1 + t11 + 256, &desc);
    if (rc) return rc;
    uint8_t* base = static_cast<uint8_t*>(desc);
    unsigned* queue = reinterpret_cast<unsigned*>(base);   // [0] Q6 passes, [1] two-Q1 passes, [2] one-Q1 passes
    ScanGroup* dgrp = reinterpret_cast<ScanGroup*>(base + qbytes);
    ScanTile* dt6 = reinterpret_cast<ScanTile*>(base + qbytes + gbytes);
    ScanTile* dt1 = reinterpret_cast<ScanTile*>(base + qbytes + gbytes + t6);
    ScanTile* dt11 = reinterpret_cast<ScanTile*>(base + qbytes + gbytes + t6 + t1);
    // pageable sources: the copies stage the descriptors before returning
    GPUDB_CUDA(ctx, cudaMemsetAsync(queue, 0, 12, call.stream()));
    GPUDB_CUDA(ctx, cudaMemcpyAsync(dgrp, groups.data(), groups.size() * sizeof(ScanGroup), cudaMemcpyHostToDevice,
                                    call.stream()));
    unsigned long long* res = reinterpret_cast<unsigned long long*>(dres + status_bytes);
    uint32_t* st = reinterpret_cast<uint32_t*>(dres);
    rc = launch_pass<0, kMaxQ6>(ctx, call, dgrp, tiles6, dt6, queue, res, st);
    if (!rc) rc = launch_pass<kMaxQ1, kMaxQ6WithQ1>(ctx, call, dgrp, tiles1, dt1, queue + 1, res, st);
    if (!rc) rc = launch_pass<1, kMaxQ6WithQ1>(ctx, call, dgrp, tiles11, dt11, queue + 2, res, st);
    if (rc) return rc;
  }
  for (const Riding& rd : riding) {
    std::vector<gpudb_q6_params> p6;
    std::vector<void*> o6;
    for (uint32_t j : rd.q6) {
      p6.push_back(reqs[ids[j]].q6);
      o6.push_back(dres + status_bytes + (size_t)offs[j] * 8);
    }
    rc = launch_q1_riders(call, rd.view, reqs[ids[rd.q1]].q1, dres + status_bytes + (size_t)offs[rd.q1] * 8,
                          reinterpret_cast<uint32_t*>(dres) + rd.q1, (int)p6.size(), p6.data(), o6.data());
    if (rc) return rc;
  }
  for (const auto& sq : solo_scans) {
    const uint32_t k = sq.first;
    const gpudb_request& q = reqs[ids[k]];
    uint8_t* w = dres + status_bytes + (size_t)offs[k] * 8;   // the kernel adds into these zeroed words
    rc = q.pipeline == GPUDB_PIPE_Q6 ? launch_q6(call, sq.second, q.q6, w)
                                     : launch_q1(call, sq.second, q.q1, w, reinterpret_cast<uint32_t*>(dres) + k);
    if (rc) return rc;
  }
  std::vector<uint32_t> ids_copy = ids;
  return call.finish(bytes, [reqs, ids_copy, offs, status_bytes, ctx, solo](const uint8_t* h) {
    for (size_t k = 0; k < ids_copy.size(); k++) {
      gpudb_request& q = reqs[ids_copy[k]];
      uint32_t st;
      std::memcpy(&st, h + 4 * k, 4);
      q.status = status_to_error(ctx, st);
      const uint8_t* w = h + status_bytes + (size_t)offs[k] * 8;
      if (q.pipeline == GPUDB_PIPE_Q6) {
        if (q.q6_out) { std::memcpy(&q.q6_out->revenue, w, 8); std::memcpy(&q.q6_out->rows_matched, w + 8, 8); }
      } else if (q.q1_out) {
        if (solo[k]) q1_result_from(w, q.q1_out);   // the Q1 kernel's words (a Q6 kernel's match a pass's)
        else q1_from_words(w, *q.q1_out);           // a shared pass's raw sums
      }
      if (ctx->on_done) ctx->on_done(ctx->on_done_arg, &q.status);
    }
    return GPUDB_OK;
  });
}


// ---- scans of host-resident tables ----------------------------------------------------
// Q6/Q1 requests over one host-resident table (same host columns and row range) share its
// chunked copy into HBM: the table streams once with the union of the columns the group
// reads (26 B/row when a Q1 request is in it, 20 B/row for Q6 alone), and every request's
// kernel runs on each chunk while it is resident (chunkedStreamLoop, src/infra.h:817-869,
// copies a table once per query). A request's result is the single-request pipeline's:
// the same kernels add into its own zeroed words chunk by chunk.
constexpr uint32_t kMaxHostGroup = 64;   // requests per shared copy (result words in one big slot)

bool host_scan_ok(const gpudb_request& r) {
  const gpudb_lineitem* li = r.li;
  if (!li || li->location != GPUDB_MEM_HOST) return false;
  if (r.pipeline == GPUDB_PIPE_Q6) return li->ship_date && li->discount && li->quantity && li->ext_price;
  return li->ship_date && li->quantity && li->ext_price && li->discount && li->tax && li->flag && li->status;
}

struct HostGroup {
  gpudb_lineitem view;          // the row range as its own table; Q1 columns from the first Q1 member
  bool has_q1 = false;
  std::vector<uint32_t> members;
};

// Rows [begin, end) of `li` as a table of their own.
gpudb_lineitem row_view(const gpudb_lineitem& li, uint64_t begin, uint64_t end) {
  gpudb_lineitem v = li;
  v.n_rows = end - begin;
  auto adv = [begin](const void* p, size_t w) { return p ? (const void*)((const uint8_t*)p + begin * w) : nullptr; };
  v.ship_date = (const int32_t*)adv(li.ship_date, 4);
  v.quantity = (const int32_t*)adv(li.quantity, 4);
  v.ext_price = (const int64_t*)adv(li.ext_price, 8);
  v.discount = (const int32_t*)adv(li.discount, 4);
  v.tax = (const int32_t*)adv(li.tax, 4);
  v.flag = (const uint8_t*)adv(li.flag, 1);
  v.status = (const uint8_t*)adv(li.status, 1);
  return v;
}

int run_host_group(gpudb_ctx* ctx, gpudb_request* reqs, const HostGroup& g, gpudb_timing* t, const gpudb_exec* ex) {
  const uint32_t m = (uint32_t)g.members.size();
  const size_t status_bytes = ((m * 4 + 15) / 16) * 16;
  std::vector<size_t> offs(m);
  size_t bytes = status_bytes;
  for (uint32_t k = 0; k < m; k++) {
    offs[k] = bytes;
    bytes += reqs[g.members[k]].pipeline == GPUDB_PIPE_Q6 ? kQ6ResultBytes : kQ1ResultBytes;
  }
  const uint32_t mask = LI_SHIP | LI_DISC | LI_QTY | LI_EXT | (g.has_q1 ? (LI_TAX | LI_FLAG | LI_STATUS) : 0u);
  int rc = lineitem_check(ctx, &g.view, mask);
  if (rc) return rc;
  Call call(ctx, ex, t);
  if ((rc = call.begin(bytes))) return rc;
  uint8_t* dres = call.result<uint8_t>();
  rc = stream_lineitem(call, &g.view, mask, 0, [&](const gpudb_lineitem& c) {
    for (uint32_t k = 0; k < m; k++) {
      const gpudb_request& q = reqs[g.members[k]];
      const int r = q.pipeline == GPUDB_PIPE_Q6
                        ? launch_q6(call, c, q.q6, dres + offs[k])
                        : launch_q1(call, c, q.q1, dres + offs[k], reinterpret_cast<uint32_t*>(dres) + k);
      if (r) return r;
    }
    return (int)GPUDB_OK;
  });
  if (rc) return rc;
  const std::vector<uint32_t> members = g.members;
  return call.finish(bytes, [reqs, members, offs, ctx](const uint8_t* h) {
    for (size_t k = 0; k < members.size(); k++) {
      gpudb_request& q = reqs[members[k]];
      uint32_t st;
      std::memcpy(&st, h + 4 * k, 4);
      q.status = status_to_error(ctx, st);
      const uint8_t* w = h + offs[k];
      if (q.pipeline == GPUDB_PIPE_Q6) {
        std::memcpy(&q.q6_out->revenue, w, 8);
        std::memcpy(&q.q6_out->rows_matched, w + 8, 8);
      } else {
        q1_result_from(w, q.q1_out);
      }
      if (ctx->on_done) ctx->on_done(ctx->on_done_arg, &q.status);
    }
    return GPUDB_OK;
  });
}

// Groups the host-table scan requests `ids` by table and row range and runs each group as
// one streamed pass.
void run_host_scans(gpudb_ctx* ctx, gpudb_request* reqs, const std::vector<uint32_t>& ids, gpudb_timing* t,
                    const gpudb_exec* ex) {
  std::vector<HostGroup> groups;
  for (uint32_t i : ids) {
    const gpudb_request& q = reqs[i];
    const gpudb_lineitem& li = *q.li;
    const uint64_t end = q.row_end ? std::min<uint64_t>(q.row_end, li.n_rows) : li.n_rows;
    const uint64_t begin = std::min<uint64_t>(q.row_begin, end);
    const gpudb_lineitem v = row_view(li, begin, end);
    const bool q1 = q.pipeline == GPUDB_PIPE_Q1;
    HostGroup* hit = nullptr;
    for (HostGroup& g : groups) {
      const gpudb_lineitem& w = g.view;
      if (g.members.size() >= kMaxHostGroup || w.n_rows != v.n_rows || w.ship_date != v.ship_date ||
          w.quantity != v.quantity || w.discount != v.discount || w.ext_price != v.ext_price)
        continue;
      if (q1 && g.has_q1 && (w.tax != v.tax || w.flag != v.flag || w.status != v.status)) continue;
      hit = &g;
      break;
    }
    if (!hit) {
      groups.emplace_back();
      hit = &groups.back();
      hit->view = v;
    }
    if (q1 && !hit->has_q1) {
      hit->has_q1 = true;
      hit->view.tax = v.tax;
      hit->view.flag = v.flag;
      hit->view.status = v.status;
    }
    hit->members.push_back(i);
  }
  for (const HostGroup& g : groups) {
    const int rc = run_host_group(ctx, reqs, g, t, ex);
    if (rc)
      for (uint32_t i : g.members) reqs[i].status = rc;
  }
}


}  // namespace
}  // namespace gpudb

using namespace gpudb;

namespace {

bool same_q3(const gpudb_request& a, const gpudb_request& b) {
  return a.q3 && b.q3 && std::memcmp(a.q3, b.q3, sizeof *a.q3) == 0 &&
         std::memcmp(&a.q3p, &b.q3p, sizeof a.q3p) == 0;
}
bool same_q9(const gpudb_request& a, const gpudb_request& b) {
  return a.q9 && b.q9 && std::memcmp(a.q9, b.q9, sizeof *a.q9) == 0 &&
         std::memcmp(&a.q9p, &b.q9p, sizeof a.q9p) == 0 && a.q9_capacity == b.q9_capacity;
}

// Completion hook of a synchronous batch: copies a coalesced request's result to its
// duplicates, then passes every completion on to the previous hook.
struct BatchHook {
  void (*prev)(void*, int32_t*);
  void* prev_arg;
  gpudb_request* reqs;
  uint32_t n;
  std::vector<std::vector<uint32_t>> dups;   // per request: identical later requests

  static void on_done(void* arg, int32_t* sink) {
    BatchHook* h = static_cast<BatchHook*>(arg);
    const uintptr_t base = reinterpret_cast<uintptr_t>(&h->reqs[0].status), at = reinterpret_cast<uintptr_t>(sink);
    if (at >= base && (at - base) % sizeof(gpudb_request) == 0 && (at - base) / sizeof(gpudb_request) < h->n) {
      const uint32_t i = (uint32_t)((at - base) / sizeof(gpudb_request));
      const gpudb_request& o = h->reqs[i];
      if (h->prev) h->prev(h->prev_arg, sink);
      for (uint32_t d : h->dups[i]) {
        gpudb_request& q = h->reqs[d];
        q.status = o.status;
        if (q.pipeline == GPUDB_PIPE_Q3) {
          *q.q3_out = *o.q3_out;
        } else {
          q.q9_groups = o.q9_groups;
          if (q.q9_capacity) std::memcpy(q.q9_out, o.q9_out, (size_t)std::min(o.q9_groups, q.q9_capacity) * sizeof(gpudb_q9_group));
        }
        if (h->prev) h->prev(h->prev_arg, &q.status);
      }
      return;
    }
    if (h->prev) h->prev(h->prev_arg, sink);
  }
};

}  // namespace

extern "C" int gpudb_batch_run(gpudb_ctx* ctx, gpudb_request* reqs, uint32_t n, gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (n && !reqs) return fail(ctx, GPUDB_E_INVALID, "batch: requests are NULL");
  const bool async = ex && ex->async;
  gpudb_exec aex{1, 0, ex ? ex->stream : nullptr};
  // synchronous batches coalesce identical join requests: the first runs, the others copy
  BatchHook hook{ctx->on_done, ctx->on_done_arg, reqs, n, {}};
  std::vector<char> skip(n, 0);
  if (!async) {
    hook.dups.resize(n);
    for (uint32_t i = 0; i < n; i++) {
      const gpudb_request& q = reqs[i];
      if (q.pipeline != GPUDB_PIPE_Q3 && q.pipeline != GPUDB_PIPE_Q9) continue;
      if (q.pipeline == GPUDB_PIPE_Q3 ? !q.q3_out : (!q.q9_out && q.q9_capacity)) continue;
      for (uint32_t j = 0; j < i; j++) {
        if (skip[j] || reqs[j].pipeline != q.pipeline) continue;
        if (q.pipeline == GPUDB_PIPE_Q3 ? (reqs[j].q3_out && same_q3(reqs[j], q)) : same_q9(reqs[j], q)) {
          hook.dups[j].push_back(i);
          skip[i] = 1;
          break;
        }
      }
    }
    ctx->on_done = &BatchHook::on_done;
    ctx->on_done_arg = &hook;
  }
  // synchronous batches time the whole batch: events around everything it enqueues
  cudaStream_t bs = (ex && ex->stream) ? static_cast<cudaStream_t>(ex->stream) : ctx->stream;
  cudaEvent_t te0 = nullptr, te1 = nullptr;
  const uint64_t launches0 = ctx->launches;
  const double host0 = now_ms();
  if (t && !async) {
    te0 = event_get(ctx);
    te1 = event_get(ctx);
    if (te0) cudaEventRecord(te0, bs);
  }
  // Scans of small tables (at most kSmallScanRows rows) and of large ones are run apart, so
  // that each group's requests complete when its own work ends.
  constexpr uint64_t kSmallScanRows = 1ull << 24;
  std::vector<uint32_t> scan_lists[2], host_scans;   // [0] small tables, [1] large
  size_t scan_bytes[2] = {0, 0};
  const uint64_t h2d0 = ctx->h2d_total, d2h0 = ctx->d2h_total;
  auto flush_scans = [&](int which) -> int {
    std::vector<uint32_t>& scans = scan_lists[which];
    if (scans.empty()) return GPUDB_OK;
    int rc = run_scan_batch(ctx, reqs, scans, async ? t : nullptr, &aex);
    if (rc) for (uint32_t i : scans) reqs[i].status = rc;
    scans.clear();
    scan_bytes[which] = 0;
    return GPUDB_OK;
  };
  // Order on the stream, by work per request (cheapest first, so that the requests of a
  // group complete early and the ones waiting for the batch's end are few): scans of small
  // tables, the joins that run alone (identical Q9 requests run once per batch), the batched
  // Q3 groups, the scans of large tables, then scans of host-resident tables.
  std::map<std::string, std::vector<uint32_t>> q3_groups;   // batchable Q3 by identical tables
  std::vector<uint32_t> joins;
  for (uint32_t i = 0; i < n; i++) {
    gpudb_request& q = reqs[i];
    q.status = GPUDB_OK;
    if (skip[i]) continue;
    if (q.pipeline == GPUDB_PIPE_Q3 || q.pipeline == GPUDB_PIPE_Q9) {
      if (n > 1 && q3_batchable(q))
        q3_groups[std::string(reinterpret_cast<const char*>(q.q3), sizeof *q.q3)].push_back(i);
      else
        joins.push_back(i);
      continue;
    }
    int rc = GPUDB_OK;
    switch (q.pipeline) {
      case GPUDB_PIPE_Q6:
      case GPUDB_PIPE_Q1: {
        if ((q.pipeline == GPUDB_PIPE_Q6 && !q.q6_out) || (q.pipeline == GPUDB_PIPE_Q1 && !q.q1_out)) {
          rc = fail(ctx, GPUDB_E_INVALID, "batch: request %u has no result struct", i);
          break;
        }
        // a lone scan runs through its own pipeline (the plain form); several share passes
        if (n > 1 && scan_columns_ok(q)) {
          const size_t b = (q.pipeline == GPUDB_PIPE_Q6 ? kQ6Words : kQ1Words) * 8 + 4;
          const uint64_t end = q.row_end ? std::min<uint64_t>(q.row_end, q.li->n_rows) : q.li->n_rows;
          const int which = end - std::min<uint64_t>(q.row_begin, end) > kSmallScanRows ? 1 : 0;
          if (scan_bytes[which] + b + 64 > kBigSlotBytes - kSlotHeader) flush_scans(which);
          scan_lists[which].push_back(i);
          scan_bytes[which] += b;
          break;
        }
        if (n > 1 && host_scan_ok(q)) {   // shares the table's copy into HBM with the others
          host_scans.push_back(i);
          break;
        }
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
      default:
        rc = fail(ctx, GPUDB_E_INVALID, "batch: request %u has unknown pipeline %d", i, q.pipeline);
    }
    if (rc != GPUDB_OK) q.status = rc;
  }
  flush_scans(0);
  auto set_failed = [&](uint32_t i, int rc) {
    reqs[i].status = rc;
    if (!async)
      for (uint32_t d : hook.dups[i]) reqs[d].status = rc;
  };
  std::vector<std::vector<uint32_t>> q3_parts;   // groups of 2..kQ3Batch; a group of one runs alone
  for (auto& kv : q3_groups) {
    std::vector<uint32_t>& l = kv.second;
    for (size_t a = 0; a < l.size(); a += kQ3Batch) {
      const size_t b = std::min(l.size(), a + (size_t)kQ3Batch);
      if (b - a == 1) joins.push_back(l[a]);
      else q3_parts.emplace_back(l.begin() + a, l.begin() + b);
    }
  }
  std::sort(joins.begin(), joins.end());
  for (uint32_t i : joins) {
    gpudb_request& q = reqs[i];
    int rc = GPUDB_OK;
    switch (q.pipeline) {
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
        break;
    }
    if (rc != GPUDB_OK) set_failed(i, rc);
  }
  for (const std::vector<uint32_t>& part : q3_parts) {
    const int rc = q3_batch_run(ctx, reqs, part, &aex);
    if (rc != GPUDB_OK)
      for (uint32_t i : part) set_failed(i, rc);
  }
  flush_scans(1);
  if (!host_scans.empty()) run_host_scans(ctx, reqs, host_scans, async ? t : nullptr, &aex);
  if (async) return GPUDB_OK;
  if (te1) cudaEventRecord(te1, bs);
  gpudb_sync(ctx);   // per-request outcomes are in each status
  ctx->on_done = hook.prev;
  ctx->on_done_arg = hook.prev_arg;
  if (t && te0 && te1) {
    float ms = -1.f;
    if (cudaEventSynchronize(te1) != cudaSuccess || cudaEventElapsedTime(&ms, te0, te1) != cudaSuccess) ms = -1.f;
    t->gpu_ms = ms;
    t->host_ms = now_ms() - host0;
    t->kernels = (uint32_t)(ctx->launches - launches0);
    t->h2d_bytes = ctx->h2d_total - h2d0;
    t->d2h_bytes = ctx->d2h_total - d2h0;
    t->chunks = 0;
  }
  event_put(ctx, te0);
  event_put(ctx, te1);
  return GPUDB_OK;
}
