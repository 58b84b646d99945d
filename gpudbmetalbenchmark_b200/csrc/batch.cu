// Batched execution: many requests per call (gpudb_batch_run).
//
// All Q6/Q1 requests over device-resident tables become tiles of at most kTileRows rows
// (request, row range) in one work list; a persistent grid pulls tiles from a device queue
// (one atomicAdd per tile), so a batch of small requests, or of uneven row ranges over
// different tables, is a single launch. A tile's block reduces its partial sums and adds
// them into the request's own result words with integer atomics (exact, order-independent).
// Q3/Q9 requests are enqueued behind it on the same stream as ordinary async pipeline calls,
// so the whole batch needs one host synchronisation.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace gpudb {
namespace {

constexpr int kBT = 256;
constexpr uint64_t kTileRows = 16384;     // per-tile block sums stay below 2^64 (Q1 domain)
constexpr int kQ6Words = 2;               // revenue, rows matched
constexpr int kQ1Words = 72;              // 6 groups x 6 raw metrics x u128

struct ScanReq {
  int32_t kind, a, b, c, d, e;            // Q6: ship_lo, ship_hi, disc_lo, disc_hi, qty_lt; Q1: ship_le
  const int32_t *ship, *qty, *disc, *tax;
  const int64_t* ext;
  const uint8_t *flag, *stat;
  uint32_t res;                           // first result word
  uint32_t idx;                           // index among the scan requests (status word)
};
struct ScanTile {
  uint32_t req, pad;
  uint64_t begin, end;
};

__device__ __forceinline__ void atomic_add_u128(unsigned long long* p, u128 v) {
  const unsigned long long lo = (unsigned long long)v;
  unsigned long long hi = (unsigned long long)(v >> 64);
  const unsigned long long old = atomicAdd(p, lo);
  if (old + lo < old) hi++;
  if (hi) atomicAdd(p + 1, hi);
}

__global__ void __launch_bounds__(kBT) scan_batch_kernel(const ScanReq* __restrict__ reqs,
                                                         const ScanTile* __restrict__ tiles, uint32_t n_tiles,
                                                         unsigned* queue, unsigned long long* res, uint32_t* req_status) {
  extern __shared__ unsigned long long acc[];   // [24][kBT] Q1 group accumulators
  __shared__ uint32_t tile_i;
  __shared__ unsigned long long red[kBT / 32][36];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (;;) {
    if (t == 0) tile_i = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t i = tile_i;
    __syncthreads();
    if (i >= n_tiles) break;
    const ScanTile T = tiles[i];
    const ScanReq R = reqs[T.req];
    if (R.kind == GPUDB_PIPE_Q6) {
      int64_t rev = 0;
      unsigned long long cnt = 0;
      for (uint64_t r = T.begin + t; r < T.end; r += kBT) {
        const int32_t s = R.ship[r], dd = R.disc[r], q = R.qty[r];
        if ((s >= R.a) & (s < R.b) & (dd >= R.c) & (dd <= R.d) & (q < R.e)) { rev += R.ext[r] * (int64_t)dd; cnt++; }
      }
      const unsigned long long a = warp_sum_u64((unsigned long long)rev), b = warp_sum_u64(cnt);
      if (lane == 0) { red[warp][0] = a; red[warp][1] = b; }
      __syncthreads();
      if (t < 2) {
        unsigned long long s = 0;
        for (int w = 0; w < kBT / 32; w++) s += red[w][t];
        if (s) atomicAdd(res + R.res + t, s);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 24; k++) acc[k * kBT + t] = 0;
      uint32_t bad = 0;
      for (uint64_t r = T.begin + t; r < T.end; r += kBT) {
        const uint32_t f = R.flag[r], st = R.stat[r];
        if (!((R.ship[r] <= R.a) & (f <= 2u) & (st <= 1u))) continue;
        const int32_t qt = R.qty[r], dd = R.disc[r], tx = R.tax[r];
        const int64_t e = R.ext[r];
        bad |= ((uint32_t)qt >= 65536u) | ((uint32_t)dd > 100u) | ((uint32_t)tx > 100u) | ((uint64_t)e >= (1ull << 36));
        const uint64_t ed = (uint64_t)e * (uint32_t)dd;
        const uint64_t edt = ((uint64_t)e * 100u - ed) * (uint32_t)tx;
        unsigned long long* p = acc + (f * 2u + st) * kBT + t;
        p[0] += ((uint64_t)(uint32_t)qt << 32) | ((uint64_t)(uint32_t)dd << 13) | 1u;
        p[6 * kBT] += (uint64_t)e;
        p[12 * kBT] += ed;
        p[18 * kBT] += edt;
      }
      if (__syncthreads_or(bad) && t == 0) atomicOr(req_status + R.idx, ST_DOMAIN);
#pragma unroll
      for (int g = 0; g < 6; g++) {
        const unsigned long long P = acc[g * kBT + t];
        const unsigned long long v[6] = {P & 0x1FFFu, P >> 32, acc[(6 + g) * kBT + t], acc[(12 + g) * kBT + t],
                                         acc[(18 + g) * kBT + t], (P >> 13) & 0x7FFFFu};
#pragma unroll
        for (int m = 0; m < 6; m++) {
          const unsigned long long w = warp_sum_u64(v[m]);
          if (lane == 0) red[warp][g * 6 + m] = w;
        }
      }
      __syncthreads();
      if (t < 36) {
        u128 s = 0;
        for (int w = 0; w < kBT / 32; w++) s += red[w][t];
        if (s) atomic_add_u128(res + R.res + 2 * t, s);
      }
    }
    __syncthreads();
  }
}

unsigned scan_grid(gpudb_ctx* ctx, uint32_t tiles, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scan_batch_kernel, kBT, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return std::max<unsigned>(1, std::min<unsigned>(tiles, (unsigned)(ctx->sm_count * per_sm)));
}

bool scan_columns_ok(const gpudb_request& r) {
  const gpudb_lineitem* li = r.li;
  if (!li || li->location != GPUDB_MEM_DEVICE) return false;
  if (r.pipeline == GPUDB_PIPE_Q6) return li->ship_date && li->discount && li->quantity && li->ext_price;
  return li->ship_date && li->quantity && li->ext_price && li->discount && li->tax && li->flag && li->status;
}

// Runs one scan batch (fits one result slot): requests `ids` of `reqs`.
int run_scan_batch(gpudb_ctx* ctx, gpudb_request* reqs, const std::vector<uint32_t>& ids, gpudb_timing* t,
                   const gpudb_exec* ex) {
  std::vector<ScanReq> sr;
  std::vector<ScanTile> tiles;
  uint32_t words = 0;
  for (uint32_t k = 0; k < ids.size(); k++) {
    gpudb_request& q = reqs[ids[k]];
    const gpudb_lineitem* li = q.li;
    ScanReq d{};
    d.kind = q.pipeline;
    if (q.pipeline == GPUDB_PIPE_Q6) {
      d.a = q.q6.ship_lo; d.b = q.q6.ship_hi; d.c = q.q6.disc_lo; d.d = q.q6.disc_hi; d.e = q.q6.qty_lt;
    } else {
      d.a = q.q1.ship_le;
    }
    d.ship = li->ship_date; d.qty = li->quantity; d.disc = li->discount; d.tax = li->tax; d.ext = li->ext_price;
    d.flag = li->flag; d.stat = li->status;
    d.res = words;
    d.idx = k;
    words += q.pipeline == GPUDB_PIPE_Q6 ? kQ6Words : kQ1Words;
    const uint64_t end = q.row_end ? std::min<uint64_t>(q.row_end, li->n_rows) : li->n_rows;
    for (uint64_t b = q.row_begin; b < end; b += kTileRows)
      tiles.push_back(ScanTile{(uint32_t)sr.size(), 0, b, std::min(b + kTileRows, end)});
    sr.push_back(d);
  }
  const size_t status_bytes = ((ids.size() * 4 + 15) / 16) * 16;
  const size_t bytes = status_bytes + (size_t)words * 8;
  Call call(ctx, ex, t);
  int rc = call.begin(bytes);
  if (rc) return rc;
  uint8_t* dres = call.result<uint8_t>();
  if (!tiles.empty()) {
    void* desc = nullptr;
    const size_t qbytes = 256, rbytes = sr.size() * sizeof(ScanReq), tbytes = tiles.size() * sizeof(ScanTile);
    rc = scratch(ctx, "batch.desc", qbytes + rbytes + tbytes + 256, &desc);
    if (rc) return rc;
    uint8_t* base = static_cast<uint8_t*>(desc);
    unsigned* queue = reinterpret_cast<unsigned*>(base);
    ScanReq* dreq = reinterpret_cast<ScanReq*>(base + qbytes);
    ScanTile* dtile = reinterpret_cast<ScanTile*>(base + qbytes + ((rbytes + 15) / 16) * 16);
    // pageable sources: the copies stage the descriptors before returning
    GPUDB_CUDA(ctx, cudaMemsetAsync(queue, 0, 4, call.stream()));
    GPUDB_CUDA(ctx, cudaMemcpyAsync(dreq, sr.data(), rbytes, cudaMemcpyHostToDevice, call.stream()));
    GPUDB_CUDA(ctx, cudaMemcpyAsync(dtile, tiles.data(), tbytes, cudaMemcpyHostToDevice, call.stream()));
    const size_t smem = (size_t)24 * kBT * 8;
    GPUDB_CUDA(ctx, cudaFuncSetAttribute(scan_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned grid = scan_grid(ctx, (uint32_t)tiles.size(), smem);
    GPUDB_LAUNCH(call, scan_batch_kernel, grid, kBT, smem, (const ScanReq*)dreq, (const ScanTile*)dtile,
                 (uint32_t)tiles.size(), queue, reinterpret_cast<unsigned long long*>(dres + status_bytes),
                 reinterpret_cast<uint32_t*>(dres));
  }
  std::vector<uint32_t> ids_copy = ids;
  std::vector<uint32_t> offs;
  for (auto& d : sr) offs.push_back(d.res);
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
