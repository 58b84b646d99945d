// Batched Q3: up to kQ3Batch requests over the same customer/orders/lineitem tables, each
// with its own segment, order-date bound, ship-date bound and k, evaluated together. Every
// stage is one launch for all requests:
//  1. q3m_bitmap_kernel: one customer bitmap per distinct segment (blockIdx.y).
//  2. q3m_orders_kernel: one pass over orders; an order that qualifies for any request is
//     staged once as (key, date, request mask), and each request's count stays on the
//     device.
//  3. q3m_clear_kernel: each request's table (blockIdx.y) is sized from its count and
//     cleared.
//  4. q3m_insert_kernel: each staged order is inserted into the tables of its mask, and
//     the request's order-key bitmap is set.
//  5. q3m_probe_kernel: one pass over the fact table. Runs of equal order keys are found
//     once per warp; per request, the run head tests the request's order-key bitmap and
//     probes its table; each row passing that request's ship bound adds its revenue and a
//     count to the slot. ext_price/discount are loaded only for rows that joined some
//     request.
//  6. q3m_hist_kernel / q3m_select_kernel: per request (blockIdx.y), the two top-k passes of
//     the single Q3 (revenue histogram, then select and rank).
// Results are the same as running each request alone (integer sums, the same top-k order).
#include <algorithm>
#include <cstring>
#include <map>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"
#include "q3.h"

namespace gpudb {
namespace {

constexpr int kB = kQ3Batch;
constexpr int kOrdersRows = 4;                // rows per thread per block step of the orders pass
constexpr size_t kReqBytes = 16 + (size_t)GPUDB_Q3_MAX_K * sizeof(u128);   // per-request result payload

struct Q3Multi {
  int K, D;                                   // requests, distinct segments
  int32_t seg[kB];                            // distinct segment values
  int32_t req_seg[kB];                        // request -> index into seg
  int32_t date_lt[kB], ship_gt[kB], k[kB];
  uint32_t* bm;                               // D customer bitmaps of `words` words
  uint32_t words;
  uint32_t* okbm;                             // K order-key bitmaps of `okwords` words (null: none)
  uint32_t okwords;
  int32_t key_max;                            // orders key bound for okbm
  Q3Slot* ht;                                 // K tables of max_cap slots
  uint32_t* hits;
  uint32_t max_cap;
  int shift;                                  // table load <= 1/2^shift
  uint32_t* cnt;                              // per request: count, capacity, okbm off, ticket
  int32_t* skey;                              // staged orders
  int32_t* sdate;
  uint32_t* smask;
  uint32_t* n_stage;
  u128* cand;                                 // per request: kTopkCandCap top-k candidates
  uint32_t* tstate;                           // per request: kTopkStateWords (histogram, count, ticket)
  uint32_t* status;                           // per request status words
  uint32_t* dstatus;                          // per distinct segment status words
  uint8_t* res;                               // per request kReqBytes
};

__global__ void q3m_bitmap_kernel(const int32_t* __restrict__ keys, const uint8_t* __restrict__ seg, uint64_t n,
                                  int32_t key_max, Q3Multi m) {
  const int d = blockIdx.y;
  bitmap_build_rows(keys, seg, m.seg[d], n, key_max, m.bm + (size_t)d * m.words, m.dstatus + d,
                    (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, (uint64_t)gridDim.x * blockDim.x);
}

__global__ void __launch_bounds__(256) q3m_orders_kernel(const int32_t* __restrict__ okey, const int32_t* __restrict__ ocust,
                                                         const int32_t* __restrict__ odate, uint64_t n, int32_t cust_max,
                                                         Q3Multi m) {
  __shared__ uint32_t sh[33];
  __shared__ uint32_t scount[kB];
  if (threadIdx.x < kB) scount[threadIdx.x] = 0;
  __syncthreads();
  uint32_t mycnt[kB];
#pragma unroll
  for (int r = 0; r < kB; r++) mycnt[r] = 0;
  const uint64_t step = (uint64_t)gridDim.x * 256 * kOrdersRows;
  for (uint64_t b = (uint64_t)blockIdx.x * 256 * kOrdersRows; b < n; b += step) {   // whole blocks
    int32_t key[kOrdersRows], date[kOrdersRows];
    uint32_t mask[kOrdersRows];
    uint32_t take = 0;
#pragma unroll
    for (int j = 0; j < kOrdersRows; j++) {
      const uint64_t i = b + (uint64_t)j * 256 + threadIdx.x;
      mask[j] = 0;
      key[j] = 0;
      date[j] = 0;
      if (i < n) {
        date[j] = ld_stream(odate + i);
        const int32_t c = ld_stream(ocust + i);
        key[j] = ld_stream(okey + i);   // with the other columns: no dependent load later
        uint32_t segs = 0;   // distinct segments whose bitmap holds the customer
        if (c >= 0 && c <= cust_max)
          for (int d = 0; d < m.D; d++) segs |= (uint32_t)bitmap_test(m.bm + (size_t)d * m.words, c) << d;
        for (int r = 0; r < m.K; r++)
          mask[j] |= (uint32_t)((date[j] < m.date_lt[r]) & ((segs >> m.req_seg[r]) & 1u)) << r;
        if (mask[j]) {
          if (key[j] == kEmptyKey) {
            for (int r = 0; r < m.K; r++)
              if (mask[j] & (1u << r)) set_status(m.status + r, ST_KEY_RANGE);
            mask[j] = 0;
          } else {
            take |= 1u << j;
#pragma unroll
            for (int r = 0; r < kB; r++) mycnt[r] += (mask[j] >> r) & 1u;
          }
        }
      }
    }
    uint32_t pos = block_reserve<256>(__popc(take), m.n_stage, sh);
#pragma unroll
    for (int j = 0; j < kOrdersRows; j++)
      if (take & (1u << j)) { m.skey[pos] = key[j]; m.sdate[pos] = date[j]; m.smask[pos] = mask[j]; pos++; }
  }
#pragma unroll
  for (int r = 0; r < kB; r++) {
    const uint32_t c = __reduce_add_sync(FULL_MASK, mycnt[r]);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&scount[r], c);
  }
  __syncthreads();
  if (threadIdx.x < (unsigned)m.K && scount[threadIdx.x]) atomicAdd(m.cnt + 4 * threadIdx.x, scount[threadIdx.x]);
}

__global__ void q3m_clear_kernel(Q3Multi m) {
  const int r = blockIdx.y;
  const uint32_t cap = table_capacity(m.cnt[4 * r], 2048, m.max_cap, m.shift);
  if (blockIdx.x == 0 && threadIdx.x == 0) m.cnt[4 * r + 1] = cap;
  Q3Slot* ht = m.ht + (size_t)r * m.max_cap;
  uint32_t* hits = m.hits + (size_t)r * m.max_cap;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
    ht[i].key = kEmptyKey;
    ht[i].date = 0;
    ht[i].rev = 0;
    hits[i] = 0;
  }
}

__global__ void q3m_insert_kernel(Q3Multi m) {
  const uint32_t n = *m.n_stage;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int32_t k = m.skey[i], date = m.sdate[i];
    uint32_t mask = m.smask[i];
    while (mask) {
      const int r = __ffs(mask) - 1;
      mask &= mask - 1;
      uint32_t* c = m.cnt + 4 * r;
      if (m.okbm) {
        if (k >= 0 && k <= m.key_max) atomicOr(m.okbm + (size_t)r * m.okwords + ((uint32_t)k >> 5), 1u << ((uint32_t)k & 31u));
        else c[2] = 1u;
      }
      const uint32_t cap = c[1], cmask = cap - 1;
      Q3Slot* ht = m.ht + (size_t)r * m.max_cap;
      uint32_t s = key_slot(k, cmask);
      bool done = false;
      for (uint32_t p = 0; p < cap && !done; p++, s = (s + 1) & cmask) {
        const int32_t prev = atomicCAS(&ht[s].key, kEmptyKey, k);
        if (prev == kEmptyKey) { ht[s].date = date; done = true; }
        else if (prev == k) { set_status(m.status + r, ST_DUPLICATE); done = true; }
      }
      if (!done) set_status(m.status + r, ST_CAPACITY);
    }
  }
}

__global__ void __launch_bounds__(256) q3m_probe_kernel(const int32_t* __restrict__ lkey, const int32_t* __restrict__ lship,
                                                        const int64_t* __restrict__ lext, const int32_t* __restrict__ ldisc,
                                                        uint64_t n, Q3Multi m) {
  __shared__ uint32_t scap[kB];
  __shared__ const uint32_t* sbm[kB];
  if (threadIdx.x < (unsigned)m.K) {
    const int r = threadIdx.x;
    scap[r] = m.cnt[4 * r + 1];
    sbm[r] = (m.okbm && m.cnt[4 * r + 2] == 0u) ? m.okbm + (size_t)r * m.okwords : nullptr;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t step = (uint64_t)gridDim.x * (blockDim.x >> 5) * 32;
  uint64_t base = ((uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32;
  // the next step's key and ship date are loaded while this step is processed
  int32_t nkey = base + lane < n ? ld_stream(lkey + base + lane) : kEmptyKey;
  int32_t nship = base + lane < n ? ld_stream(lship + base + lane) : INT32_MIN;
  for (; base < n; base += step) {
    const uint64_t row = base + lane;
    const bool valid = row < n;
    const int32_t key = nkey, ship = nship;
    nkey = row + step < n ? ld_stream(lkey + row + step) : kEmptyKey;
    nship = row + step < n ? ld_stream(lship + row + step) : INT32_MIN;
    const int32_t prev = __shfl_up_sync(FULL_MASK, key, 1);
    const bool head = (lane == 0) || (key != prev);
    const uint32_t heads = __ballot_sync(FULL_MASK, head);
    const int my_head = 31 - __clz(heads & lanemask_le());
    const uint32_t later = heads & lanemask_gt();
    const uint32_t upto = later ? (1u << (__ffs(later) - 1)) - 1u : 0xFFFFFFFFu;
    const uint32_t run_mask = upto & ~((1u << lane) - 1u);   // used by head lanes only
    int32_t slot[kB];
    uint32_t hitbits = 0;   // requests this row joins
#pragma unroll
    for (int r = 0; r < kB; r++) {
      slot[r] = -1;
      if (r >= m.K) continue;
      const bool pass = valid && ship > m.ship_gt[r];
      const uint32_t passm = __ballot_sync(FULL_MASK, pass);
      int32_t s = -1;
      if (head && (passm & run_mask) && key != kEmptyKey) {
        const uint32_t* bm = sbm[r];
        if (!bm || (key >= 0 && key <= m.key_max && bitmap_test(bm, key)))
          s = ht_find(m.ht + (size_t)r * m.max_cap, scap[r], key);
      }
      slot[r] = __shfl_sync(FULL_MASK, s, my_head);
      hitbits |= (uint32_t)(pass && slot[r] >= 0) << r;
    }
    // rows that join add their revenue and count per request (integer sums: order-free)
    if (hitbits) {
      const int64_t v = ld_stream(lext + row) * (int64_t)(100 - ld_stream(ldisc + row));
#pragma unroll
      for (int r = 0; r < kB; r++) {
        if ((hitbits >> r) & 1u) {
          const size_t at = (size_t)r * m.max_cap + (uint32_t)slot[r];
          atomicAdd(&m.ht[at].rev, (unsigned long long)v);
          atomicAdd(&m.hits[at], 1u);
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kTopkThreads) q3m_hist_kernel(Q3Multi m) {
  __shared__ uint32_t sh[kRevBins];
  const int r = blockIdx.y;
  q3_table_hist(m.ht + (size_t)r * m.max_cap, m.hits + (size_t)r * m.max_cap, m.cnt[4 * r + 1],
                m.tstate + (size_t)r * kTopkStateWords, reinterpret_cast<unsigned long long*>(m.res + (size_t)r * kReqBytes),
                sh);
}

__global__ void __launch_bounds__(kTopkThreads) q3m_select_kernel(Q3Multi m) {
  __shared__ u128 sm[kTopkScratch];
  __shared__ u128 carry[GPUDB_Q3_MAX_K];
  const int r = blockIdx.y;
  q3_table_select(m.ht + (size_t)r * m.max_cap, m.hits + (size_t)r * m.max_cap, m.cnt[4 * r + 1], m.k[r],
                  m.tstate + (size_t)r * kTopkStateWords, m.cand + (size_t)r * kTopkCandCap,
                  reinterpret_cast<u128*>(m.res + (size_t)r * kReqBytes + 16), sm, carry);
}

}  // namespace

bool q3_batchable(const gpudb_request& q) {
  if (q.pipeline != GPUDB_PIPE_Q3 || !q.q3 || !q.q3_out) return false;
  const gpudb_q3_params& p = q.q3p;
  const gpudb_q3_tables& t = *q.q3;
  if (p.join_mode != GPUDB_JOIN_GLOBAL || p.k < 1 || p.k > GPUDB_Q3_MAX_K || p.segment < 0 || p.segment > 255) return false;
  if (t.li.location != GPUDB_MEM_DEVICE || !t.li.order_key || !t.li.ship_date || !t.li.ext_price || !t.li.discount)
    return false;
  if (!t.cu.n_rows || !t.cu.cust_key || !t.cu.segment || t.cu.key_max < 0) return false;
  if (!t.od.n_rows || !t.od.order_key || !t.od.cust_key || !t.od.order_date || t.od.n_rows > (1ull << 30)) return false;
  return true;
}

int q3_batch_run(gpudb_ctx* ctx, gpudb_request* reqs, const std::vector<uint32_t>& ids, const gpudb_exec* ex) {
  const int K = (int)ids.size();
  if (K < 1 || K > kB) return fail(ctx, GPUDB_E_INVALID, "q3 batch: 1..%d requests", kB);
  const gpudb_q3_tables& T = *reqs[ids[0]].q3;
  const gpudb_customer& cu = T.cu;
  const gpudb_orders& od = T.od;
  const gpudb_lineitem& li = T.li;
  Q3Multi m{};
  m.K = K;
  std::vector<int32_t> segs;
  for (int r = 0; r < K; r++) {
    const gpudb_q3_params& p = reqs[ids[r]].q3p;
    auto it = std::find(segs.begin(), segs.end(), p.segment);
    m.req_seg[r] = (int32_t)(it - segs.begin());
    if (it == segs.end()) segs.push_back(p.segment);
    m.date_lt[r] = p.order_date_lt;
    m.ship_gt[r] = p.ship_date_gt;
    m.k[r] = p.k;
  }
  m.D = (int)segs.size();
  for (int d = 0; d < m.D; d++) m.seg[d] = segs[d];
  const uint64_t n_or = od.n_rows;
  uint32_t max_cap = 2048;
  while (max_cap < (n_or << ctx->ht_shift) && max_cap < (1u << 31)) max_cap <<= 1;
  m.max_cap = max_cap;
  m.shift = ctx->ht_shift;
  m.words = (uint32_t)((uint32_t)cu.key_max >> 5) + 1;
  const bool use_okbm = od.key_max >= 0;
  m.okwords = use_okbm ? (uint32_t)((uint32_t)od.key_max >> 5) + 1 : 0;
  m.key_max = od.key_max;

  // result slot: K status words, D segment status words, K payloads
  const size_t st_bytes = 64, bytes = st_bytes + (size_t)K * kReqBytes;
  Call call(ctx, ex, nullptr);
  int rc = call.begin(bytes);
  if (rc) return rc;
  cudaStream_t s = call.stream();
  uint8_t* res = call.result<uint8_t>();
  m.status = reinterpret_cast<uint32_t*>(res);
  m.dstatus = m.status + kB;
  m.res = res + st_bytes;
  void *bm, *okbm = nullptr, *stage, *cnt, *ht, *hits, *cand;
  rc = scratch(ctx, "q3m.bitmaps", (size_t)m.D * m.words * 4, &bm);
  if (!rc && use_okbm) rc = scratch(ctx, "q3m.okbm", (size_t)K * m.okwords * 4, &okbm);
  if (!rc) rc = scratch(ctx, "q3m.stage", n_or * 12 + 256, &stage);
  if (!rc) rc = scratch(ctx, "q3m.count", 256, &cnt);
  if (!rc) rc = scratch(ctx, "q3m.ht", (size_t)K * max_cap * sizeof(Q3Slot), &ht);
  if (!rc) rc = scratch(ctx, "q3m.hits", (size_t)K * max_cap * 4, &hits);
  void* tstate = nullptr;
  if (!rc) rc = scratch(ctx, "q3m.topk", (size_t)K * kTopkStateWords * 4, &tstate);
  if (!rc) rc = scratch(ctx, "q3m.cand", (size_t)K * kTopkCandCap * sizeof(u128), &cand);
  if (rc) return rc;
  m.bm = static_cast<uint32_t*>(bm);
  m.okbm = static_cast<uint32_t*>(okbm);
  m.skey = static_cast<int32_t*>(stage);
  m.sdate = m.skey + n_or;
  m.smask = reinterpret_cast<uint32_t*>(m.sdate + n_or);
  m.cnt = static_cast<uint32_t*>(cnt);
  m.n_stage = m.cnt + 4 * kB;
  m.ht = static_cast<Q3Slot*>(ht);
  m.hits = static_cast<uint32_t*>(hits);
  m.cand = static_cast<u128*>(cand);
  m.tstate = static_cast<uint32_t*>(tstate);
  GPUDB_CUDA(ctx, cudaMemsetAsync(bm, 0, (size_t)m.D * m.words * 4, s));
  if (use_okbm) GPUDB_CUDA(ctx, cudaMemsetAsync(okbm, 0, (size_t)K * m.okwords * 4, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(cnt, 0, (4 * kB + 1) * 4, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(tstate, 0, (size_t)K * kTopkStateWords * 4, s));
  const int sms = ctx->sm_count;
  auto grid = [&](uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 16)); };
  GPUDB_LAUNCH(call, q3m_bitmap_kernel, dim3(grid(cu.n_rows), m.D), 256, 0, cu.cust_key, cu.segment, cu.n_rows, cu.key_max, m);
  GPUDB_LAUNCH(call, q3m_orders_kernel, grid((n_or + kOrdersRows - 1) / kOrdersRows), 256, 0, od.order_key, od.cust_key,
               od.order_date, n_or, cu.key_max, m);
  GPUDB_LAUNCH(call, q3m_clear_kernel, dim3(std::max(1u, grid(max_cap) / 4), K), 256, 0, m);
  GPUDB_LAUNCH(call, q3m_insert_kernel, grid(n_or / 4), 256, 0, m);
  const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((li.n_rows + 255) / 256, (uint64_t)sms * 8));
  if (li.n_rows)
    GPUDB_LAUNCH(call, q3m_probe_kernel, g, 256, 0, li.order_key, li.ship_date, li.ext_price, li.discount, li.n_rows, m);
  GPUDB_LAUNCH(call, q3m_hist_kernel, dim3(q3_topk_grid(max_cap, sms, K, 4), K), kTopkThreads, 0, m);
  GPUDB_LAUNCH(call, q3m_select_kernel, dim3(q3_topk_grid(max_cap, sms, K, 2), K), kTopkThreads, 0, m);
  std::vector<uint32_t> idv = ids;
  std::vector<int32_t> req_seg(m.req_seg, m.req_seg + K);
  return call.finish(bytes, [ctx, reqs, idv, req_seg, st_bytes](const uint8_t* h) {
    for (size_t r = 0; r < idv.size(); r++) {
      gpudb_request& q = reqs[idv[r]];
      uint32_t st, dst;
      std::memcpy(&st, h + 4 * r, 4);
      std::memcpy(&dst, h + 4 * (kB + req_seg[r]), 4);
      q.status = status_to_error(ctx, st | dst);
      if (q.status == GPUDB_OK) q3_result_from(h + st_bytes + r * kReqBytes, q.q3p.k, q.q3_out, GPUDB_JOIN_GLOBAL);
      if (ctx->on_done) ctx->on_done(ctx->on_done_arg, &q.status);
    }
    return GPUDB_OK;
  });
}

}  // namespace gpudb
