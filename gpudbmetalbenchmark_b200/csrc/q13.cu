// Q13 (customer distribution): orders whose comment is NOT LIKE '%word1%word2%' are counted
// per customer, then customers are counted per order count (custdist), ordered by custdist
// desc, c_count desc.
// Reference: kernels/q13.metal:33-168 (pattern match into a qualifies byte, per-customer
// counts with device atomics, threadgroup-privatised histogram), src/q13.cpp:8-117 (driver),
// postProcessQ13 src/infra.h:778-800 (sort of the histogram).
//
// B200 design:
//  - q13_count_kernel: one order per thread; its 80-byte comment slot goes into 20 registers
//    (five 16-byte loads), and one branch-free pass marks with SWAR tests the positions whose
//    first two bytes match word1 or word2; only those (rare) candidates are compared in full,
//    so the lanes of a warp stay converged. Qualifying orders add 1 to their customer's count
//    (L2-resident counter array, one atomic per order).
//  - q13_hist_kernel: every customer row looks up its count and adds to a shared-memory
//    histogram of GPUDB_Q13_MAX_COUNT + 1 bins, flushed with one atomic per nonzero bin.
//  - q13_sort_kernel: one block ranks the nonzero bins (custdist desc, c_count desc).
#include <cstring>

#include "common.cuh"
#include "engine.h"

namespace gpudb {
namespace {

constexpr int kQ13Threads = 256;
constexpr int kSlotWords = GPUDB_COMMENT_WIDTH / 4;   // 20
constexpr int kBins = GPUDB_Q13_MAX_COUNT + 1;

struct Q13Pattern {
  uint8_t w[2][16];   // NUL-padded
  int32_t len[2];
};

// High bit of every byte of x that is zero (exact per byte).
__device__ __forceinline__ uint32_t zero_bytes(uint32_t x) {
  const uint32_t y = (x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu;
  return ~(y | x | 0x7F7F7F7Fu);
}

__device__ __forceinline__ bool word_at(const uint8_t* row, int pos, const uint8_t* w, int len) {
  if (pos + len > GPUDB_COMMENT_WIDTH) return false;
  for (int c = 1; c < len; c++)   // the first letter is known to match
    if (row[pos + c] != w[c]) return false;
  return true;
}

// LIKE '%w0%w1%' on one NUL-padded row: its kSlotWords words in registers, its bytes at
// `row` (global memory, read again only to verify candidates). One branch-free pass marks,
// for both words, the positions whose first two bytes match (SWAR on the row word and the row
// word shifted by one byte); only those candidates, rare for two-letter prefixes, are
// compared in full: the first verified w0, then any verified w1 at or after its end.
// Candidate flags (bits 7, 15, 23, 31 of a word's test) are packed eight words to a register
// with two operations: word k's flags land on bits (k & 7) + {0, 8, 16, 24} of c[k >> 3], so
// bit b of c[q] is position 4 * (8q + (b & 7)) + (b >> 3). Bits are visited in bit order,
// not position order: the first w0 is the smallest verified position.
__device__ bool like2(const uint32_t (&rw)[kSlotWords], const uint8_t* row, const uint8_t (&w)[2][16],
                      const int32_t (&len)[2]) {
  const uint32_t a0 = w[0][0] * 0x01010101u, b0 = w[0][1] * 0x01010101u;
  const uint32_t a1 = w[1][0] * 0x01010101u, b1 = w[1][1] * 0x01010101u;
  const bool two0 = len[0] > 1, two1 = len[1] > 1;
  uint32_t c0[3] = {0, 0, 0}, c1[3] = {0, 0, 0};
#pragma unroll
  for (int k = 0; k < kSlotWords; k++) {
    const uint32_t x = rw[k], nx = k + 1 < kSlotWords ? rw[k + 1] : 0u;
    const uint32_t y = __funnelshift_r(x, nx, 8);   // the byte after each byte of x
    const uint32_t m0 = zero_bytes(x ^ a0) & (two0 ? zero_bytes(y ^ b0) : 0x80808080u);
    const uint32_t m1 = zero_bytes(x ^ a1) & (two1 ? zero_bytes(y ^ b1) : 0x80808080u);
    const int j = k & 7;
    c0[k >> 3] |= (m0 >> (7 - j)) & (0x01010101u << j);
    c1[k >> 3] |= (m1 >> (7 - j)) & (0x01010101u << j);
  }
  constexpr int kNone = 1 << 30;
  int first = kNone;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    uint32_t m = c0[q];
    while (m) {
      const int b = __ffs(m) - 1;
      m &= m - 1;
      const int pos = 4 * (8 * q + (b & 7)) + (b >> 3);
      if (pos < first && word_at(row, pos, w[0], len[0])) first = pos;
    }
  }
  if (first == kNone) return false;
  const int start = first + len[0];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    uint32_t m = c1[q];
    while (m) {
      const int b = __ffs(m) - 1;
      m &= m - 1;
      const int pos = 4 * (8 * q + (b & 7)) + (b >> 3);
      if (pos >= start && word_at(row, pos, w[1], len[1])) return true;
    }
  }
  return false;
}

// One order per thread (grid-stride): its comment goes straight into registers (five 16-byte
// loads when the column is aligned), no shared staging and no block barrier.
__global__ void __launch_bounds__(kQ13Threads) q13_count_kernel(const char* __restrict__ comment,
                                                                 const int32_t* __restrict__ ocust, uint64_t n,
                                                                 int32_t cust_max, Q13Pattern pat, uint32_t* counts) {
  __shared__ uint8_t sw[2][16];
  __shared__ int32_t slen[2];
  if (threadIdx.x < 32) sw[threadIdx.x >> 4][threadIdx.x & 15] = pat.w[threadIdx.x >> 4][threadIdx.x & 15];
  if (threadIdx.x < 2) slen[threadIdx.x] = pat.len[threadIdx.x];
  __syncthreads();
  const bool vec = (reinterpret_cast<uintptr_t>(comment) & 15u) == 0;
  const uint64_t stride = (uint64_t)gridDim.x * kQ13Threads;
  for (uint64_t r = (uint64_t)blockIdx.x * kQ13Threads + threadIdx.x; r < n; r += stride) {
    const int32_t c = ld_stream(ocust + r);
    if (c < 0 || c > cust_max) continue;   // an order of no known customer: its comment is not read
    const uint8_t* row = reinterpret_cast<const uint8_t*>(comment) + r * GPUDB_COMMENT_WIDTH;
    uint32_t rw[kSlotWords];
    if (vec) {
#pragma unroll
      for (int q = 0; q < kSlotWords / 4; q++) {
        const uint4 v = ld_stream(reinterpret_cast<const uint4*>(row) + q);
        rw[4 * q] = v.x; rw[4 * q + 1] = v.y; rw[4 * q + 2] = v.z; rw[4 * q + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < kSlotWords; k++)
        rw[k] = row[4 * k] | (uint32_t)row[4 * k + 1] << 8 | (uint32_t)row[4 * k + 2] << 16 | (uint32_t)row[4 * k + 3] << 24;
    }
    if (!like2(rw, row, sw, slen)) atomicAdd(counts + c, 1u);
  }
}

__global__ void __launch_bounds__(256) q13_hist_kernel(const int32_t* __restrict__ ckey, uint64_t n, int32_t cust_max,
                                                       const uint32_t* __restrict__ counts, uint32_t* hist,
                                                       uint32_t* status) {
  __shared__ uint32_t sh[kBins];
  for (int i = threadIdx.x; i < kBins; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const int32_t k = ld_stream(ckey + i);
    if (k < 0 || k > cust_max) { set_status(status, ST_KEY_RANGE); continue; }
    const uint32_t c = counts[k];
    if (c >= (uint32_t)kBins) { set_status(status, ST_CAPACITY); continue; }
    atomicAdd(&sh[c], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kBins; i += blockDim.x)
    if (sh[i]) atomicAdd(hist + i, sh[i]);
}

// out = {u32 n, pad[3], rows[n] of (c_count, custdist)} ordered by custdist desc, c_count desc.
__global__ void __launch_bounds__(kBins) q13_sort_kernel(const uint32_t* __restrict__ hist, uint8_t* out) {
  __shared__ uint32_t h[kBins];
  const uint32_t b = threadIdx.x;
  h[b] = hist[b];
  const uint32_t cd = h[b];
  const int n = __syncthreads_count(cd != 0);
  if (cd) {
    uint32_t r = 0;
    for (uint32_t j = 0; j < (uint32_t)kBins; j++) {
      const uint32_t o = h[j];
      r += (o > cd) | ((o == cd) & (j > b));
    }
    reinterpret_cast<uint2*>(out + 16)[r] = make_uint2(b, cd);
  }
  if (b == 0) *reinterpret_cast<uint32_t*>(out) = (uint32_t)n;
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_q13_distribution(gpudb_ctx* ctx, const gpudb_customer* cu, const gpudb_orders* od,
                                      const gpudb_q13_params* p, gpudb_q13_row* out, uint32_t capacity,
                                      uint32_t* n_rows, gpudb_timing* t, const gpudb_exec* ex) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!cu || !od || !p || !n_rows || (capacity && !out))
    return fail(ctx, GPUDB_E_INVALID, "q13: customer, orders, params and n_rows are required");
  if (cu->n_rows && (!cu->cust_key || cu->key_max < 0))
    return fail(ctx, GPUDB_E_INVALID, "q13: customer.cust_key and key_max >= 0 are required");
  if (od->n_rows && (!od->cust_key || !od->comment))
    return fail(ctx, GPUDB_E_INVALID, "q13: orders.cust_key and orders.comment are required");
  Q13Pattern pat{};
  for (int i = 0; i < 2; i++) {
    const char* w = i ? p->word2 : p->word1;
    const size_t l = strnlen(w, 16);
    if (l < 1 || l > 15) return fail(ctx, GPUDB_E_INVALID, "q13: word%d must be 1..15 characters", i + 1);
    std::memcpy(pat.w[i], w, l);
    pat.len[i] = (int32_t)l;
  }
  Call call(ctx, ex, t);
  const size_t bytes = 16 + (size_t)kBins * sizeof(gpudb_q13_row);
  int rc = call.begin(bytes);
  if (rc) return rc;
  cudaStream_t s = call.stream();
  const int32_t cust_max = cu->n_rows ? cu->key_max : 0;
  void *counts = nullptr, *hist = nullptr;
  if ((rc = scratch(ctx, "q13.counts", ((size_t)cust_max + 1) * 4, &counts))) return rc;
  if ((rc = scratch(ctx, "q13.hist", (size_t)kBins * 4, &hist))) return rc;
  GPUDB_CUDA(ctx, cudaMemsetAsync(counts, 0, ((size_t)cust_max + 1) * 4, s));
  GPUDB_CUDA(ctx, cudaMemsetAsync(hist, 0, (size_t)kBins * 4, s));
  const int sms = ctx->sm_count;
  if (od->n_rows && cu->n_rows) {
    const unsigned g = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((od->n_rows + kQ13Threads - 1) / kQ13Threads, (uint64_t)sms * 8));
    GPUDB_LAUNCH(call, q13_count_kernel, g, kQ13Threads, 0, od->comment, od->cust_key, od->n_rows, cust_max, pat,
                 (uint32_t*)counts);
  }
  if (cu->n_rows) {
    const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((cu->n_rows + 255) / 256, (uint64_t)sms * 4));
    GPUDB_LAUNCH(call, q13_hist_kernel, g, 256, 0, cu->cust_key, cu->n_rows, cust_max, (const uint32_t*)counts,
                 (uint32_t*)hist, call.status());
  }
  GPUDB_LAUNCH(call, q13_sort_kernel, 1, kBins, 0, (const uint32_t*)hist, call.result<uint8_t>());
  const uint32_t cap = capacity;
  return call.finish(bytes, [out, cap, n_rows](const uint8_t* h) {
    uint32_t n;
    std::memcpy(&n, h, 4);
    *n_rows = n;
    if (cap) std::memcpy(out, h + 16, (size_t)std::min(n, cap) * sizeof(gpudb_q13_row));
    return GPUDB_OK;
  });
}
