// gpudb_q6_sum_noalloc: the Q6-like filtered sum for callers that cannot allocate.
//
// Some callers cannot call cudaMalloc at all: host programs embedded in a process whose
// device memory is owned and budgeted by someone else (a database server whose memory
// manager hands out all of the GPU, where a stray allocation would fail or push the server
// over its budget), and plugins loaded where no context object of this library exists
// (the context is what owns this library's scratch buffers). This entry point needs
// neither a context nor any allocation: the caller passes the device columns and a device
// output buffer, and the only scratch memory (the per-block partial sums and the last-block
// ticket) is a file-scope __device__ array of fixed size that every GPU which loads this
// library holds until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "engine.h"

namespace {

constexpr int kThreads = 256;
constexpr int kQuadsPerThread = 4;                                   // 16 rows per thread
constexpr uint64_t kRowsPerBlock = (uint64_t)kThreads * kQuadsPerThread * 4;   // 4096
constexpr uint32_t kMaxBlocks = 16384;
constexpr uint64_t kMaxRows = kRowsPerBlock * kMaxBlocks;            // 67,108,864 rows
constexpr size_t kHeader = 256;                                      // the ticket word, padded
constexpr size_t kScratchBytes = kHeader + (size_t)kMaxBlocks * 16;  // 262,400 bytes

// Scratch shared by every call on a device: [ticket | revenue partials | count partials].
static __device__ __align__(256) unsigned char g_q6_scratch[kScratchBytes];

struct Params { int32_t lo, hi, dlo, dhi, qlt; };

__device__ __forceinline__ bool pass(int32_t s, int32_t d, int32_t q, const Params& p) {
  return (s >= p.lo) & (s < p.hi) & (d >= p.dlo) & (d <= p.dhi) & (q < p.qlt);
}

// Block b owns rows [b*4096, (b+1)*4096); `vec` selects 128-bit loads (all columns
// 16-byte aligned) or one row at a time. The last block to finish writes the totals to
// out[0] (revenue) and out[1] (rows matched), overwriting them.
__global__ void __launch_bounds__(kThreads) q6_noalloc_kernel(const int32_t* __restrict__ ship,
                                                              const int32_t* __restrict__ disc,
                                                              const int32_t* __restrict__ qty,
                                                              const int64_t* __restrict__ ext, uint64_t n, Params p,
                                                              bool vec, unsigned char* scratch, int64_t* out) {
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch);
  int64_t* part_rev = reinterpret_cast<int64_t*>(scratch + kHeader);
  uint64_t* part_cnt = reinterpret_cast<uint64_t*>(part_rev + kMaxBlocks);
  const uint64_t row0 = (uint64_t)blockIdx.x * kRowsPerBlock;
  int64_t rev = 0;
  uint64_t cnt = 0;
  if (vec && row0 + kRowsPerBlock <= n) {
    const int4* s4 = reinterpret_cast<const int4*>(ship + row0);
    const int4* d4 = reinterpret_cast<const int4*>(disc + row0);
    const int4* q4 = reinterpret_cast<const int4*>(qty + row0);
#pragma unroll
    for (int j = 0; j < kQuadsPerThread; j++) {
      const int qd = j * kThreads + threadIdx.x;
      const int4 s = ld_stream(s4 + qd), d = ld_stream(d4 + qd), q = ld_stream(q4 + qd);
      const uint64_t r = row0 + 4ull * qd;
      if (pass(s.x, d.x, q.x, p)) { rev += ld_stream(ext + r + 0) * (int64_t)d.x; cnt++; }
      if (pass(s.y, d.y, q.y, p)) { rev += ld_stream(ext + r + 1) * (int64_t)d.y; cnt++; }
      if (pass(s.z, d.z, q.z, p)) { rev += ld_stream(ext + r + 2) * (int64_t)d.z; cnt++; }
      if (pass(s.w, d.w, q.w, p)) { rev += ld_stream(ext + r + 3) * (int64_t)d.w; cnt++; }
    }
  } else {
    for (uint64_t r = row0 + threadIdx.x; r < row0 + kRowsPerBlock && r < n; r += kThreads)
      if (pass(ship[r], disc[r], qty[r], p)) { rev += ext[r] * (int64_t)disc[r]; cnt++; }
  }
  __shared__ uint64_t sr[kThreads / 32], sc[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t a = warp_sum_u64((uint64_t)rev), b = warp_sum_u64(cnt);
  if (lane == 0) { sr[warp] = a; sc[warp] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t ta = 0, tb = 0;
    for (int w = 0; w < kThreads / 32; w++) { ta += sr[w]; tb += sc[w]; }
    part_rev[blockIdx.x] = (int64_t)ta;
    part_cnt[blockIdx.x] = tb;
  }
  if (!grid_last_block(ticket)) return;
  a = 0;
  b = 0;
  for (unsigned i = threadIdx.x; i < gridDim.x; i += kThreads) {
    a += (uint64_t)__ldcg(part_rev + i);
    b += __ldcg(part_cnt + i);
  }
  a = warp_sum_u64(a);
  b = warp_sum_u64(b);
  __syncthreads();
  if (lane == 0) { sr[warp] = a; sc[warp] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t ta = 0, tb = 0;
    for (int w = 0; w < kThreads / 32; w++) { ta += sr[w]; tb += sc[w]; }
    out[0] = (int64_t)ta;
    out[1] = (int64_t)tb;
  }
}

// Device address of g_q6_scratch, looked up once per device (with that device current) and
// kept for the life of the process: a device reset (cudaDeviceReset) after the first call
// on that device is not supported, since the array may then load at another address.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

int scratch_address(int device, void** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_q6_scratch) != cudaSuccess || !p) return GPUDB_E_CUDA;
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return GPUDB_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

extern "C" int gpudb_q6_sum_noalloc(const gpudb_lineitem* li, const gpudb_q6_params* p, int64_t* out,
                                    void* stream) {
  if (!li || !p || !out) return GPUDB_E_INVALID;
  if (li->location != GPUDB_MEM_DEVICE) return GPUDB_E_INVALID;
  if (li->n_rows > kMaxRows) return GPUDB_E_CAPACITY;   // beyond the fixed scratch
  if (li->n_rows && (!li->ship_date || !li->discount || !li->quantity || !li->ext_price)) return GPUDB_E_INVALID;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return GPUDB_E_CUDA;
  void* scratch = nullptr;
  int rc = scratch_address(device, &scratch);
  if (rc != GPUDB_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (li->n_rows == 0) {
    // nothing to scan: the totals are zero
    return cudaMemsetAsync(out, 0, 2 * sizeof(int64_t), s) == cudaSuccess ? GPUDB_OK : GPUDB_E_CUDA;
  }
  // An error that the caller's own earlier CUDA work left in the runtime's last-error slot
  // is the caller's: it is neither reported as this call's failure nor cleared here.
  const bool clean_before = cudaPeekAtLastError() == cudaSuccess;
  // the ticket must start at zero; the partials are fully rewritten by each launch
  if (cudaMemsetAsync(scratch, 0, sizeof(unsigned), s) != cudaSuccess) return GPUDB_E_CUDA;
  const unsigned grid = (unsigned)((li->n_rows + kRowsPerBlock - 1) / kRowsPerBlock);
  const bool vec = aligned16(li->ship_date) && aligned16(li->discount) && aligned16(li->quantity);
  const Params pp{p->ship_lo, p->ship_hi, p->disc_lo, p->disc_hi, p->qty_lt};
  q6_noalloc_kernel<<<grid, kThreads, 0, s>>>(li->ship_date, li->discount, li->quantity, li->ext_price, li->n_rows, pp,
                                              vec, static_cast<unsigned char*>(scratch), out);
  if (!clean_before) return GPUDB_OK;
  return cudaGetLastError() == cudaSuccess ? GPUDB_OK : GPUDB_E_CUDA;
}
