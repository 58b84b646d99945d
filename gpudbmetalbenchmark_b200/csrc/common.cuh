// Device-side helpers shared by every kernel of the engine (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

typedef unsigned __int128 u128;
typedef __int128 i128;

#define FULL_MASK 0xFFFFFFFFu

// Device status bits, OR-ed into the call's status word by any kernel that detects a
// condition the host must report (never a trap: the kernel skips the access and returns).
enum : uint32_t {
  ST_CAPACITY = 1u,    // a hash table / partition / output buffer would overflow
  ST_KEY_RANGE = 2u,   // a key outside the declared key range
  ST_DOMAIN = 4u,      // a value outside the exact-arithmetic domain of the pipeline
  ST_TIMEOUT = 8u,     // a bounded device wait ran out
  ST_DUPLICATE = 16u   // a unique build side holds a key twice
};

__device__ __forceinline__ void set_status(uint32_t* status, uint32_t bits) {
  if (status) atomicOr(status, bits);
}

// ---- warp reductions -----------------------------------------------------------------
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(FULL_MASK, v, d);
  return v;
}

__device__ __forceinline__ u128 warp_sum_u128(u128 v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    uint64_t lo = __shfl_down_sync(FULL_MASK, (uint64_t)v, d);
    uint64_t hi = __shfl_down_sync(FULL_MASK, (uint64_t)(v >> 64), d);
    v += ((u128)hi << 64) | lo;
  }
  return v;
}

constexpr int kRadixMaxBits = 16;   // radix partitioning: largest fan-out, in bits

// ---- last-block-done grid reduction ---------------------------------------------------
// Each block publishes its partials, then takes a ticket; the block that draws the last
// ticket sees every partial (fence before the ticket) and resets the ticket to zero so
// the next launch starts clean without a memset.
__device__ __forceinline__ bool grid_last_block(unsigned* ticket) {
  __shared__ bool last;
  __threadfence();   // every thread's partial results are visible device-wide before the ticket
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
    if (last) __threadfence();   // the last block then reads every block's partials
  }
  __syncthreads();
  if (last && threadIdx.x == 0) *ticket = 0u;
  return last;
}

// ---- hashing ----------------------------------------------------------------------------
// The reference's 32-bit key hash (sf100_hash_key, kernels/common.h:81-87): an xorshift-
// multiply finaliser; used for radix partition numbers so partitions match the reference.
__host__ __device__ __forceinline__ uint32_t key_hash32(int32_t key) {
  uint32_t h = (uint32_t)key;
  h ^= h >> 16;
  h *= 0x45d9f3bu;
  h ^= h >> 16;
  return h;
}

// Hash-table slot hash: a full 64-bit finaliser (SplitMix64 output function) of the key,
// folded to 32 bits; independent of the radix bits taken from key_hash32.
__host__ __device__ __forceinline__ uint32_t slot_hash64(uint64_t k) {
  k ^= k >> 30; k *= 0xBF58476D1CE4E5B9ull;
  k ^= k >> 27; k *= 0x94D049BB133111EBull;
  k ^= k >> 31;
  return (uint32_t)k;
}

// ---- bitmaps ------------------------------------------------------------------------------
__device__ __forceinline__ bool bitmap_test(const uint32_t* bm, int32_t key) {
  return (__ldg(bm + ((uint32_t)key >> 5)) >> ((uint32_t)key & 31u)) & 1u;
}

// ---- streaming loads (read once: do not keep in L1) ---------------------------------------
template <class T> __device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }
