// Q3-like pipeline entry points shared between the global-table (q3.cu) and the
// radix-partitioned (radix.cu) implementations.
#pragma once
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "join_common.cuh"

namespace gpudb {

// Orders hash-table slot; the table doubles as the per-order aggregation table.
struct Q3Slot {
  int32_t key;
  int32_t date;
  unsigned long long rev;
};

__device__ __forceinline__ int32_t ht_find(const Q3Slot* ht, uint32_t cap, int32_t key) {
  const uint32_t mask = cap - 1;
  uint32_t s = key_slot(key, mask);
  for (uint32_t p = 0; p < cap; p++, s = (s + 1) & mask) {
    const int32_t k = __ldg(&ht[s].key);
    if (k == key) return (int32_t)s;
    if (k == kEmptyKey) return -1;
  }
  return -1;
}

// Other blocks' top-k candidates, read past L1.
__device__ __forceinline__ u128 ld_cg_u128(const u128* p) {
  const ulonglong2 q = __ldcg(reinterpret_cast<const ulonglong2*>(p));
  return ((u128)q.y << 64) | q.x;
}

// Result conversion shared by the single and the batched Q3: payload {u64 groups, u64 pad,
// u128 rows[k]} -> gpudb_q3_result.
void q3_result_from(const uint8_t* h, int k, gpudb_q3_result* out);

// Q3 requests (global-table mode, device-resident lineitem, identical tables) evaluated
// together: every stage is one launch for all of them and the fact table is probed once.
// Returns GPUDB_OK if enqueued; each request's outcome arrives in its status.
constexpr int kQ3Batch = 8;
bool q3_batchable(const gpudb_request& q);
int q3_batch_run(gpudb_ctx* ctx, gpudb_request* reqs, const std::vector<uint32_t>& ids, const gpudb_exec* ex);

// Result payload of both modes: {u64 groups, u64 pad, u128 rows[k]} (rows as top-k
// composites, see topk_compose).
int q3_global(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_lineitem* li,
              const gpudb_q3_params& p, uint8_t* result);
int q3_radix(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_lineitem* li,
             const gpudb_q3_params& p, uint8_t* result);
// Reduces n_cand composites to the top k (k per 4096-candidate tile per level).
int q3_topk_levels(Call& call, u128* cand, uint64_t n_cand, int k, u128* scratch_a, u128* scratch_b, u128* final_out);

}  // namespace gpudb
