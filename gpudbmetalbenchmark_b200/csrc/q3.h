// Q3-like pipeline entry points shared between the global-table (q3.cu) and the
// radix-partitioned (radix.cu) implementations.
#pragma once
#include "common.cuh"
#include "engine.h"

namespace gpudb {

// Result payload of both modes: {u64 groups, u64 pad, u128 rows[k]} (rows as top-k
// composites, see topk_compose).
int q3_global(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_lineitem* li,
              const gpudb_q3_params& p, uint8_t* result);
int q3_radix(Call& call, const gpudb_customer& cu, const gpudb_orders& od, const gpudb_lineitem* li,
             const gpudb_q3_params& p, uint8_t* result);
// Reduces n_cand composites to the top k (k per 4096-candidate tile per level).
int q3_topk_levels(Call& call, u128* cand, uint64_t n_cand, int k, u128* scratch_a, u128* scratch_b, u128* final_out);

}  // namespace gpudb
