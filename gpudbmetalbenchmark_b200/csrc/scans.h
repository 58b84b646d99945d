// Launchers of the Q6/Q1 scan kernels (scans.cu), shared with the batch path (batch.cu).
#pragma once
#include "engine.h"

namespace gpudb {

constexpr size_t kQ6ResultBytes = 16;              // int64 revenue, uint64 rows matched
constexpr size_t kQ1ResultBytes = 6 * 6 * 16;      // 6 groups x {count, qty, base, disc_price, charge, discount} u128

// Enqueue one scan of device-resident columns on the call's stream, adding into `out`
// (device; kQ6ResultBytes / kQ1ResultBytes, zeroed before the first chunk). Q1 reports a
// value outside its exact-arithmetic domain in `status` (the call's status word if null).
int launch_q6(Call& call, const gpudb_lineitem& c, const gpudb_q6_params& p, void* out);
int launch_q1(Call& call, const gpudb_lineitem& c, const gpudb_q1_params& p, void* out, uint32_t* status = nullptr);

// Host result from the kQ1ResultBytes device words of one Q1 scan.
void q1_result_from(const uint8_t* words, gpudb_q1_result* out);

}  // namespace gpudb
