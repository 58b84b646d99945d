// Launchers of the Q6/Q1 scan kernels (scans.cu), shared with the batch path (batch.cu).
#pragma once
#include "engine.h"

namespace gpudb {

constexpr size_t kQ6ResultBytes = 16;              // int64 revenue, uint64 rows matched
constexpr size_t kQ1ResultBytes = 6 * 6 * 16;      // 6 groups x {count, qty, base, disc_price, charge, discount} u128

// Enqueue one scan of device-resident columns on the call's stream, adding into `out`
// (device; kQ6ResultBytes / kQ1ResultBytes, zeroed before the first chunk). Q1 reports a
// value outside its exact-arithmetic domain in `status` (the call's status word if null).
// Q6 with `hstatus` (the status word of the call's mapped host slot, Call::begin_direct)
// overwrites `out` in that slot instead: one launch over the whole table.
int launch_q6(Call& call, const gpudb_lineitem& c, const gpudb_q6_params& p, void* out, uint32_t* hstatus = nullptr);
int launch_q1(Call& call, const gpudb_lineitem& c, const gpudb_q1_params& p, void* out, uint32_t* status = nullptr);
// One Q1 scan that also evaluates up to 4 Q6 requests on the rows it reads (one read of the
// table for all of them); each Q6 request adds into its own kQ6ResultBytes words. Falls back
// to one kernel per request for columns off 16 bytes, more Q6 requests, or a Q1 kernel
// variant chosen on the context.
int launch_q1_riders(Call& call, const gpudb_lineitem& c, const gpudb_q1_params& p, void* out, uint32_t* status,
                     int n6, const gpudb_q6_params* q6, void* const* q6out);

// Host result from the kQ1ResultBytes device words of one Q1 scan.
void q1_result_from(const uint8_t* words, gpudb_q1_result* out);

}  // namespace gpudb
