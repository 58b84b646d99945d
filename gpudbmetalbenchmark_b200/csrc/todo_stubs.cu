// Entry points whose kernels are not written yet: they report GPUDB_E_UNSUPPORTED.
#include "engine.h"
#include "q3.h"
namespace gpudb {
int q3_radix(Call& call, const gpudb_customer&, const gpudb_orders&, const gpudb_lineitem*, const gpudb_q3_params&,
             uint8_t*) {
  return fail(call.ctx(), GPUDB_E_UNSUPPORTED, "radix mode not built yet");
}
}  // namespace gpudb
using namespace gpudb;
extern "C" {
int gpudb_select_lt(gpudb_ctx* ctx, const int32_t*, uint64_t, int32_t, uint32_t*, uint32_t*, uint64_t*,
                    gpudb_timing*, const gpudb_exec*) { return fail(ctx, GPUDB_E_UNSUPPORTED, "not built yet"); }
int gpudb_sum_i32(gpudb_ctx* ctx, const int32_t*, uint64_t, int64_t*, gpudb_timing*, const gpudb_exec*) {
  return fail(ctx, GPUDB_E_UNSUPPORTED, "not built yet");
}
int gpudb_hash_join_count(gpudb_ctx* ctx, const int32_t*, uint64_t, const int32_t*, uint64_t, int32_t, uint64_t*,
                          gpudb_timing*, const gpudb_exec*) { return fail(ctx, GPUDB_E_UNSUPPORTED, "not built yet"); }
int gpudb_radix_partition(gpudb_ctx* ctx, const int32_t*, const int32_t*, uint64_t, int32_t, int32_t*, int32_t*,
                          uint32_t*, gpudb_timing*, const gpudb_exec*) { return fail(ctx, GPUDB_E_UNSUPPORTED, "not built yet"); }
int gpudb_radix_join_pairs(gpudb_ctx* ctx, const int32_t*, uint64_t, const int32_t*, uint64_t, int32_t*, int32_t*,
                           uint64_t, uint64_t*, gpudb_timing*, const gpudb_exec*) {
  return fail(ctx, GPUDB_E_UNSUPPORTED, "not built yet");
}
}
