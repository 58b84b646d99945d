// Self-test of the bounded device waits: one warp waits, through the same mbar_wait the
// TMA scan kernels use, on a shared-memory mbarrier. With `arrive` a thread arrives first
// and the wait completes; without, nothing ever arrives and the wait gives up after `polls`
// polls, sets ST_TIMEOUT and the kernel returns normally: the call reports
// GPUDB_E_TIMEOUT and the context stays usable. This is how a stalled copy in a scan kernel
// surfaces, tested without stalling one.
#include "common.cuh"
#include "engine.h"
#include "tma.cuh"

namespace gpudb {
namespace {

__global__ void bounded_wait_kernel(uint32_t polls, int arrive, uint32_t* status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (arrive) mbar_arrive(&bar);
    if (!mbar_wait(&bar, 0, polls)) set_status(status, ST_TIMEOUT);
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&bar)) : "memory");
  }
  __syncthreads();
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_selftest_bounded_wait(gpudb_ctx* ctx, uint32_t polls, int32_t arrive) {
  if (!ctx) return GPUDB_E_INVALID;
  if (polls < 1 || polls > kMbarPollLimit) return fail(ctx, GPUDB_E_INVALID, "selftest: polls must be in 1..%u", kMbarPollLimit);
  Call call(ctx, nullptr, nullptr);
  int rc = call.begin(8);
  if (rc) return rc;
  GPUDB_LAUNCH(call, bounded_wait_kernel, 1, 32, 0, polls, arrive ? 1 : 0, call.status());
  return call.finish(8, [](const uint8_t*) { return GPUDB_OK; });
}
