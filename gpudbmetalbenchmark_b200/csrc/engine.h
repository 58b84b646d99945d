// Engine internals: the context object behind gpudb_ctx*, call scopes, scratch memory,
// result slots, launch accounting and the chunked host->HBM streaming loop.
//
// These replace the reference's host infrastructure (src/infra.h): createPipeline /
// releaseAll / createFilledBuffer (src/infra.h:178-189, 519-531) become the scratch arena
// and RAII buffers, ChunkConfig + chunkedStreamLoop (src/infra.h:42-57, 816-869) become
// stream_lineitem(), and GPUStartTime/GPUEndTime timing becomes CUDA events per call.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/gpudb_capi.h"

namespace gpudb {

constexpr int kResultSlots = 1024;
constexpr size_t kSlotHeader = 16;                  // status word + padding
constexpr size_t kSlotBytes = 4096;                 // header + largest fixed-size result
constexpr int kBigSlots = 8;                        // slots for variable-size results
constexpr size_t kBigSlotBytes = 256 * 1024;
constexpr int kStreamSlots = 3;                     // device buffers of the streaming ring
constexpr uint64_t kDefaultChunkRows = 64ull << 20; // 64M rows per streamed chunk

struct Buffer {
  void* p = nullptr;
  size_t bytes = 0;
};

double now_ms();

}  // namespace gpudb

struct gpudb_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;       // compute stream
  cudaStream_t copy_stream = nullptr;  // host->device copies of streamed chunks
  cudaStream_t side_stream = nullptr;  // independent stages of one call (Call::side_begin)
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  std::string err;
  uint64_t launches = 0;
  uint64_t h2d_total = 0, d2h_total = 0;   // bytes moved by finished calls (batch timing)
  uint64_t chunk_rows = gpudb::kDefaultChunkRows;
  int scan_variant = 0;                // Q1 scan kernel choice (GPUDB_OPT_SCAN_VARIANT)
  int q6_variant = 0;                  // Q6 scan kernel choice (GPUDB_OPT_Q6_VARIANT)
  int ht_shift = 1;                    // hash tables hold <= 1/2^ht_shift load (GPUDB_OPT_HT_LOAD)
  int radix_bits = 0;                  // Q3 radix fan-out when a call leaves it 0 (GPUDB_OPT_RADIX_BITS)
  int radix_shape = 0;                 // radix scatter block shape (GPUDB_OPT_RADIX_SHAPE)
  int q3_auto_mode = -1;               // what a Q3 AUTO call runs; -1: the 30% rule (GPUDB_OPT_Q3_AUTO_MODE)
  int q9_smem_slots = 1024;            // Q9 aggregation slots when a call leaves them 0
  int q9_global_slots = 4096;
  struct Tuned {                       // autotuner choices (gpudb_autotune), for gpudb_tune_save
    int32_t pipeline, rows_log2, option;
    int64_t value;
  };
  std::vector<Tuned> tuned;
  // captured pipelines (CUDA graphs), replayed while the key and the scratch layout hold
  struct Graph {
    std::string key;
    cudaGraphExec_t exec;
    uint64_t scratch_gen;
    uint32_t kernels;
    uint64_t last_use;
  };
  std::vector<Graph> graphs;
  bool use_graphs = true;              // GPUDB_OPT_GRAPHS
  uint64_t scratch_gen = 0;            // bumped whenever a scratch buffer is (re)allocated
  uint64_t graph_clock = 0;
  std::unordered_map<std::string, gpudb::Buffer> scratch;
  std::vector<void*> retired;          // outgrown scratch, freed once the context is idle
  uint8_t* d_slots = nullptr;          // result slots (device)
  uint8_t* h_slots = nullptr;          // their pinned host mirror
  uint8_t* h_slots_dev = nullptr;      // the mirror's address in the device's address space (mapped), or null
  bool slot_busy[gpudb::kResultSlots] = {};
  int next_slot = 0;
  uint8_t* d_big = nullptr;            // large result slots (device) and their pinned mirror
  uint8_t* h_big = nullptr;
  bool big_busy[gpudb::kBigSlots] = {};
  int32_t* status_sink = nullptr;      // batch: where the next call reports its final status
  // called after a call's final status is written to its status sink (batches, serving)
  void (*on_done)(void* arg, int32_t* sink) = nullptr;
  void* on_done_arg = nullptr;
  struct Pending {
    cudaEvent_t done;                  // recorded after the call's result copy
    std::function<int()> finish;       // converts the result, writes the outputs
  };
  std::vector<Pending> pending;        // async calls in issue order
  std::vector<cudaStream_t> pending_streams;
  std::vector<cudaEvent_t> event_pool;
};

namespace gpudb {

int fail(gpudb_ctx* ctx, int code, const char* fmt, ...);
int cuda_fail(gpudb_ctx* ctx, cudaError_t e, const char* what);

#define GPUDB_CUDA(ctx, expr)                                  \
  do {                                                         \
    cudaError_t e_ = (expr);                                   \
    if (e_ != cudaSuccess) return gpudb::cuda_fail(ctx, e_, #expr); \
  } while (0)

// Grow-only named scratch buffer on the device (never shrinks; freed at gpudb_destroy);
// a new buffer is zero-filled before the call returns.
// Stream-ordered allocation: growing one context's buffer waits for that context's compute
// stream only, never for the whole device, and the outgrown buffer is freed in stream order
// once the context is idle (gpudb_sync, or a synchronous call with nothing pending).
int scratch(gpudb_ctx* ctx, const char* name, size_t bytes, void** out);

// Captured pipelines: the cached graph of `key` (null if none, or if a scratch buffer was
// reallocated since it was captured), and storing a newly instantiated one (the cache keeps
// kMaxGraphs, least recently used out).
constexpr size_t kMaxGraphs = 16;
gpudb_ctx::Graph* graph_find(gpudb_ctx* ctx, const std::string& key);
void graph_store(gpudb_ctx* ctx, const std::string& key, cudaGraphExec_t exec, uint32_t kernels);

// Kernel attributes cached per device (the runtime calls cost host time on every pipeline
// call otherwise): kernel_smem raises a kernel's dynamic shared-memory limit when `smem` is
// above what was set before; kernel_occupancy is the blocks per SM (at least 1) of a launch
// shape.
cudaError_t kernel_smem(gpudb_ctx* ctx, const void* fn, size_t smem);
int kernel_occupancy(gpudb_ctx* ctx, const void* fn, int threads, size_t smem);

cudaEvent_t event_get(gpudb_ctx* ctx);
void event_put(gpudb_ctx* ctx, cudaEvent_t e);

// One API call: picks the stream, owns a result slot and the timing events, and finishes
// synchronously or by deferring the completion to gpudb_sync().
class Call {
 public:
  Call(gpudb_ctx* ctx, const gpudb_exec* ex, gpudb_timing* t);
  ~Call();
  int begin(size_t result_bytes);          // acquires a slot and zeroes header + payload
  // Direct result: for a pipeline whose result comes from ONE kernel's last block. The slot
  // is not cleared and nothing is copied back: that block writes the status word and every
  // result byte (overwriting, not adding) straight into the call's pinned host slot, through
  // the slot's mapped device address, which direct_slot() returns (header, then payload).
  // Falls back to begin() when the slot cannot be written that way (large results, no
  // mapping); direct_slot() is then null and the pipeline launches as for begin().
  int begin_direct(size_t result_bytes);
  uint8_t* direct_slot() const { return direct_; }
  cudaStream_t stream() const { return s_; }
  uint32_t* status() const { return reinterpret_cast<uint32_t*>(dwork_ ? dwork_ : dslot_); }
  template <class T> T* result() const { return reinterpret_cast<T*>((dwork_ ? dwork_ : dslot_) + kSlotHeader); }
  // Kernels write status and result into `base` (slot layout: header, payload) instead of the
  // call's slot: a captured graph needs fixed pointers; the caller copies base into the slot.
  void redirect(uint8_t* base) { dwork_ = base; }
  uint8_t* slot_device() const { return dslot_; }
  uint32_t kernels() const { return kernels_; }
  void count_launch() { kernels_++; ctx_->launches++; }
  // launches recorded into a graph are not launches; a replay counts the graph's kernels
  void uncount_launches(uint32_t n) { kernels_ -= n; ctx_->launches -= n; }
  void count_launches(uint32_t n) { kernels_ += n; ctx_->launches += n; }
  void add_h2d(uint64_t b) { h2d_ += b; }
  void add_chunk() { chunks_++; }
  // Copies the result back and converts it with `convert(host_payload)`.
  int finish(size_t result_bytes, std::function<int(const uint8_t*)> convert);
  gpudb_ctx* ctx() const { return ctx_; }
  int check_launch(const char* name);
  // Independent stages on the context's side stream: side_begin() makes the side stream wait
  // for what the call has queued so far and sends the call's work there (stream() is the side
  // stream), side_end() sends it back without waiting, side_join() makes the call's stream
  // wait for the side stream's work. Under stream capture the side stream joins the capture
  // through the fork event and leaves it at the join.
  int side_begin();
  void side_end();
  int side_join();

 private:
  gpudb_ctx* ctx_;
  cudaStream_t s_;
  cudaStream_t main_ = nullptr;   // the call's stream while stream() is the side stream
  bool side_open_ = false;        // side work queued that the call's stream has not waited for
  bool async_;
  gpudb_timing* t_;
  cudaEvent_t e0_ = nullptr, e1_ = nullptr;
  double host0_;
  int slot_ = -1;
  bool big_ = false;
  uint8_t* dslot_ = nullptr;
  uint8_t* hslot_ = nullptr;
  uint8_t* dwork_ = nullptr;
  uint8_t* direct_ = nullptr;     // device address of hslot_ when the kernel writes it directly
  bool want_direct_ = false;
  uint32_t kernels_ = 0, chunks_ = 0;
  uint64_t h2d_ = 0, d2h_ = 0;
  bool handed_off_ = false;
  int32_t* status_sink_ = nullptr;
};

// Launch helper: counts the launch on the call and checks the launch error.
#define GPUDB_LAUNCH(call, kernel, grid, block, smem, ...)                          \
  do {                                                                              \
    kernel<<<(grid), (block), (smem), (call).stream()>>>(__VA_ARGS__);             \
    (call).count_launch();                                                          \
    int rc_ = (call).check_launch(#kernel);                                         \
    if (rc_ != GPUDB_OK) return rc_;                                                \
  } while (0)

// Status word -> error code (0 if clean).
int status_to_error(gpudb_ctx* ctx, uint32_t st);

// Columns of a lineitem chunk that a pipeline reads.
enum : uint32_t {
  LI_SHIP = 1u << 0, LI_QTY = 1u << 1, LI_EXT = 1u << 2, LI_DISC = 1u << 3, LI_TAX = 1u << 4,
  LI_FLAG = 1u << 5, LI_STATUS = 1u << 6, LI_ORDER = 1u << 7, LI_PART = 1u << 8, LI_SUPP = 1u << 9,
  LI_COMMIT = 1u << 10, LI_RECEIPT = 1u << 11, LI_MODE = 1u << 12
};
uint64_t lineitem_row_bytes(uint32_t mask);
int lineitem_check(gpudb_ctx* ctx, const gpudb_lineitem* li, uint32_t mask);

// Runs `dispatch(chunk)` once per chunk of a lineitem table. Device-resident tables are
// one chunk that points at the caller's columns. Host-resident tables are copied in
// chunks of `chunk_rows` rows into a ring of kStreamSlots device buffers on the copy
// stream while the compute stream runs the previous chunk (events order the two).
int stream_lineitem(Call& call, const gpudb_lineitem* li, uint32_t mask, uint64_t chunk_rows,
                    const std::function<int(const gpudb_lineitem&)>& dispatch);

}  // namespace gpudb
