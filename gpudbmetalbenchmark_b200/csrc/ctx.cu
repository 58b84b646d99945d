// Context lifecycle, memory, result slots, async completion and chunked streaming.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"
#include "engine.h"

namespace gpudb {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

int fail(gpudb_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

int cuda_fail(gpudb_ctx* ctx, cudaError_t e, const char* what) {
  (void)cudaGetLastError();   // reported here: a later launch check must not see it again
  int code = (e == cudaErrorMemoryAllocation) ? GPUDB_E_OOM : GPUDB_E_CUDA;
  return fail(ctx, code, "%s: %s", what, cudaGetErrorString(e));
}

int scratch(gpudb_ctx* ctx, const char* name, size_t bytes, void** out) {
  Buffer& b = ctx->scratch[name];
  if (b.bytes < bytes) {
    if (b.p) {
      // queued work may still read the old buffer: retire it until the context is idle
      ctx->retired.push_back(b.p);
      b.p = nullptr;
      b.bytes = 0;
    }
    size_t sz = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMallocAsync(&b.p, sz, ctx->stream);
    // pool memory holds whatever its last owner left: new scratch starts zeroed (last-block
    // tickets and counters rely on it), and the allocation and the fill complete before any
    // stream of this context (or a caller's) uses the buffer
    if (e == cudaSuccess) e = cudaMemsetAsync(b.p, 0, sz, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    ctx->scratch_gen++;   // captured graphs hold scratch pointers
    if (e != cudaSuccess) {
      b.p = nullptr;
      return e == cudaErrorMemoryAllocation ? fail(ctx, GPUDB_E_OOM, "scratch %s: %zu bytes", name, sz)
                                            : cuda_fail(ctx, e, "cudaMallocAsync");
    }
    b.bytes = sz;
  }
  *out = b.p;
  return GPUDB_OK;
}

gpudb_ctx::Graph* graph_find(gpudb_ctx* ctx, const std::string& key) {
  for (auto& g : ctx->graphs)
    if (g.key == key) {
      if (g.scratch_gen != ctx->scratch_gen) return nullptr;
      g.last_use = ++ctx->graph_clock;
      return &g;
    }
  return nullptr;
}

void graph_store(gpudb_ctx* ctx, const std::string& key, cudaGraphExec_t exec, uint32_t kernels) {
  for (auto it = ctx->graphs.begin(); it != ctx->graphs.end(); ++it)
    if (it->key == key) {   // stale (a scratch buffer moved): replace
      cudaGraphExecDestroy(it->exec);
      ctx->graphs.erase(it);
      break;
    }
  if (ctx->graphs.size() >= kMaxGraphs) {
    auto lru = std::min_element(ctx->graphs.begin(), ctx->graphs.end(),
                                [](const gpudb_ctx::Graph& a, const gpudb_ctx::Graph& b) { return a.last_use < b.last_use; });
    cudaGraphExecDestroy(lru->exec);
    ctx->graphs.erase(lru);
  }
  ctx->graphs.push_back({key, exec, ctx->scratch_gen, kernels, ++ctx->graph_clock});
}

// Frees outgrown scratch; only when no work of the context can still be queued.
void release_retired(gpudb_ctx* ctx) {
  for (void* p : ctx->retired) cudaFreeAsync(p, ctx->stream);
  ctx->retired.clear();
}

namespace {
std::mutex g_attr_mu;
std::map<std::pair<int, const void*>, size_t> g_smem_set;
std::map<std::tuple<int, const void*, int, size_t>, int> g_occupancy;
}  // namespace

cudaError_t kernel_smem(gpudb_ctx* ctx, const void* fn, size_t smem) {
  std::lock_guard<std::mutex> lk(g_attr_mu);
  size_t& have = g_smem_set[{ctx->device, fn}];
  if (smem <= have) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) have = smem;
  return e;
}

int kernel_occupancy(gpudb_ctx* ctx, const void* fn, int threads, size_t smem) {
  std::lock_guard<std::mutex> lk(g_attr_mu);
  auto it = g_occupancy.find({ctx->device, fn, threads, smem});
  if (it != g_occupancy.end()) return it->second;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess || per_sm < 1) {
    (void)cudaGetLastError();
    per_sm = 1;
  }
  g_occupancy[{ctx->device, fn, threads, smem}] = per_sm;
  return per_sm;
}

cudaEvent_t event_get(gpudb_ctx* ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

void event_put(gpudb_ctx* ctx, cudaEvent_t e) {
  if (e) ctx->event_pool.push_back(e);
}

int status_to_error(gpudb_ctx* ctx, uint32_t st) {
  if (st == 0) return GPUDB_OK;
  if (st & ST_CAPACITY)
    return fail(ctx, GPUDB_E_CAPACITY, "device status 0x%x: a hash table, partition or output buffer overflowed", st);
  if (st & ST_KEY_RANGE)
    return fail(ctx, GPUDB_E_KEY_RANGE, "device status 0x%x: a key is outside the declared key range", st);
  if (st & ST_DOMAIN)
    return fail(ctx, GPUDB_E_INVALID, "device status 0x%x: a value is outside the exact-arithmetic domain", st);
  if (st & ST_DUPLICATE)
    return fail(ctx, GPUDB_E_INVALID, "device status 0x%x: a key occurs twice on a unique build side", st);
  if (st & ST_TIMEOUT)
    return fail(ctx, GPUDB_E_TIMEOUT, "device status 0x%x: a bounded device wait ran out", st);
  return fail(ctx, GPUDB_E_CUDA, "device status 0x%x", st);
}

// ---- Call ------------------------------------------------------------------------------
Call::Call(gpudb_ctx* ctx, const gpudb_exec* ex, gpudb_timing* t)
    : ctx_(ctx), s_(ctx->stream), async_(false), t_(t), host0_(now_ms()) {
  cudaSetDevice(ctx->device);
  status_sink_ = ctx->status_sink;
  if (ex) {
    async_ = ex->async != 0;
    if (ex->stream) s_ = static_cast<cudaStream_t>(ex->stream);
  }
}

Call::~Call() {
  // a call that failed between side_begin() and side_join(): later work on its stream still
  // waits for the side stream, so scratch buffers are not reused under it
  if (side_open_) (void)side_join();
  if (!handed_off_) {
    if (slot_ >= 0) (big_ ? ctx_->big_busy : ctx_->slot_busy)[slot_] = false;
    event_put(ctx_, e0_);
    event_put(ctx_, e1_);
  }
}

int Call::begin(size_t result_bytes) {
  // a non-sticky error left by earlier, unrelated runtime calls is not this call's (a
  // sticky one still shows at this call's first launch)
  (void)cudaGetLastError();
  big_ = kSlotHeader + result_bytes > kSlotBytes;
  if (kSlotHeader + result_bytes > (big_ ? kBigSlotBytes : kSlotBytes))
    return fail(ctx_, GPUDB_E_INVALID, "result too large");
  const int n = big_ ? kBigSlots : kResultSlots;
  bool* busy = big_ ? ctx_->big_busy : ctx_->slot_busy;
  // find a free slot; if all are waiting for completion, drain the pending calls
  for (int pass = 0; pass < 2 && slot_ < 0; pass++) {
    for (int i = 0; i < n; i++) {
      int s = big_ ? i : (ctx_->next_slot + i) % n;
      if (!busy[s]) { slot_ = s; break; }
    }
    if (slot_ < 0) {
      int rc = gpudb_sync(ctx_);
      if (rc != GPUDB_OK) return rc;
    }
  }
  if (slot_ < 0) return fail(ctx_, GPUDB_E_CUDA, "no free result slot");
  busy[slot_] = true;
  if (big_) {
    dslot_ = ctx_->d_big + (size_t)slot_ * kBigSlotBytes;
    hslot_ = ctx_->h_big + (size_t)slot_ * kBigSlotBytes;
  } else {
    ctx_->next_slot = (slot_ + 1) % kResultSlots;
    dslot_ = ctx_->d_slots + (size_t)slot_ * kSlotBytes;
    hslot_ = ctx_->h_slots + (size_t)slot_ * kSlotBytes;
  }
  if (want_direct_ && !big_ && !dwork_ && ctx_->h_slots_dev)
    direct_ = ctx_->h_slots_dev + (size_t)slot_ * kSlotBytes;
  else
    GPUDB_CUDA(ctx_, cudaMemsetAsync(dslot_, 0, kSlotHeader + result_bytes, s_));
  if (t_) {
    // the timed region starts after the result slot is cleared: kernels (and copies) only
    e0_ = event_get(ctx_);
    e1_ = event_get(ctx_);
    if (!e0_ || !e1_) return fail(ctx_, GPUDB_E_CUDA, "cudaEventCreate failed");
    GPUDB_CUDA(ctx_, cudaEventRecord(e0_, s_));
  }
  return GPUDB_OK;
}

int Call::begin_direct(size_t result_bytes) {
  want_direct_ = true;
  return begin(result_bytes);
}

int Call::check_launch(const char* name) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx_, e, name);
  return GPUDB_OK;
}

int Call::side_begin() {
  if (main_) return fail(ctx_, GPUDB_E_INVALID, "side stream already in use by this call");
  GPUDB_CUDA(ctx_, cudaEventRecord(ctx_->fork_ev, s_));
  GPUDB_CUDA(ctx_, cudaStreamWaitEvent(ctx_->side_stream, ctx_->fork_ev, 0));
  main_ = s_;
  s_ = ctx_->side_stream;
  side_open_ = true;
  return GPUDB_OK;
}

void Call::side_end() {
  if (main_) {
    s_ = main_;
    main_ = nullptr;
  }
}

int Call::side_join() {
  side_end();
  side_open_ = false;
  GPUDB_CUDA(ctx_, cudaEventRecord(ctx_->join_ev, ctx_->side_stream));
  GPUDB_CUDA(ctx_, cudaStreamWaitEvent(s_, ctx_->join_ev, 0));
  return GPUDB_OK;
}

int Call::finish(size_t result_bytes, std::function<int(const uint8_t*)> convert) {
  side_end();   // (a stage that failed on the side stream may have left it selected)
  if (t_) GPUDB_CUDA(ctx_, cudaEventRecord(e1_, s_));
  size_t bytes = kSlotHeader + result_bytes;
  // (a direct result is already in hslot_ when the kernel completes; its bytes crossed the
  // link all the same)
  if (!direct_) GPUDB_CUDA(ctx_, cudaMemcpyAsync(hslot_, dslot_, bytes, cudaMemcpyDeviceToHost, s_));
  d2h_ += bytes;
  ctx_->h2d_total += h2d_;
  ctx_->d2h_total += d2h_;
  gpudb_ctx* ctx = ctx_;
  int slot = slot_;
  bool big = big_;
  uint8_t* hs = hslot_;
  gpudb_timing* t = t_;
  cudaEvent_t e0 = e0_, e1 = e1_;
  double host0 = host0_;
  uint32_t kernels = kernels_, chunks = chunks_;
  uint64_t h2d = h2d_, d2h = d2h_;
  int32_t* sink = status_sink_;
  auto done = [=]() -> int {
    uint32_t st;
    std::memcpy(&st, hs, sizeof st);
    int rc = status_to_error(ctx, st);
    if (rc == GPUDB_OK) rc = convert(hs + kSlotHeader);
    if (sink) {
      *sink = rc;
      if (ctx->on_done) ctx->on_done(ctx->on_done_arg, sink);
    }
    if (t) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) ms = -1.f;
      t->gpu_ms = ms;
      t->host_ms = now_ms() - host0;
      t->h2d_bytes = h2d;
      t->d2h_bytes = d2h;
      t->kernels = kernels;
      t->chunks = chunks;
    }
    (big ? ctx->big_busy : ctx->slot_busy)[slot] = false;
    event_put(ctx, e0);
    event_put(ctx, e1);
    return rc;
  };
  handed_off_ = true;
  if (async_) {
    cudaEvent_t ev = event_get(ctx_);
    GPUDB_CUDA(ctx_, cudaEventRecord(ev, s_));
    ctx_->pending.push_back(gpudb_ctx::Pending{ev, done});
    if (std::find(ctx_->pending_streams.begin(), ctx_->pending_streams.end(), s_) == ctx_->pending_streams.end())
      ctx_->pending_streams.push_back(s_);
    return GPUDB_OK;
  }
  cudaError_t e = cudaStreamSynchronize(s_);
  if (e != cudaSuccess) {
    done();
    return cuda_fail(ctx_, e, "cudaStreamSynchronize");
  }
  if (ctx_->pending.empty() && s_ == ctx_->stream) release_retired(ctx_);
  return done();
}

// ---- lineitem helpers --------------------------------------------------------------------
uint64_t lineitem_row_bytes(uint32_t m) {
  uint64_t b = 0;
  if (m & LI_SHIP) b += 4;
  if (m & LI_QTY) b += 4;
  if (m & LI_EXT) b += 8;
  if (m & LI_DISC) b += 4;
  if (m & LI_TAX) b += 4;
  if (m & LI_FLAG) b += 1;
  if (m & LI_STATUS) b += 1;
  if (m & LI_ORDER) b += 4;
  if (m & LI_PART) b += 4;
  if (m & LI_SUPP) b += 4;
  if (m & LI_COMMIT) b += 4;
  if (m & LI_RECEIPT) b += 4;
  if (m & LI_MODE) b += 1;
  return b;
}

int lineitem_check(gpudb_ctx* ctx, const gpudb_lineitem* li, uint32_t m) {
  if (!li) return fail(ctx, GPUDB_E_INVALID, "lineitem is NULL");
  if (li->location != GPUDB_MEM_DEVICE && li->location != GPUDB_MEM_HOST)
    return fail(ctx, GPUDB_E_INVALID, "lineitem.location must be GPUDB_MEM_DEVICE or GPUDB_MEM_HOST");
  if (li->n_rows == 0) return GPUDB_OK;
  struct { uint32_t bit; const void* p; const char* name; } cols[] = {
      {LI_SHIP, li->ship_date, "ship_date"}, {LI_QTY, li->quantity, "quantity"},
      {LI_EXT, li->ext_price, "ext_price"},  {LI_DISC, li->discount, "discount"},
      {LI_TAX, li->tax, "tax"},              {LI_FLAG, li->flag, "flag"},
      {LI_STATUS, li->status, "status"},     {LI_ORDER, li->order_key, "order_key"},
      {LI_PART, li->part_key, "part_key"},   {LI_SUPP, li->supp_key, "supp_key"},
      {LI_COMMIT, li->commit_date, "commit_date"}, {LI_RECEIPT, li->receipt_date, "receipt_date"},
      {LI_MODE, li->ship_mode, "ship_mode"}};
  for (auto& c : cols)
    if ((m & c.bit) && !c.p) return fail(ctx, GPUDB_E_INVALID, "lineitem.%s is NULL", c.name);
  return GPUDB_OK;
}

int stream_lineitem(Call& call, const gpudb_lineitem* li, uint32_t mask, uint64_t chunk_rows,
                    const std::function<int(const gpudb_lineitem&)>& dispatch) {
  gpudb_ctx* ctx = call.ctx();
  if (li->location == GPUDB_MEM_DEVICE || li->n_rows == 0) return dispatch(*li);

  if (chunk_rows == 0) chunk_rows = ctx->chunk_rows;
  chunk_rows = std::min<uint64_t>(chunk_rows, li->n_rows);
  chunk_rows = (chunk_rows + 15) & ~15ull;   // keeps every slot column 16-byte aligned
  const uint64_t row_bytes = lineitem_row_bytes(mask);

  struct Col { uint32_t bit; const void* host; size_t w; size_t off; };
  Col cols[] = {{LI_SHIP, li->ship_date, 4, 0}, {LI_QTY, li->quantity, 4, 0},
                {LI_EXT, li->ext_price, 8, 0},  {LI_DISC, li->discount, 4, 0},
                {LI_TAX, li->tax, 4, 0},        {LI_FLAG, li->flag, 1, 0},
                {LI_STATUS, li->status, 1, 0},  {LI_ORDER, li->order_key, 4, 0},
                {LI_PART, li->part_key, 4, 0},  {LI_SUPP, li->supp_key, 4, 0},
                {LI_COMMIT, li->commit_date, 4, 0}, {LI_RECEIPT, li->receipt_date, 4, 0},
                {LI_MODE, li->ship_mode, 1, 0}};
  size_t slot_bytes = 0;
  for (auto& c : cols)
    if (mask & c.bit) { c.off = slot_bytes; slot_bytes += ((chunk_rows * c.w + 255) / 256) * 256; }
  void* ring = nullptr;
  int rc = scratch(ctx, "stream.ring", slot_bytes * kStreamSlots, &ring);
  if (rc) return rc;

  cudaEvent_t copied[kStreamSlots], consumed[kStreamSlots], start = event_get(ctx);
  for (int i = 0; i < kStreamSlots; i++) { copied[i] = event_get(ctx); consumed[i] = event_get(ctx); }
  auto release = [&]() {
    for (int i = 0; i < kStreamSlots; i++) { event_put(ctx, copied[i]); event_put(ctx, consumed[i]); }
    event_put(ctx, start);
  };
  // copies start after everything already queued on the compute stream (timing events)
  cudaError_t e = cudaEventRecord(start, call.stream());
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_stream, start, 0);
  if (e != cudaSuccess) { release(); return cuda_fail(ctx, e, "stream setup"); }

  uint64_t done_rows = 0;
  int chunk = 0;
  while (done_rows < li->n_rows) {
    const uint64_t rows = std::min<uint64_t>(chunk_rows, li->n_rows - done_rows);
    const int s = chunk % kStreamSlots;
    uint8_t* base = static_cast<uint8_t*>(ring) + (size_t)s * slot_bytes;
    if (chunk >= kStreamSlots) e = cudaStreamWaitEvent(ctx->copy_stream, consumed[s], 0);
    gpudb_lineitem dev = *li;
    dev.location = GPUDB_MEM_DEVICE;
    dev.n_rows = rows;
    for (auto& c : cols) {
      if (!(mask & c.bit) || e != cudaSuccess) continue;
      void* dst = base + c.off;
      const uint8_t* src = static_cast<const uint8_t*>(c.host) + done_rows * c.w;
      e = cudaMemcpyAsync(dst, src, rows * c.w, cudaMemcpyHostToDevice, ctx->copy_stream);
      switch (c.bit) {
        case LI_SHIP: dev.ship_date = (const int32_t*)dst; break;
        case LI_QTY: dev.quantity = (const int32_t*)dst; break;
        case LI_EXT: dev.ext_price = (const int64_t*)dst; break;
        case LI_DISC: dev.discount = (const int32_t*)dst; break;
        case LI_TAX: dev.tax = (const int32_t*)dst; break;
        case LI_FLAG: dev.flag = (const uint8_t*)dst; break;
        case LI_STATUS: dev.status = (const uint8_t*)dst; break;
        case LI_ORDER: dev.order_key = (const int32_t*)dst; break;
        case LI_PART: dev.part_key = (const int32_t*)dst; break;
        case LI_SUPP: dev.supp_key = (const int32_t*)dst; break;
        case LI_COMMIT: dev.commit_date = (const int32_t*)dst; break;
        case LI_RECEIPT: dev.receipt_date = (const int32_t*)dst; break;
        case LI_MODE: dev.ship_mode = (const uint8_t*)dst; break;
      }
    }
    if (e == cudaSuccess) e = cudaEventRecord(copied[s], ctx->copy_stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(call.stream(), copied[s], 0);
    if (e != cudaSuccess) { release(); return cuda_fail(ctx, e, "chunk copy"); }
    call.add_h2d(rows * row_bytes);
    call.add_chunk();
    rc = dispatch(dev);
    if (rc != GPUDB_OK) { release(); return rc; }
    e = cudaEventRecord(consumed[s], call.stream());
    if (e != cudaSuccess) { release(); return cuda_fail(ctx, e, "chunk event"); }
    done_rows += rows;
    chunk++;
  }
  release();
  return GPUDB_OK;
}

}  // namespace gpudb

using namespace gpudb;

extern "C" {

int gpudb_abi_version(void) { return GPUDB_ABI_VERSION; }

int gpudb_create(int device, gpudb_ctx** out) {
  if (!out) return GPUDB_E_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return GPUDB_E_NODEVICE;
  if (device < 0 || device >= n) return GPUDB_E_INVALID;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return GPUDB_E_NODEVICE;
  if (prop.major != 10) return GPUDB_E_NODEVICE;   // built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return GPUDB_E_CUDA;
  gpudb_ctx* ctx = new gpudb_ctx();
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_slots, (size_t)kResultSlots * kSlotBytes);
  if (e == cudaSuccess) e = cudaHostAlloc(&ctx->h_slots, (size_t)kResultSlots * kSlotBytes, cudaHostAllocMapped);
  if (e == cudaSuccess) {
    // kernels that write a call's result straight into its host slot (Call::begin_direct)
    // need the slots' device address; without one every call copies its slot back
    void* dev = nullptr;
    if (cudaHostGetDevicePointer(&dev, ctx->h_slots, 0) == cudaSuccess) ctx->h_slots_dev = static_cast<uint8_t*>(dev);
    (void)cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_big, (size_t)kBigSlots * kBigSlotBytes);
  if (e == cudaSuccess) e = cudaHostAlloc(&ctx->h_big, (size_t)kBigSlots * kBigSlotBytes, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    gpudb_destroy(ctx);
    return e == cudaErrorMemoryAllocation ? GPUDB_E_OOM : GPUDB_E_CUDA;
  }
  *out = ctx;
  return GPUDB_OK;
}

int gpudb_destroy(gpudb_ctx* ctx) {
  if (!ctx) return GPUDB_OK;
  cudaSetDevice(ctx->device);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  if (ctx->side_stream) cudaStreamSynchronize(ctx->side_stream);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    release_retired(ctx);
    for (auto& kv : ctx->scratch)
      if (kv.second.p) cudaFreeAsync(kv.second.p, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
  }
  for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.exec);
  for (auto e : ctx->event_pool) cudaEventDestroy(e);
  if (ctx->d_slots) cudaFree(ctx->d_slots);
  if (ctx->h_slots) cudaFreeHost(ctx->h_slots);
  if (ctx->d_big) cudaFree(ctx->d_big);
  if (ctx->h_big) cudaFreeHost(ctx->h_big);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
  delete ctx;
  return GPUDB_OK;
}

const char* gpudb_last_error_string(const gpudb_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int gpudb_sync(gpudb_ctx* ctx) {
  if (!ctx) return GPUDB_E_INVALID;
  int rc = GPUDB_OK;
  // finish the calls in issue order, each as soon as its own result has arrived
  std::vector<gpudb_ctx::Pending> work;
  work.swap(ctx->pending);
  for (auto& w : work) {
    cudaError_t e = cudaEventSynchronize(w.done);
    if (e != cudaSuccess && rc == GPUDB_OK) rc = cuda_fail(ctx, e, "cudaEventSynchronize");
    event_put(ctx, w.done);
    const int r = w.finish();
    if (r != GPUDB_OK && rc == GPUDB_OK) rc = r;
  }
  for (cudaStream_t s : ctx->pending_streams) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess && rc == GPUDB_OK) rc = cuda_fail(ctx, e, "cudaStreamSynchronize");
  }
  ctx->pending_streams.clear();
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess && rc == GPUDB_OK) rc = cuda_fail(ctx, e, "cudaStreamSynchronize");
  if (rc == GPUDB_OK && ctx->pending.empty()) release_retired(ctx);
  return rc;
}

void* gpudb_stream(gpudb_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

uint64_t gpudb_kernel_launches(const gpudb_ctx* ctx) { return ctx ? ctx->launches : 0; }

int gpudb_set_option(gpudb_ctx* ctx, int32_t option, int64_t value) {
  if (!ctx) return GPUDB_E_INVALID;
  switch (option) {
    case GPUDB_OPT_CHUNK_ROWS:
      if (value < 16) return fail(ctx, GPUDB_E_INVALID, "chunk rows must be >= 16");
      ctx->chunk_rows = (uint64_t)value;
      return GPUDB_OK;
    case GPUDB_OPT_SCAN_VARIANT:
      if (value < 0 || value > 10) return fail(ctx, GPUDB_E_INVALID, "scan variant must be 0..10");
      ctx->scan_variant = (int)value;
      return GPUDB_OK;
    case GPUDB_OPT_Q6_VARIANT:
      if (value < 0 || value > 4) return fail(ctx, GPUDB_E_INVALID, "Q6 variant must be 0..4");
      ctx->q6_variant = (int)value;
      return GPUDB_OK;
    case GPUDB_OPT_HT_LOAD:
      if (value != 50 && value != 25) return fail(ctx, GPUDB_E_INVALID, "hash-table load must be 50 or 25");
      ctx->ht_shift = value == 50 ? 1 : 2;
      return GPUDB_OK;
    case GPUDB_OPT_RADIX_BITS:
      if (value != 0 && (value < 1 || value > kRadixMaxBits))
        return fail(ctx, GPUDB_E_INVALID, "radix bits must be 0 or 1..%d", (int)kRadixMaxBits);
      ctx->radix_bits = (int)value;
      return GPUDB_OK;
    case GPUDB_OPT_RADIX_SHAPE:
      if (value < 0 || value > 7) return fail(ctx, GPUDB_E_INVALID, "radix shape must be 0..7");
      ctx->radix_shape = (int)value;
      return GPUDB_OK;
    case GPUDB_OPT_Q3_AUTO_MODE:
      if (value != -1 && value != GPUDB_JOIN_GLOBAL && value != GPUDB_JOIN_RADIX && value != GPUDB_JOIN_DIRECT)
        return fail(ctx, GPUDB_E_INVALID, "Q3 AUTO mode must be -1 or a join mode (global, radix, direct)");
      ctx->q3_auto_mode = (int)value;
      return GPUDB_OK;
    case GPUDB_OPT_GRAPHS:
      if (value != 0 && value != 1) return fail(ctx, GPUDB_E_INVALID, "graphs option must be 0 or 1");
      ctx->use_graphs = value != 0;
      return GPUDB_OK;
    case GPUDB_OPT_Q9_SMEM_SLOTS:
    case GPUDB_OPT_Q9_GLOBAL_SLOTS:
      if (value < 32 || value > 8192 || (value & (value - 1)))
        return fail(ctx, GPUDB_E_INVALID, "Q9 slots must be a power of two in 32..8192");
      (option == GPUDB_OPT_Q9_SMEM_SLOTS ? ctx->q9_smem_slots : ctx->q9_global_slots) = (int)value;
      return GPUDB_OK;
    default:
      return fail(ctx, GPUDB_E_INVALID, "unknown option %d", option);
  }
}

int gpudb_get_option(const gpudb_ctx* ctx, int32_t option, int64_t* value) {
  if (!ctx || !value) return GPUDB_E_INVALID;
  switch (option) {
    case GPUDB_OPT_CHUNK_ROWS: *value = (int64_t)ctx->chunk_rows; return GPUDB_OK;
    case GPUDB_OPT_SCAN_VARIANT: *value = ctx->scan_variant; return GPUDB_OK;
    case GPUDB_OPT_Q6_VARIANT: *value = ctx->q6_variant; return GPUDB_OK;
    case GPUDB_OPT_HT_LOAD: *value = ctx->ht_shift == 1 ? 50 : 25; return GPUDB_OK;
    case GPUDB_OPT_RADIX_BITS: *value = ctx->radix_bits; return GPUDB_OK;
    case GPUDB_OPT_Q9_SMEM_SLOTS: *value = ctx->q9_smem_slots; return GPUDB_OK;
    case GPUDB_OPT_Q9_GLOBAL_SLOTS: *value = ctx->q9_global_slots; return GPUDB_OK;
    case GPUDB_OPT_GRAPHS: *value = ctx->use_graphs ? 1 : 0; return GPUDB_OK;
    case GPUDB_OPT_Q3_AUTO_MODE: *value = ctx->q3_auto_mode; return GPUDB_OK;
    case GPUDB_OPT_RADIX_SHAPE: *value = ctx->radix_shape; return GPUDB_OK;
    default: return GPUDB_E_INVALID;
  }
}

int gpudb_device_alloc(gpudb_ctx* ctx, size_t bytes, void** out) {
  if (!ctx || !out) return GPUDB_E_INVALID;
  GPUDB_CUDA(ctx, cudaMalloc(out, bytes ? bytes : 1));
  return GPUDB_OK;
}

int gpudb_device_free(gpudb_ctx* ctx, void* p) {
  if (!ctx) return GPUDB_E_INVALID;
  if (p) GPUDB_CUDA(ctx, cudaFree(p));
  return GPUDB_OK;
}

int gpudb_host_alloc(gpudb_ctx* ctx, size_t bytes, void** out) {
  if (!ctx || !out) return GPUDB_E_INVALID;
  GPUDB_CUDA(ctx, cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault));
  return GPUDB_OK;
}

int gpudb_host_free(gpudb_ctx* ctx, void* p) {
  if (!ctx) return GPUDB_E_INVALID;
  if (p) GPUDB_CUDA(ctx, cudaFreeHost(p));
  return GPUDB_OK;
}

int gpudb_copy(gpudb_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (!ctx || (!dst && bytes) || (!src && bytes)) return GPUDB_E_INVALID;
  if (!bytes) return GPUDB_OK;
  GPUDB_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
  GPUDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GPUDB_OK;
}

}  // extern "C"
