// Host infrastructure of the command-line drivers, over the C ABI only.
//
// Mirrors the reference's src/infra.h: buffers (newBuffer / createFilledBuffer /
// createBitmapBuffer / releaseAll, src/infra.h:173-229,499-531) become RAII DeviceBuffer /
// HostBuffer; the .tbl loaders (src/infra.h:262-361) become the seeded generator, or with
// --data the GPU text loader (load_tbl, gpudb_tbl_parse); the
// chunk configuration (src/infra.h:42-57) becomes gpudb_set_option(GPUDB_OPT_CHUNK_ROWS);
// printTimingSummary (src/infra.h:511-516) keeps its exact text so the reference's
// harness (scripts/benchmark_gpu.sh:50-60) parses our output unchanged.
#pragma once
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "gpudb_capi.h"

namespace gpudb_host {

inline double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

[[noreturn]] inline void die(gpudb_ctx* ctx, const char* what, int rc) {
  std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, ctx ? gpudb_last_error_string(ctx) : "");
  std::exit(2);
}

inline void check(gpudb_ctx* ctx, int rc, const char* what) {
  if (rc != GPUDB_OK) die(ctx, what, rc);
}

// Device (HBM) or pinned-host buffer owned by the driver.
class Buffer {
 public:
  Buffer() = default;
  Buffer(gpudb_ctx* ctx, size_t bytes, int location) : ctx_(ctx), loc_(location), bytes_(bytes) {
    int rc = loc_ == GPUDB_MEM_DEVICE ? gpudb_device_alloc(ctx_, bytes ? bytes : 1, &p_)
                                      : gpudb_host_alloc(ctx_, bytes ? bytes : 1, &p_);
    check(ctx_, rc, "allocation");
  }
  Buffer(const Buffer&) = delete;
  Buffer& operator=(const Buffer&) = delete;
  Buffer(Buffer&& o) noexcept { *this = std::move(o); }
  Buffer& operator=(Buffer&& o) noexcept {
    release();
    ctx_ = o.ctx_; p_ = o.p_; loc_ = o.loc_; bytes_ = o.bytes_;
    o.p_ = nullptr;
    return *this;
  }
  ~Buffer() { release(); }
  template <class T> T* as() const { return static_cast<T*>(p_); }
  size_t bytes() const { return bytes_; }

 private:
  void release() {
    if (p_) {
      if (loc_ == GPUDB_MEM_DEVICE) gpudb_device_free(ctx_, p_);
      else gpudb_host_free(ctx_, p_);
      p_ = nullptr;
    }
  }
  gpudb_ctx* ctx_ = nullptr;
  void* p_ = nullptr;
  int loc_ = GPUDB_MEM_DEVICE;
  size_t bytes_ = 0;
};

// Table sizes of one scale name (sf1 / sf10 / sf100), as in BASELINE's configs.
struct Scale {
  std::string name;
  uint64_t lineitem, customer, orders, part, supplier;
  bool streamed;   // lineitem lives in pinned host memory and streams in chunks
};

inline Scale scale_of(const std::string& name, double factor) {
  Scale s;
  s.name = name;
  double base = name == "sf100" ? 100 : name == "sf10" ? 10 : 1;
  auto n = [&](double per_sf) { return (uint64_t)(per_sf * base * factor + 0.5); };
  s.lineitem = n(6e6);
  s.customer = n(150e3);
  s.orders = n(1.5e6);
  s.part = n(200e3);
  s.supplier = (n(10e3) / 4) * 4;
  if (s.supplier < 4) s.supplier = 4;
  s.streamed = name == "sf100";
  return s;
}

// One generated column of `rows` rows starting at `offset`.
inline Buffer generate(gpudb_ctx* ctx, const gpudb_gen_spec& base, int32_t column, int location) {
  const int w = gpudb_column_width(column);
  Buffer b(ctx, (size_t)base.n_rows * w, location);
  check(ctx, gpudb_generate(ctx, &base, column, b.as<void>(), location), "gpudb_generate");
  return b;
}

inline void printTimingSummary(double parseMs, double gpuMs, double postMs) {
  std::printf("  CPU Parsing (.tbl): %10.2f ms\n", parseMs);
  std::printf("  GPU Execution:      %10.2f ms\n", gpuMs);
  std::printf("  CPU Post Process:   %10.2f ms\n", postMs);
  std::printf("  Total Execution:    %10.2f ms  (GPU + CPU post)\n", gpuMs + postMs);
}

// Signed 128-bit value -> decimal text.
inline std::string i128_str(const gpudb_i128& v) {
  __int128 x = ((__int128)v.hi << 64) | (__int128)v.lo;
  bool neg = x < 0;
  unsigned __int128 u = neg ? (unsigned __int128)(-x) : (unsigned __int128)x;
  std::string s;
  do { s.insert(s.begin(), char('0' + (int)(u % 10))); u /= 10; } while (u);
  return neg ? "-" + s : s;
}

struct RunOptions {
  Scale scale;
  uint64_t seed = 42;
  int reps = 3;             // the reference times the third of three runs
  std::string data_dir;     // non-empty: tables come from <data_dir>/<table>.tbl (dbgen text)
  size_t tbl_piece = (size_t)1 << 30;   // bytes of text read and parsed at a time
};

// One table read from dbgen text: device columns in gpudb_tbl_parse's order for its kind
// (only the requested ones are kept), the row count and the int32 columns' largest values.
struct TblTable {
  std::vector<Buffer> cols;
  uint64_t rows = 0;
  int32_t col_max[GPUDB_TBL_MAX_COLS];
  template <class T> T* col(int i) const { return cols[i].bytes() ? cols[i].template as<T>() : nullptr; }
};

// Reads `dir`/`name`.tbl in pieces of about `piece` bytes that end at a line end, through
// one pinned host buffer, and parses every piece on the GPU straight into the columns at its
// row offset (a first pass counts the rows). `keep` marks the columns to store; `widths` are
// their element sizes. The reference's equivalent is loadColumnsMulti (src/infra.h:262-361).
inline TblTable load_tbl(gpudb_ctx* ctx, const std::string& dir, const char* name, int32_t table,
                         const std::vector<int>& keep, const std::vector<int>& widths,
                         size_t piece = (size_t)1 << 30) {
  const std::string path = dir + "/" + name + ".tbl";
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    std::fprintf(stderr, "Cannot open: %s\n", path.c_str());
    std::exit(1);
  }
  Buffer host(ctx, piece + 1, GPUDB_MEM_HOST);
  char* buf = host.as<char>();
  // visits the file as pieces that end at a newline (or at the end of the file)
  auto pieces = [&](const std::function<void(const char*, size_t)>& fn) {
    std::fseek(f, 0, SEEK_SET);
    size_t carry = 0;
    for (;;) {
      const size_t got = std::fread(buf + carry, 1, piece - carry, f);
      const size_t have = carry + got;
      if (have == 0) break;
      size_t cut = have;
      if (got != 0 && have == piece) {
        while (cut > 0 && buf[cut - 1] != '\n') cut--;
        if (cut == 0) {
          std::fprintf(stderr, "%s: a line longer than %zu bytes\n", path.c_str(), piece);
          std::exit(1);
        }
      }
      fn(buf, cut);
      carry = have - cut;
      std::memmove(buf, buf + cut, carry);
      if (got == 0) break;   // the last piece (carry is 0: at the end of the file nothing is cut)
    }
  };
  TblTable t;
  pieces([&](const char* p, size_t n) {
    uint64_t r = 0;
    check(ctx, gpudb_tbl_count_rows(ctx, p, n, GPUDB_MEM_HOST, &r), "gpudb_tbl_count_rows");
    t.rows += r;
  });
  const std::vector<int>& k = keep;
  const std::vector<int>& w = widths;
  t.cols.resize(GPUDB_TBL_MAX_COLS);
  for (size_t i = 0; i < k.size(); i++) t.cols[k[i]] = Buffer(ctx, t.rows * (size_t)w[i], GPUDB_MEM_DEVICE);
  for (int i = 0; i < GPUDB_TBL_MAX_COLS; i++) t.col_max[i] = INT32_MIN;
  uint64_t done = 0;
  pieces([&](const char* p, size_t n) {
    void* cols[GPUDB_TBL_MAX_COLS] = {};
    for (size_t i = 0; i < k.size(); i++) cols[k[i]] = t.cols[k[i]].as<uint8_t>() + done * (size_t)w[i];
    uint64_t r = 0;
    int32_t mx[GPUDB_TBL_MAX_COLS];
    check(ctx, gpudb_tbl_parse(ctx, table, p, n, GPUDB_MEM_HOST, cols, t.rows - done, &r, mx, nullptr),
          "gpudb_tbl_parse");
    for (int i = 0; i < GPUDB_TBL_MAX_COLS; i++) t.col_max[i] = std::max(t.col_max[i], mx[i]);
    done += r;
  });
  std::fclose(f);
  return t;
}

using Driver = void (*)(gpudb_ctx*, const RunOptions&);

void runQ1Benchmark(gpudb_ctx*, const RunOptions&);
void runQ3Benchmark(gpudb_ctx*, const RunOptions&);
void runQ4Benchmark(gpudb_ctx*, const RunOptions&);
void runQ5Benchmark(gpudb_ctx*, const RunOptions&);
void runQ7Benchmark(gpudb_ctx*, const RunOptions&);
void runQ8Benchmark(gpudb_ctx*, const RunOptions&);
void runQ10Benchmark(gpudb_ctx*, const RunOptions&);
void runQ12Benchmark(gpudb_ctx*, const RunOptions&);
void runQ13Benchmark(gpudb_ctx*, const RunOptions&);
void runQ6Benchmark(gpudb_ctx*, const RunOptions&);
void runQ9Benchmark(gpudb_ctx*, const RunOptions&);
void runSelectionBenchmark(gpudb_ctx*, const RunOptions&);
void runAggregationBenchmark(gpudb_ctx*, const RunOptions&);
void runJoinBenchmark(gpudb_ctx*, const RunOptions&);

}  // namespace gpudb_host
