// .tbl text loader on the GPU: dbgen-style rows ('|'-separated fields, one row per line)
// parsed straight into the engine's columns. Replaces the reference's host-side parsing
// (MappedFile + countLines + buildLineIndex + parse*ColumnChunk, src/infra.h:60-171, and
// loadColumnsMulti, src/infra.h:262-361), which dominates its run time (8-500 s per table).
//
// Three phases, all on the device:
//  1. newline_count_kernel: newlines per 16 KB tile of the text (128-bit loads);
//  2. exclusive_scan of the tile counts, then newline_write_kernel: every tile writes the
//     start offsets of the lines that begin in it, in order (block prefix sum), so
//     starts[r] is where row r begins;
//  3. parse_kernel<table>: one thread per row walks its fields, parses the ones the table
//     keeps and writes them to the columns; any malformed field sets a status bit, and the
//     largest value of every int32 column is kept (key bounds for bitmaps and maps).
// Encodings: integers as int32; decimals (at most two fraction digits) as hundredths; dates
// "YYYY-MM-DD" as days since 1992-01-01 (days_from_civil, the proleptic Gregorian day count
// published by H. Hinnant); return flag A/N/R -> 0/1/2; line status F/O -> 0/1; market
// segment AUTOMOBILE/BUILDING/FURNITURE/HOUSEHOLD/MACHINERY -> 0..4; part name -> 1 if it
// contains "green" (the Q9 part filter), else 0.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "scan.cuh"

namespace gpudb {
namespace {

constexpr int kTT = 256;                              // threads per tile
constexpr uint64_t kTileBytes = (uint64_t)kTT * 64;   // 64 bytes per thread

enum FieldType : int32_t {
  F_I32, F_DEC64, F_DEC32, F_QTY, F_DATE, F_RETFLAG, F_LINESTATUS, F_SEGMENT, F_GREEN, F_U8, F_SHIPMODE, F_PRIORITY,
  F_COMMENT, F_PTYPE
};

struct TblSpec {
  int32_t n;                                  // columns kept
  int32_t field[GPUDB_TBL_MAX_COLS];          // dbgen field index of each, ascending
  int32_t type[GPUDB_TBL_MAX_COLS];
  void* col[GPUDB_TBL_MAX_COLS];              // device column (null = parse, keep nothing)
};

bool spec_for(int32_t table, TblSpec* s) {
  static const struct { int32_t table, n, field[GPUDB_TBL_MAX_COLS], type[GPUDB_TBL_MAX_COLS]; } specs[] = {
      {GPUDB_TBL_LINEITEM, 13, {0, 1, 2, 4, 5, 6, 7, 8, 9, 10, 11, 12, 14},
       {F_I32, F_I32, F_I32, F_QTY, F_DEC64, F_DEC32, F_DEC32, F_RETFLAG, F_LINESTATUS, F_DATE, F_DATE, F_DATE,
        F_SHIPMODE}},
      {GPUDB_TBL_ORDERS, 5, {0, 1, 4, 5, 8}, {F_I32, F_I32, F_DATE, F_PRIORITY, F_COMMENT}},
      {GPUDB_TBL_CUSTOMER, 3, {0, 3, 6}, {F_I32, F_U8, F_SEGMENT}},
      {GPUDB_TBL_PART, 3, {0, 1, 4}, {F_I32, F_GREEN, F_PTYPE}},
      {GPUDB_TBL_SUPPLIER, 2, {0, 3}, {F_I32, F_U8}},
      {GPUDB_TBL_PARTSUPP, 3, {0, 1, 3}, {F_I32, F_I32, F_DEC64}},
  };
  for (const auto& e : specs)
    if (e.table == table) {
      std::memset(s, 0, sizeof *s);
      s->n = e.n;
      for (int i = 0; i < e.n; i++) { s->field[i] = e.field[i]; s->type[i] = e.type[i]; }
      return true;
    }
  return false;
}

__global__ void __launch_bounds__(kTT) newline_count_kernel(const uint8_t* __restrict__ text, uint64_t bytes,
                                                            uint32_t* counts) {
  const uint64_t b0 = (uint64_t)blockIdx.x * kTileBytes + (uint64_t)threadIdx.x * 64;
  uint32_t c = 0;
  if (b0 + 64 <= bytes) {
    const uint4* p = reinterpret_cast<const uint4*>(text + b0);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint4 v = __ldcs(p + k);
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int j = 0; j < 4; j++) {
        // bytes equal to '\n' (0x0A): the classic "has zero byte" test on w ^ 0x0A0A0A0A
        const uint32_t x = w[j] ^ 0x0A0A0A0Au;
        c += __popc((x - 0x01010101u) & ~x & 0x80808080u);
      }
    }
  } else {
    for (uint64_t i = b0; i < bytes && i < b0 + 64; i++) c += text[i] == '\n';
  }
  __shared__ uint32_t red[kTT / 32];
  c = __reduce_add_sync(FULL_MASK, c);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int w = 0; w < kTT / 32; w++) s += red[w];
    counts[blockIdx.x] = s;
  }
}

// starts[0] = 0; starts[1 + k] = offset after the k-th newline of the text.
__global__ void __launch_bounds__(kTT) newline_write_kernel(const uint8_t* __restrict__ text, uint64_t bytes,
                                                            const uint32_t* __restrict__ offs, uint64_t* starts) {
  __shared__ uint32_t warp_tot[kTT / 32];
  const uint64_t b0 = (uint64_t)blockIdx.x * kTileBytes + (uint64_t)threadIdx.x * 64;
  uint8_t buf[64];
  const uint64_t n = b0 < bytes ? (bytes - b0 < 64 ? bytes - b0 : 64) : 0;
  if (n == 64) {
    const uint4* p = reinterpret_cast<const uint4*>(text + b0);
#pragma unroll
    for (int k = 0; k < 4; k++) *reinterpret_cast<uint4*>(buf + 16 * k) = __ldcs(p + k);
  } else {
    for (uint64_t i = 0; i < 64; i++) buf[i] = i < n ? text[b0 + i] : 0;
  }
  uint32_t c = 0;
#pragma unroll
  for (int i = 0; i < 64; i++) c += buf[i] == '\n';
  const uint32_t inc = block_inclusive_scan<uint32_t>(c, warp_tot);
  uint64_t at = 1 + (uint64_t)offs[blockIdx.x] + (inc - c);
#pragma unroll
  for (int i = 0; i < 64; i++)
    if (buf[i] == '\n') starts[at++] = b0 + i + 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) starts[0] = 0;
}

// Days since 1992-01-01 of a proleptic Gregorian date (days_from_civil).
__device__ __forceinline__ int32_t days_since_1992(int32_t y, int32_t m, int32_t d) {
  y -= m <= 2;
  const int32_t era = (y >= 0 ? y : y - 399) / 400;
  const int32_t yoe = y - era * 400;
  const int32_t doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5 + d - 1;
  const int32_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + doe - 719468 - 8035;   // 8035 = days from 1970-01-01 to 1992-01-01
}

__device__ __forceinline__ bool parse_int(const uint8_t* s, const uint8_t* e, int64_t lim, int64_t* out) {
  bool neg = false;
  if (s < e && *s == '-') { neg = true; s++; }
  if (s == e) return false;
  int64_t v = 0;
  for (; s < e; s++) {
    if (*s < '0' || *s > '9') return false;
    v = v * 10 + (*s - '0');
    if (v > lim) return false;
  }
  *out = neg ? -v : v;
  return true;
}

// Decimal with at most two fraction digits -> hundredths.
__device__ __forceinline__ bool parse_dec(const uint8_t* s, const uint8_t* e, int64_t* out) {
  const uint8_t* dot = s;
  while (dot < e && *dot != '.') dot++;
  int64_t ip;
  const bool neg = s < e && *s == '-';
  if (!parse_int(s, dot, (1ll << 55), &ip)) return false;
  int64_t frac = 0;
  if (dot < e) {
    const int nd = (int)(e - dot - 1);
    if (nd < 1 || nd > 2) return false;
    for (const uint8_t* p = dot + 1; p < e; p++) {
      if (*p < '0' || *p > '9') return false;
      frac = frac * 10 + (*p - '0');
    }
    if (nd == 1) frac *= 10;
  }
  const int64_t mag = (neg ? -ip : ip) * 100 + frac;
  *out = neg ? -mag : mag;
  return true;
}

__device__ __forceinline__ bool field_equals(const uint8_t* s, const uint8_t* e, const char* w) {
  for (; *w; w++, s++)
    if (s == e || *s != (uint8_t)*w) return false;
  return s == e;
}

// Position of [s, e) in the n words of `words` (separated by '|'), or -1.
__device__ __forceinline__ int word_index(const uint8_t* s, const uint8_t* e, const char* words) {
  int i = 0;
  const char* w = words;
  while (*w) {
    const uint8_t* p = s;
    const char* q = w;
    while (*q && *q != '|' && p < e && *p == (uint8_t)*q) { p++; q++; }
    if (p == e && (*q == '|' || *q == 0)) return i;
    while (*q && *q != '|') q++;
    if (*q == '|') q++;
    w = q;
    i++;
  }
  return -1;
}

// p_type "S1 S2 S3" -> s1 * 25 + s2 * 5 + s3 (the syllable lists of the TPC-H part types), or -1.
__device__ int part_type_code(const uint8_t* s, const uint8_t* e) {
  const uint8_t* a = s;
  while (a < e && *a != ' ') a++;
  if (a >= e) return -1;
  const uint8_t* b = a + 1;
  while (b < e && *b != ' ') b++;
  if (b >= e) return -1;
  const int i1 = word_index(s, a, "STANDARD|SMALL|MEDIUM|LARGE|ECONOMY|PROMO");
  const int i2 = word_index(a + 1, b, "ANODIZED|BURNISHED|PLATED|POLISHED|BRUSHED");
  const int i3 = word_index(b + 1, e, "TIN|NICKEL|BRASS|STEEL|COPPER");
  return (i1 < 0 || i2 < 0 || i3 < 0) ? -1 : i1 * 25 + i2 * 5 + i3;
}

template <int MAXF>
__global__ void __launch_bounds__(256) parse_kernel(const uint8_t* __restrict__ text, uint64_t bytes,
                                                    const uint64_t* __restrict__ starts, const uint32_t* __restrict__ n_lines_p,
                                                    TblSpec spec, uint64_t capacity, uint8_t* res, uint32_t* status) {
  const uint64_t n_lines = *n_lines_p;
  const bool tail = starts[n_lines] < bytes;   // text after the last newline is one more row
  const uint64_t n_rows = n_lines + (tail ? 1 : 0);
  if (blockIdx.x == 0 && threadIdx.x == 0) *reinterpret_cast<unsigned long long*>(res) = n_rows;
  uint32_t* col_max = reinterpret_cast<uint32_t*>(res + 8);   // biased: value ^ 0x80000000
  uint32_t local_max[GPUDB_TBL_MAX_COLS];
#pragma unroll
  for (int c = 0; c < GPUDB_TBL_MAX_COLS; c++) local_max[c] = 0;
  uint32_t bad = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += stride) {
    if (r >= capacity) { bad |= ST_CAPACITY; continue; }
    const uint8_t* s = text + starts[r];
    const uint8_t* end = text + (r < n_lines ? starts[r + 1] - 1 : bytes);
    if (end > s && end[-1] == '\r') end--;
    int f = 0, k = 0;
    while (k < spec.n) {
      const uint8_t* fe = s;
      while (fe < end && *fe != '|') fe++;
      if (fe == end && f < spec.field[spec.n - 1]) { bad |= ST_DOMAIN; break; }   // too few fields
      if (f == spec.field[k]) {
        int64_t v = 0;
        bool ok = true;
        switch (spec.type[k]) {
          case F_I32: ok = parse_int(s, fe, 0x7FFFFFFFll, &v); break;
          case F_U8: ok = parse_int(s, fe, 255, &v) && v >= 0; break;
          case F_DEC64: ok = parse_dec(s, fe, &v); break;
          case F_DEC32: ok = parse_dec(s, fe, &v) && v >= INT32_MIN && v <= INT32_MAX; break;
          case F_QTY: ok = parse_dec(s, fe, &v) && v % 100 == 0 && v / 100 <= INT32_MAX && v / 100 >= INT32_MIN; v /= 100; break;
          case F_DATE: {
            ok = fe - s == 10 && s[4] == '-' && s[7] == '-';
            int64_t y = 0, m = 0, d = 0;
            ok = ok && parse_int(s, s + 4, 9999, &y) && parse_int(s + 5, s + 7, 12, &m) && parse_int(s + 8, s + 10, 31, &d) &&
                 m >= 1 && d >= 1;
            if (ok) v = days_since_1992((int32_t)y, (int32_t)m, (int32_t)d);
            break;
          }
          case F_RETFLAG:
            ok = fe - s == 1 && (*s == 'A' || *s == 'N' || *s == 'R');
            v = !ok ? 0 : *s == 'A' ? 0 : *s == 'N' ? 1 : 2;
            break;
          case F_LINESTATUS:
            ok = fe - s == 1 && (*s == 'F' || *s == 'O');
            v = ok && *s == 'O' ? 1 : 0;
            break;
          case F_SEGMENT:
            v = field_equals(s, fe, "AUTOMOBILE") ? 0 : field_equals(s, fe, "BUILDING") ? 1
                : field_equals(s, fe, "FURNITURE") ? 2 : field_equals(s, fe, "HOUSEHOLD") ? 3
                : field_equals(s, fe, "MACHINERY") ? 4 : -1;
            ok = v >= 0;
            break;
          case F_SHIPMODE:   // alphabetical codes: ORDER BY l_shipmode
            v = field_equals(s, fe, "AIR") ? 0 : field_equals(s, fe, "FOB") ? 1 : field_equals(s, fe, "MAIL") ? 2
                : field_equals(s, fe, "RAIL") ? 3 : field_equals(s, fe, "REG AIR") ? 4
                : field_equals(s, fe, "SHIP") ? 5 : field_equals(s, fe, "TRUCK") ? 6 : -1;
            ok = v >= 0;
            break;
          case F_PRIORITY:   // "1-URGENT" .. "5-LOW": the leading digit
            ok = fe - s >= 2 && *s >= '1' && *s <= '5' && s[1] == '-';
            v = ok ? *s - '0' : 0;
            break;
          case F_COMMENT: {   // at most 79 bytes, copied into a NUL-padded slot
            ok = fe - s < GPUDB_COMMENT_WIDTH;
            if (ok && spec.col[k]) {
              char* d = static_cast<char*>(spec.col[k]) + r * GPUDB_COMMENT_WIDTH;
              int i = 0;
              for (const uint8_t* p = s; p < fe; p++) d[i++] = (char)*p;
              for (; i < GPUDB_COMMENT_WIDTH; i++) d[i] = 0;
            }
            break;
          }
          case F_PTYPE:
            v = part_type_code(s, fe);
            ok = v >= 0;
            break;
          case F_GREEN: {
            v = 0;
            for (const uint8_t* p = s; p + 5 <= fe && !v; p++)
              v = p[0] == 'g' && p[1] == 'r' && p[2] == 'e' && p[3] == 'e' && p[4] == 'n';
            break;
          }
        }
        if (!ok) bad |= ST_DOMAIN;
        void* col = spec.type[k] == F_COMMENT ? nullptr : spec.col[k];   // comments are written above
        if (col) {
          switch (spec.type[k]) {
            case F_DEC64: static_cast<int64_t*>(col)[r] = v; break;
            case F_RETFLAG: case F_LINESTATUS: case F_SEGMENT: case F_GREEN: case F_U8: case F_SHIPMODE:
            case F_PRIORITY: case F_PTYPE:
              static_cast<uint8_t*>(col)[r] = (uint8_t)v; break;
            default: static_cast<int32_t*>(col)[r] = (int32_t)v; break;
          }
        }
        if (spec.type[k] == F_I32 || spec.type[k] == F_DATE || spec.type[k] == F_QTY || spec.type[k] == F_DEC32) {
          const uint32_t b = (uint32_t)(int32_t)v ^ 0x80000000u;
#pragma unroll
          for (int c = 0; c < GPUDB_TBL_MAX_COLS; c++)
            if (c == k) local_max[c] = max(local_max[c], b);
        }
        k++;
      }
      if (fe == end) break;
      s = fe + 1;
      f++;
    }
    if (k < spec.n) bad |= ST_DOMAIN;
  }
#pragma unroll
  for (int c = 0; c < GPUDB_TBL_MAX_COLS; c++) {
    const uint32_t m = __reduce_max_sync(FULL_MASK, local_max[c]);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(col_max + c, m);
  }
  bad = __reduce_or_sync(FULL_MASK, bad);
  if ((threadIdx.x & 31) == 0 && bad) set_status(status, bad);
}

// Text on the device (copied there when it lives in host memory), line index built.
int index_lines(Call& call, const char* text, uint64_t bytes, int32_t location, const uint8_t** dtext,
                uint64_t** starts, uint32_t** n_lines) {
  gpudb_ctx* ctx = call.ctx();
  cudaStream_t s = call.stream();
  const uint64_t tiles = std::max<uint64_t>(1, (bytes + kTileBytes - 1) / kTileBytes);
  void *tbuf = nullptr, *sbuf = nullptr, *cbuf = nullptr;
  int rc = GPUDB_OK;
  if (location == GPUDB_MEM_HOST) {
    rc = scratch(ctx, "tbl.text", bytes + 64, &tbuf);
    if (rc) return rc;
    GPUDB_CUDA(ctx, cudaMemcpyAsync(tbuf, text, bytes, cudaMemcpyHostToDevice, s));
    call.add_h2d(bytes);
    *dtext = static_cast<const uint8_t*>(tbuf);
  } else {
    *dtext = reinterpret_cast<const uint8_t*>(text);
  }
  const uint64_t stmp = scan_tiles_count(tiles) + 8;
  if ((rc = scratch(ctx, "tbl.counts", (tiles * 2 + stmp + 8) * 4, &cbuf))) return rc;
  uint32_t* counts = static_cast<uint32_t*>(cbuf);
  uint32_t* offs = counts + tiles;
  uint32_t* total = offs + tiles;
  uint32_t* tmp = total + 4;
  GPUDB_LAUNCH(call, newline_count_kernel, (unsigned)tiles, kTT, 0, *dtext, bytes, counts);
  rc = exclusive_scan<uint32_t, uint32_t>(call, counts, tiles, offs, tmp, total);
  if (rc) return rc;
  // the line index is sized from the newline count (one read-back; a pageable copy waits)
  uint32_t lines = 0;
  GPUDB_CUDA(ctx, cudaMemcpyAsync(&lines, total, 4, cudaMemcpyDeviceToHost, s));
  GPUDB_CUDA(ctx, cudaStreamSynchronize(s));
  if ((rc = scratch(ctx, "tbl.starts", ((uint64_t)lines + 2) * 8, &sbuf))) return rc;
  GPUDB_LAUNCH(call, newline_write_kernel, (unsigned)tiles, kTT, 0, *dtext, bytes, (const uint32_t*)offs,
               static_cast<uint64_t*>(sbuf));
  *starts = static_cast<uint64_t*>(sbuf);
  *n_lines = total;
  return GPUDB_OK;
}

int check_text(gpudb_ctx* ctx, const char* text, uint64_t bytes, int32_t location) {
  if (bytes && !text) return fail(ctx, GPUDB_E_INVALID, "tbl: text is NULL");
  if (location != GPUDB_MEM_HOST && location != GPUDB_MEM_DEVICE) return fail(ctx, GPUDB_E_INVALID, "tbl: bad location");
  if (location == GPUDB_MEM_DEVICE && (reinterpret_cast<uintptr_t>(text) & 15u))
    return fail(ctx, GPUDB_E_INVALID, "tbl: device text must be 16-byte aligned");
  if (bytes >= (1ull << 36)) return fail(ctx, GPUDB_E_INVALID, "tbl: at most 64 GB of text per call");
  if (bytes / kTileBytes >= (1ull << 31)) return fail(ctx, GPUDB_E_INVALID, "tbl: text too large");
  return GPUDB_OK;
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_tbl_count_rows(gpudb_ctx* ctx, const char* text, uint64_t bytes, int32_t location,
                                    uint64_t* n_rows) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!n_rows) return fail(ctx, GPUDB_E_INVALID, "tbl: n_rows is required");
  int rc = check_text(ctx, text, bytes, location);
  if (rc) return rc;
  *n_rows = 0;
  if (bytes == 0) return GPUDB_OK;
  Call call(ctx, nullptr, nullptr);
  if ((rc = call.begin(16))) return rc;
  const uint8_t* dtext;
  uint64_t* starts;
  uint32_t* n_lines;
  if ((rc = index_lines(call, text, bytes, location, &dtext, &starts, &n_lines))) return rc;
  // rows = newlines, plus one if text follows the last newline
  uint8_t last = 0;
  GPUDB_CUDA(ctx, cudaMemcpyAsync(call.result<uint8_t>(), n_lines, 4, cudaMemcpyDeviceToDevice, call.stream()));
  GPUDB_CUDA(ctx, cudaMemcpyAsync(&last, dtext + bytes - 1, 1, cudaMemcpyDeviceToHost, call.stream()));
  return call.finish(16, [n_rows, &last](const uint8_t* h) {
    uint32_t n;
    std::memcpy(&n, h, 4);
    *n_rows = (uint64_t)n + (last != '\n' ? 1 : 0);
    return GPUDB_OK;
  });
}

extern "C" int gpudb_tbl_parse(gpudb_ctx* ctx, int32_t table, const char* text, uint64_t bytes, int32_t location,
                               void* const* cols, uint64_t capacity, uint64_t* n_rows, int32_t* col_max,
                               gpudb_timing* t) {
  if (!ctx) return GPUDB_E_INVALID;
  TblSpec spec;
  if (!spec_for(table, &spec)) return fail(ctx, GPUDB_E_INVALID, "tbl: unknown table %d", table);
  if (!n_rows) return fail(ctx, GPUDB_E_INVALID, "tbl: n_rows is required");
  int rc = check_text(ctx, text, bytes, location);
  if (rc) return rc;
  for (int i = 0; i < spec.n; i++) spec.col[i] = cols ? cols[i] : nullptr;
  *n_rows = 0;
  if (col_max)
    for (int i = 0; i < GPUDB_TBL_MAX_COLS; i++) col_max[i] = INT32_MIN;
  if (bytes == 0) return GPUDB_OK;
  Call call(ctx, nullptr, t);
  const size_t rbytes = 8 + GPUDB_TBL_MAX_COLS * 4;
  if ((rc = call.begin(rbytes))) return rc;
  const uint8_t* dtext;
  uint64_t* starts;
  uint32_t* n_lines;
  if ((rc = index_lines(call, text, bytes, location, &dtext, &starts, &n_lines))) return rc;
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(bytes / 64 / 256 + 1, (uint64_t)ctx->sm_count * 8));
  GPUDB_LAUNCH(call, parse_kernel<GPUDB_TBL_MAX_COLS>, grid, 256, 0, dtext, bytes, (const uint64_t*)starts,
               (const uint32_t*)n_lines, spec, capacity, call.result<uint8_t>(), call.status());
  return call.finish(rbytes, [n_rows, col_max, spec](const uint8_t* h) {
    unsigned long long n;
    std::memcpy(&n, h, 8);
    *n_rows = n;
    if (col_max)
      for (int i = 0; i < GPUDB_TBL_MAX_COLS; i++) {
        uint32_t b;
        std::memcpy(&b, h + 8 + 4 * i, 4);
        const bool int_col = i < spec.n && (spec.type[i] == F_I32 || spec.type[i] == F_DATE || spec.type[i] == F_QTY ||
                                            spec.type[i] == F_DEC32);
        col_max[i] = (int_col && b) ? (int32_t)(b ^ 0x80000000u) : INT32_MIN;
      }
    return GPUDB_OK;
  });
}
