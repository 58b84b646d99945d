// Autotuner: times the candidate configurations of a pipeline on the caller's own tables and
// keeps the fastest on the context. The knobs are the ones the kernels expose as context
// options: the Q1 kernel variant (block size, rows per thread, 128-bit loads, TMA staging,
// shared-memory accumulators), the Q6 kernel variant (row kernel or 128-bit loads with 1, 2
// or 4 quads per thread per step), the hash-table load factor of the Q3 build (50% or 25%),
// the radix fan-out of the Q3 radix mode, the join mode that a Q3 AUTO request runs (direct
// map, global table or radix partitions), and the Q9 aggregation slot counts (shared and
// global). Every candidate must give the same result as the default configuration; a
// candidate that does not is dropped (and reported) rather than chosen.
//
// Choices are kept per context and can be written to, and read back from, a small text
// cache keyed by the device name (gpudb_tune_save / gpudb_tune_load).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace gpudb {
namespace {

struct Candidate {
  int32_t option;
  int64_t value;
  int32_t option2;    // 0: none
  int64_t value2;
};

std::string device_name(gpudb_ctx* ctx) {
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) return "unknown";
  std::string n = prop.name;
  for (char& c : n)
    if (c == '|' || c == '\n') c = ' ';
  return n;
}

// The result of one run of a request, kept until the run completes (an async run writes it
// at gpudb_sync).
struct Outs {
  gpudb_q6_result q6{};
  gpudb_q1_result q1{};
  gpudb_q3_result q3{};
  std::vector<gpudb_q9_group> q9 = std::vector<gpudb_q9_group>(256);
  uint32_t n9 = 0;
  gpudb_timing t{};
};

// Enqueues one run of the request through its single-request pipeline (synchronous when
// `ex` is null), writing into `o`.
int run(gpudb_ctx* ctx, const gpudb_request& q, Outs& o, const gpudb_exec* ex) {
  switch (q.pipeline) {
    case GPUDB_PIPE_Q6: return gpudb_q6_sum(ctx, q.li, &q.q6, &o.q6, &o.t, ex);
    case GPUDB_PIPE_Q1: return gpudb_q1_group6(ctx, q.li, &q.q1, &o.q1, &o.t, ex);
    case GPUDB_PIPE_Q3:
      return gpudb_q3_join_topk(ctx, &q.q3->cu, &q.q3->od, &q.q3->li, &q.q3p, &o.q3, &o.t, ex);
    case GPUDB_PIPE_Q9:
      return gpudb_q9_star(ctx, &q.q9->pa, &q.q9->su, &q.q9->ps, &q.q9->od, &q.q9->li, &q.q9p, o.q9.data(), 256,
                           &o.n9, &o.t, ex);
    default:
      return fail(ctx, GPUDB_E_INVALID, "autotune: unknown pipeline %d", q.pipeline);
  }
}

// A digest of a completed run's result (the bytes of the result struct).
std::string digest_of(const gpudb_request& q, Outs& o) {
  switch (q.pipeline) {
    case GPUDB_PIPE_Q6: return std::string(reinterpret_cast<const char*>(&o.q6), sizeof o.q6);
    case GPUDB_PIPE_Q1: return std::string(reinterpret_cast<const char*>(&o.q1), sizeof o.q1);
    case GPUDB_PIPE_Q3: {
      gpudb_q3_result r = o.q3;
      r.join_mode = 0;   // the mode that ran differs between candidates; the answer must not
      return std::string(reinterpret_cast<const char*>(&r), sizeof r);
    }
    default: {
      std::string d(reinterpret_cast<const char*>(o.q9.data()), std::min<uint32_t>(o.n9, 256) * sizeof(gpudb_q9_group));
      d.append(reinterpret_cast<const char*>(&o.n9), sizeof o.n9);
      return d;
    }
  }
}

int apply(gpudb_ctx* ctx, const Candidate& c) {
  int rc = gpudb_set_option(ctx, c.option, c.value);
  if (!rc && c.option2) rc = gpudb_set_option(ctx, c.option2, c.value2);
  return rc;
}

// Median device time of `reps` runs issued back to back on the context's stream (as calls
// run when a batch or a served stream keeps the GPU busy; an isolated call after idle time
// measures a microsecond or two more), after one synchronous run that sizes scratch and
// gives the digest. Every timed run's result must equal that digest.
int measure(gpudb_ctx* ctx, const gpudb_request& q, uint32_t reps, double* median, std::string* digest) {
  Outs first;
  int rc = run(ctx, q, first, nullptr);
  if (rc) return rc;
  *digest = digest_of(q, first);
  std::vector<Outs> outs(reps);
  gpudb_exec ex{};
  ex.async = 1;
  for (uint32_t i = 0; i < reps && !rc; i++) rc = run(ctx, q, outs[i], &ex);
  const int rs = gpudb_sync(ctx);   // also when an enqueue failed: no run is left in flight
  if (rc) return rc;
  if (rs) return rs;
  std::vector<double> v;
  for (uint32_t i = 0; i < reps; i++) {
    if (digest_of(q, outs[i]) != *digest) return fail(ctx, GPUDB_E_CUDA, "autotune: a configuration is not deterministic");
    v.push_back(outs[i].t.gpu_ms);
  }
  std::sort(v.begin(), v.end());
  *median = v.empty() ? first.t.gpu_ms : v[v.size() / 2];
  return GPUDB_OK;
}

uint64_t rows_of(const gpudb_request& q) {
  switch (q.pipeline) {
    case GPUDB_PIPE_Q6:
    case GPUDB_PIPE_Q1: return q.li ? q.li->n_rows : 0;
    case GPUDB_PIPE_Q3: return q.q3 ? q.q3->li.n_rows : 0;
    case GPUDB_PIPE_Q9: return q.q9 ? q.q9->li.n_rows : 0;
    default: return 0;
  }
}

}  // namespace
}  // namespace gpudb

using namespace gpudb;

extern "C" int gpudb_autotune(gpudb_ctx* ctx, const gpudb_request* req, uint32_t reps, gpudb_tune_result* out) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!req || !out) return fail(ctx, GPUDB_E_INVALID, "autotune: request and result are required");
  const gpudb_request& q = *req;
  if ((q.pipeline == GPUDB_PIPE_Q6 || q.pipeline == GPUDB_PIPE_Q1) && !q.li)
    return fail(ctx, GPUDB_E_INVALID, "autotune: scan request without a table");
  if ((q.pipeline == GPUDB_PIPE_Q3 && !q.q3) || (q.pipeline == GPUDB_PIPE_Q9 && !q.q9))
    return fail(ctx, GPUDB_E_INVALID, "autotune: join request without tables");
  reps = std::max<uint32_t>(1, std::min<uint32_t>(reps, 1000));
  std::vector<Candidate> cands;
  Candidate def{};
  switch (q.pipeline) {
    case GPUDB_PIPE_Q1:
      def = {GPUDB_OPT_SCAN_VARIANT, 0, 0, 0};
      for (int v = 1; v <= 10; v++) cands.push_back({GPUDB_OPT_SCAN_VARIANT, v, 0, 0});
      break;
    case GPUDB_PIPE_Q6:
      def = {GPUDB_OPT_Q6_VARIANT, 0, 0, 0};
      for (int v = 1; v <= 4; v++) cands.push_back({GPUDB_OPT_Q6_VARIANT, v, 0, 0});
      break;
    case GPUDB_PIPE_Q3:
      if (q.q3p.join_mode == GPUDB_JOIN_AUTO) {
        // the join mode itself: direct map (when the orders carry a key bound), global
        // table, radix partitions
        def = {GPUDB_OPT_Q3_AUTO_MODE, -1, 0, 0};
        if (q.q3->od.key_max >= 0) cands.push_back({GPUDB_OPT_Q3_AUTO_MODE, GPUDB_JOIN_DIRECT, 0, 0});
        cands.push_back({GPUDB_OPT_Q3_AUTO_MODE, GPUDB_JOIN_GLOBAL, 0, 0});
        cands.push_back({GPUDB_OPT_Q3_AUTO_MODE, GPUDB_JOIN_RADIX, 0, 0});
      } else if (q.q3p.join_mode == GPUDB_JOIN_RADIX) {
        // fan-outs around the default (about 16K orders rows per partition): fewer partitions
        // re-probe the fact rows once per shared-table chunk, more than 1024 take a second
        // partitioning pass
        def = {GPUDB_OPT_RADIX_BITS, 0, 0, 0};
        int lo = 4;
        while (lo < kRadixMaxBits && (q.q3->od.n_rows >> lo) > 65536) lo++;
        for (int b = std::max(lo, 8); b <= std::min(lo + 5, (int)kRadixMaxBits); b++)
          cands.push_back({GPUDB_OPT_RADIX_BITS, b, 0, 0});
      } else {
        def = {GPUDB_OPT_HT_LOAD, 50, 0, 0};
        cands.push_back({GPUDB_OPT_HT_LOAD, 25, 0, 0});
      }
      break;
    case GPUDB_PIPE_Q9:
      def = {GPUDB_OPT_Q9_SMEM_SLOTS, 1024, GPUDB_OPT_Q9_GLOBAL_SLOTS, 4096};
      for (int sm : {256, 512, 1024, 2048, 4096})
        for (int gl : {1024, 4096, 8192}) cands.push_back({GPUDB_OPT_Q9_SMEM_SLOTS, sm, GPUDB_OPT_Q9_GLOBAL_SLOTS, gl});
      break;
    default:
      return fail(ctx, GPUDB_E_INVALID, "autotune: unknown pipeline %d", q.pipeline);
  }
  // the previous settings come back if anything fails
  int64_t prev1 = 0, prev2 = 0;
  gpudb_get_option(ctx, def.option, &prev1);
  if (def.option2) gpudb_get_option(ctx, def.option2, &prev2);
  auto restore = [&]() {
    gpudb_set_option(ctx, def.option, prev1);
    if (def.option2) gpudb_set_option(ctx, def.option2, prev2);
  };
  int rc = apply(ctx, def);
  std::string want;
  double def_ms = 0;
  if (!rc) rc = measure(ctx, q, reps, &def_ms, &want);
  if (rc) { restore(); return rc; }
  Candidate best = def;
  double best_ms = def_ms;
  uint32_t timed = 1, dropped = 0;
  for (const Candidate& c : cands) {
    if (apply(ctx, c)) { dropped++; continue; }
    std::string got;
    double ms = 0;
    const int r = measure(ctx, q, reps, &ms, &got);
    timed++;
    if (r != GPUDB_OK || got != want) { dropped++; continue; }
    if (ms < best_ms) { best_ms = ms; best = c; }
  }
  rc = apply(ctx, best);
  if (rc) { restore(); return rc; }
  const uint64_t rows = rows_of(q);
  const int32_t rl = rows ? (int32_t)std::floor(std::log2((double)rows)) : 0;
  auto remember = [&](int32_t option, int64_t value) {
    for (auto& t : ctx->tuned)
      if (t.pipeline == q.pipeline && t.rows_log2 == rl && t.option == option) { t.value = value; return; }
    ctx->tuned.push_back({q.pipeline, rl, option, value});
  };
  remember(best.option, best.value);
  if (best.option2) remember(best.option2, best.value2);
  out->pipeline = q.pipeline;
  out->candidates = timed;
  out->dropped = dropped;
  out->option = best.option;
  out->value = best.value;
  out->option2 = best.option2;
  out->value2 = best.value2;
  out->best_ms = best_ms;
  out->default_ms = def_ms;
  return GPUDB_OK;
}

extern "C" int gpudb_tune_save(gpudb_ctx* ctx, const char* path) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!path) return fail(ctx, GPUDB_E_INVALID, "tune cache: path is required");
  const std::string dev = device_name(ctx);
  // keep other devices' lines, replace this device's
  std::vector<std::string> keep;
  if (FILE* f = std::fopen(path, "r")) {
    char line[512];
    while (std::fgets(line, sizeof line, f)) {
      std::string l(line);
      if (l.compare(0, dev.size() + 1, dev + "|") != 0 && !l.empty() && l[0] != '#') keep.push_back(l);
    }
    std::fclose(f);
  }
  FILE* f = std::fopen(path, "w");
  if (!f) return fail(ctx, GPUDB_E_INVALID, "tune cache: cannot write %s", path);
  std::fprintf(f, "# device|pipeline|rows_log2|option|value\n");
  for (const auto& l : keep) std::fputs(l.c_str(), f);
  for (const auto& t : ctx->tuned)
    std::fprintf(f, "%s|%d|%d|%d|%lld\n", dev.c_str(), t.pipeline, t.rows_log2, t.option, (long long)t.value);
  std::fclose(f);
  return GPUDB_OK;
}

extern "C" int gpudb_tune_load(gpudb_ctx* ctx, const char* path, uint32_t* applied) {
  if (!ctx) return GPUDB_E_INVALID;
  if (!path) return fail(ctx, GPUDB_E_INVALID, "tune cache: path is required");
  if (applied) *applied = 0;
  FILE* f = std::fopen(path, "r");
  if (!f) return fail(ctx, GPUDB_E_INVALID, "tune cache: cannot read %s", path);
  const std::string dev = device_name(ctx);
  char line[512];
  int rc = GPUDB_OK;
  while (std::fgets(line, sizeof line, f)) {
    std::string l(line);
    if (l.empty() || l[0] == '#' || l.compare(0, dev.size() + 1, dev + "|") != 0) continue;
    int pipeline = 0, rl = 0, option = 0;
    long long value = 0;
    if (std::sscanf(l.c_str() + dev.size() + 1, "%d|%d|%d|%lld", &pipeline, &rl, &option, &value) != 4) continue;
    if (gpudb_set_option(ctx, option, value) != GPUDB_OK) { rc = GPUDB_E_INVALID; continue; }
    bool found = false;
    for (auto& t : ctx->tuned)
      if (t.pipeline == pipeline && t.rows_log2 == rl && t.option == option) { t.value = value; found = true; }
    if (!found) ctx->tuned.push_back({pipeline, rl, option, value});
    if (applied) (*applied)++;
  }
  std::fclose(f);
  if (rc) return fail(ctx, rc, "tune cache: a line of %s holds an invalid option value", path);
  return GPUDB_OK;
}
