// gpudb -- command-line entry of the engine, with the reference's surface:
//     gpudb [sf1|sf10|sf100] [query]      (src/main.cpp:48-72)
// where query is one of the registered pipelines or `all` (src/main.cpp:158-203). sf100
// keeps the fact table in pinned host memory and streams it in chunks, like the
// reference's SF-100 mode. Extra options: --scale F (multiply every table size), --seed N,
// --reps N, --device N, and --data DIR: read DIR/<table>.tbl (dbgen text, parsed on the GPU)
// instead of generating the tables (the reference reads data/SF-N/*.tbl).
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "infra.hpp"

using namespace gpudb_host;

static void show_help() {
  std::printf("Usage: gpudb [sf1|sf10|sf100] [query] [--scale F] [--seed N] [--reps N] [--device N] [--data DIR]\n");
  std::printf("Queries: q1 q3 q4 q5 q6 q7 q8 q9 q10 q12 q13 selection aggregation join all (default: all)\n");
  std::printf("Examples:\n  gpudb            # all pipelines on SF-1\n  gpudb sf10 q1\n  gpudb sf100 q6   # streamed\n"
              "  gpudb q3 --data data/SF-1   # tables from dbgen .tbl files\n");
}

int main(int argc, const char* argv[]) {
  std::string size = "sf1", query = "all";
  double factor = 1.0;
  RunOptions o;
  int device = 0;
  for (int i = 1; i < argc; ++i) {
    std::string a(argv[i]);
    if (a == "help" || a == "--help" || a == "-h") { show_help(); return 0; }
    if (a == "sf1" || a == "sf10" || a == "sf100") { size = a; continue; }
    if (a == "--scale" && i + 1 < argc) { factor = std::atof(argv[++i]); continue; }
    if (a == "--seed" && i + 1 < argc) { o.seed = std::strtoull(argv[++i], nullptr, 10); continue; }
    if (a == "--reps" && i + 1 < argc) { o.reps = std::max(1, std::atoi(argv[++i])); continue; }
    if (a == "--device" && i + 1 < argc) { device = std::atoi(argv[++i]); continue; }
    if (a == "--data" && i + 1 < argc) { o.data_dir = argv[++i]; continue; }
    if (a == "--tbl-piece" && i + 1 < argc) { o.tbl_piece = std::max<size_t>(4096, std::strtoull(argv[++i], nullptr, 10)); continue; }
    query = a;
  }
  o.scale = scale_of(size, factor);
  if (!o.data_dir.empty()) o.scale.streamed = false;   // parsed tables live in HBM
  const std::vector<std::pair<std::string, Driver>> pipelines = {
      {"selection", runSelectionBenchmark}, {"aggregation", runAggregationBenchmark}, {"join", runJoinBenchmark},
      {"q1", runQ1Benchmark},          {"q3", runQ3Benchmark},                {"q4", runQ4Benchmark},
      {"q6", runQ6Benchmark},          {"q9", runQ9Benchmark},                {"q12", runQ12Benchmark},
      {"q5", runQ5Benchmark},          {"q7", runQ7Benchmark},                {"q8", runQ8Benchmark},
      {"q10", runQ10Benchmark},        {"q13", runQ13Benchmark}};
  Driver fn = nullptr;
  if (query != "all") {
    for (auto& e : pipelines)
      if (e.first == query) fn = e.second;
    if (!fn) {
      std::fprintf(stderr, "Unknown query: %s\nUse 'help' to see available options.\n", query.c_str());
      return 1;
    }
  }
  gpudb_ctx* ctx = nullptr;
  int rc = gpudb_create(device, &ctx);
  if (rc != GPUDB_OK) {
    std::fprintf(stderr, "gpudb_create(%d) failed (%d): no sm_100 device\n", device, rc);
    return 1;
  }
  if (o.scale.streamed) {
    std::printf("=== SF100 Chunked Streaming Mode ===\n");
    std::printf("lineitem rows: %llu (pinned host memory, 64M-row chunks)\n", (unsigned long long)o.scale.lineitem);
  }
  if (fn) {
    fn(ctx, o);
  } else {
    for (auto& e : pipelines) e.second(ctx, o);
  }
  gpudb_destroy(ctx);
  return 0;
}
