// Join-count helpers shared by micro.cu (global-table mode) and radix.cu (radix mode).
#pragma once
#include "engine.h"

namespace gpudb {

// Open-addressing set of the build keys in the "join.set" scratch buffer.
int build_key_set(Call& call, const int32_t* keys, uint64_t n, int32_t** set_out, uint32_t* cap_out);
// Semi-join count (probe rows with at least one matching build key) via radix partitioning;
// adds into *count (device).
int radix_join_count(Call& call, const int32_t* build_keys, uint64_t n_build, const int32_t* probe_keys,
                     uint64_t n_probe, unsigned long long* count);

}  // namespace gpudb
