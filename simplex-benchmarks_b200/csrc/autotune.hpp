// Kernel-shape autotuner: times every kernel variant (cells per CTA, thread
// or warp roles per cell) of an operator or a multi-problem batch with CUDA
// events and keeps the fastest.  Choices are cached per
// (kind, degree, precision, components, log2 cells, GPU name) in memory and,
// when a cache file is set, as JSON lines on disk.  No counterpart in the
// reference (deal.II picks its vectorisation width at compile time).
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "operator.hpp"

namespace sfem {

// candidate kernel variants of an operator configuration
std::vector<int> tune_candidates(const OpConfig& cfg);
// cache key of a configuration with `cells` cells in total
std::string tune_key(const OpConfig& cfg, int64_t cells);
// median device time (us) of `run` on `s` over `reps` launches after 2 warm-ups
double time_launches(const std::function<void(cudaStream_t)>& run, int reps, cudaStream_t s);
// cache access (thread-safe); lookup returns 0 when absent
int tune_lookup(const std::string& key);
void tune_store(const std::string& key, int variant, const std::vector<double>& us);
void tune_set_cache_file(const std::string& path);

// tune one operator: sets op.cfg.kernel_variant to the winner
TuneResult autotune(Operator& op, int reps, bool use_cache);

}  // namespace sfem
