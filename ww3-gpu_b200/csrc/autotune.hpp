// ww3-gpu_b200/csrc/autotune.hpp
// The library's autotuner: launch choices timed with CUDA events on the device at set-up, the
// fastest kept per (choice, grid shape, device) for the rest of the process.
//
// What it picks: the DIA kernel of a grid (ww_snl1_autotune: the pair-tile, pair, band, tile,
// row-shift and gather kernels that fit its tables, on synthetic points) and the CTAs per SM of
// the W3SRCE persistent kernels with the shared-memory carveout that goes with them
// (ww_srce_autotune, on a sample of the caller's own points). ww_autotune_report lists every
// choice with its candidates' times.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

namespace wwb {
namespace tune {

/// Times each candidate: run(c, stream) enqueues candidate c's work; one untimed run, then
/// `reps` timed runs (prepare(c, stream), when given, is enqueued before each run and not
/// timed). Records the fastest (least median time) under `key` and returns it.
int pick(const std::string& key, const std::vector<int>& cands,
         const std::function<void(int, cudaStream_t)>& run,
         const std::function<void(int, cudaStream_t)>& prepare, cudaStream_t st, int reps = 3);

/// The choice recorded under key, or `fallback`.
int cached(const std::string& key, int fallback);

/// "sm100 x148 dev0": the device part of a key.
std::string device_key();

/// Every recorded choice as a JSON object: {"key": {"choice": c, "ms": {"c": t, ...}}, ...}.
std::string report();

}  // namespace tune
}  // namespace wwb
