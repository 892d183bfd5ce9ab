// Launch-shape autotuner: per (kernel, shape) key, the fastest of a list of
// candidate parameter vectors, timed on the device the first time the key is
// seen and cached for the process and, optionally, in a tab-separated file.
// Plays the role of the reference's tuneAndRun / TuneKey cache
// (lib/kernels/PLEGMA_kernel_tuner.cuh:61-140) for this library's kernels.
#pragma once
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace p2host {

struct TuneChoice {
  std::vector<int> params;
  double ms = 0;
};

struct Tuner {
  bool on = false;
  std::string path;  // empty: in-memory cache only
  std::map<std::string, TuneChoice> cache;
  std::mutex mu;
  // "key\tp0,p1,...\tms" per line; unknown or malformed lines are skipped
  void load();
  bool save();
};

using LaunchFn = std::function<cudaError_t(const std::vector<int>&)>;

// The parameters to launch with for `key`: the cached choice when there is
// one (and it is still a candidate); otherwise, when tuning is on and `may_time`
// holds, every candidate is launched on `stream` (one untimed launch, then the
// mean of two timed ones) and the fastest is cached; otherwise cands[0].  The
// caller launches the returned parameters itself: candidate launches must
// overwrite the same outputs completely.
cudaError_t tune_choose(Tuner* t, const std::string& key, const std::vector<std::vector<int>>& cands,
                        cudaStream_t stream, bool may_time, const LaunchFn& launch, std::vector<int>& out);

}  // namespace p2host
