// Autotuner (tuner.h) and its C ABI (p2_tune_enable, p2_tune_count).
#include <algorithm>
#include <cstdio>
#include <fstream>
#include <sstream>

#include "ctx.h"

namespace p2host {

void Tuner::load() {
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::stringstream ss(line);
    std::string key, ps, ms;
    if (!std::getline(ss, key, '\t') || !std::getline(ss, ps, '\t') || !std::getline(ss, ms)) continue;
    TuneChoice c;
    std::stringstream ps2(ps);
    std::string v;
    bool ok = true;
    while (std::getline(ps2, v, ',')) {
      try {
        c.params.push_back(std::stoi(v));
      } catch (...) {
        ok = false;
      }
    }
    try {
      c.ms = std::stod(ms);
    } catch (...) {
      ok = false;
    }
    if (ok && !c.params.empty()) cache[key] = c;
  }
}

bool Tuner::save() {
  if (path.empty()) return true;
  const std::string tmp = path + ".tmp";
  {
    std::ofstream f(tmp, std::ios::trunc);
    if (!f) return false;
    for (const auto& kv : cache) {
      f << kv.first << '\t';
      for (size_t i = 0; i < kv.second.params.size(); i++) f << (i ? "," : "") << kv.second.params[i];
      f << '\t' << kv.second.ms << '\n';
    }
    if (!f) return false;
  }
  return std::rename(tmp.c_str(), path.c_str()) == 0;
}

cudaError_t tune_choose(Tuner* t, const std::string& key, const std::vector<std::vector<int>>& cands,
                        cudaStream_t stream, bool may_time, const LaunchFn& launch, std::vector<int>& out) {
  out = cands.at(0);
  if (!t) return cudaSuccess;
  {
    std::lock_guard<std::mutex> lk(t->mu);
    auto it = t->cache.find(key);
    if (it != t->cache.end() && std::find(cands.begin(), cands.end(), it->second.params) != cands.end()) {
      out = it->second.params;
      return cudaSuccess;
    }
    if (!t->on || !may_time || cands.size() < 2) return cudaSuccess;
  }
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e != cudaSuccess) return e;
  e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cudaEventDestroy(e0);
    return e;
  }
  double best = 1e300;
  size_t pick = 0;
  for (size_t i = 0; i < cands.size() && e == cudaSuccess; i++) {
    e = launch(cands[i]);  // untimed: first-touch and instruction cache
    if (e == cudaSuccess) e = cudaEventRecord(e0, stream);
    for (int r = 0; r < 2 && e == cudaSuccess; r++) e = launch(cands[i]);
    if (e == cudaSuccess) e = cudaEventRecord(e1, stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && ms / 2 < best) {
      best = ms / 2;
      pick = i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return e;
  out = cands[pick];
  std::lock_guard<std::mutex> lk(t->mu);
  t->cache[key] = TuneChoice{out, best};
  t->save();
  return cudaSuccess;
}

}  // namespace p2host

extern "C" {

p2_status p2_tune_enable(p2_ctx* c, int on, const char* cache_path) {
  if (!c) return P2_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(c->tuner->mu);
  c->tuner->on = on != 0;
  if (cache_path) {
    c->tuner->path = cache_path;
    c->tuner->load();
  }
  return P2_OK;
}

int p2_tune_count(p2_ctx* c) {
  if (!c) return -1;
  std::lock_guard<std::mutex> lk(c->tuner->mu);
  return (int)c->tuner->cache.size();
}

}  // extern "C"
