// Kernel-shape autotuner (see autotune.hpp).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

#include "autotune.hpp"

namespace sfem {

namespace {

std::mutex g_mu;
std::map<std::string, int> g_cache;
std::string g_path;

std::string device_name() {
  int dev = 0;
  cudaDeviceProp prop{};
  if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
  std::string n = prop.name;
  std::replace(n.begin(), n.end(), ' ', '_');
  std::replace(n.begin(), n.end(), '"', '_');
  return n;
}

// cache file lines: {"key": "...", "variant": v}
void load_file_locked() {
  g_cache.clear();
  std::ifstream in(g_path);
  std::string line;
  while (std::getline(in, line)) {
    const size_t k0 = line.find("\"key\": \"");
    const size_t v0 = line.find("\"variant\": ");
    if (k0 == std::string::npos || v0 == std::string::npos) continue;
    const size_t ks = k0 + 8, ke = line.find('"', ks);
    if (ke == std::string::npos) continue;
    const int v = std::atoi(line.c_str() + v0 + 11);
    if (v > 0) g_cache[line.substr(ks, ke - ks)] = v;
  }
}

}  // namespace

std::vector<int> tune_candidates(const OpConfig& cfg) {
  if (cfg.kind == FEM_CG) return {1, 2, 5, 6, 7};
  return {1, 2, 3, 4, 5};
}

std::string tune_key(const OpConfig& cfg, int64_t cells) {
  std::ostringstream os;
  const int lg = cells > 0 ? int(std::lround(std::log2(double(cells)))) : 0;
  os << "kind=" << cfg.kind << ",p=" << cfg.degree << ",prec=" << cfg.precision << ",nc=" << cfg.n_components
     << ",log2cells=" << lg << ",gpu=" << device_name();
  return os.str();
}

double time_launches(const std::function<void(cudaStream_t)>& run, int reps, cudaStream_t s) {
  SFEM_REQUIRE(reps >= 1 && reps <= 10000, FEM_ERR_ARG, "autotune: reps must be 1..10000");
  run(s);
  run(s);
  std::vector<cudaEvent_t> ev(2 * reps);
  for (auto& e : ev) SFEM_CUDA(cudaEventCreate(&e));
  for (int r = 0; r < reps; ++r) {
    SFEM_CUDA(cudaEventRecord(ev[2 * r], s));
    run(s);
    SFEM_CUDA(cudaEventRecord(ev[2 * r + 1], s));
  }
  SFEM_CUDA(cudaStreamSynchronize(s));
  std::vector<float> ms(reps);
  for (int r = 0; r < reps; ++r) SFEM_CUDA(cudaEventElapsedTime(&ms[r], ev[2 * r], ev[2 * r + 1]));
  for (auto& e : ev) cudaEventDestroy(e);
  std::sort(ms.begin(), ms.end());
  return 1e3 * double(ms[reps / 2]);
}

int tune_lookup(const std::string& key) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cache.find(key);
  return it == g_cache.end() ? 0 : it->second;
}

void tune_store(const std::string& key, int variant, const std::vector<double>& us) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache[key] = variant;
  if (g_path.empty()) return;
  std::ofstream out(g_path, std::ios::app);
  out << "{\"key\": \"" << key << "\", \"variant\": " << variant << ", \"us\": [";
  for (size_t i = 0; i < us.size(); ++i) out << (i ? ", " : "") << us[i];
  out << "]}\n";
  SFEM_REQUIRE(bool(out), FEM_ERR_ARG, "autotune: cannot write the cache file");
}

void tune_set_cache_file(const std::string& path) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_path = path;
  if (path.empty()) {
    g_cache.clear();
    return;
  }
  load_file_locked();
}

TuneResult autotune(Operator& op, int reps, bool use_cache) {
  TuneResult res;
  const std::vector<int> cand = tune_candidates(op.cfg);
  res.us.assign(8, 0.0);
  const std::string key = tune_key(op.cfg, op.n_cells);
  if (use_cache) {
    const int v = tune_lookup(key);
    if (v > 0 && std::find(cand.begin(), cand.end(), v) != cand.end()) {
      op.cfg.kernel_variant = v;
      res.variant = v;
      res.cached = true;
      return res;
    }
  }
  const size_t bytes = size_t(op.m) * op.elem_size();
  DevBuf<unsigned char> src(bytes), dst(bytes);
  SFEM_CUDA(cudaMemset(src.p, 0, bytes));
  cudaStream_t s = nullptr;
  SFEM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const int keep = op.cfg.kernel_variant;
  double best = 1e300;
  try {
    for (int v : cand) {
      op.cfg.kernel_variant = v;
      const double us = time_launches([&](cudaStream_t st) { op.vmult(dst.p, src.p, st); }, reps, s);
      res.us[v - 1] = us;
      if (us < best) {
        best = us;
        res.variant = v;
      }
    }
  } catch (...) {
    op.cfg.kernel_variant = keep;
    cudaStreamDestroy(s);
    throw;
  }
  cudaStreamDestroy(s);
  op.cfg.kernel_variant = res.variant;
  tune_store(key, res.variant, res.us);
  return res;
}

}  // namespace sfem
