// autotune.h -- measured kernel-variant selection with a JSON cache.
//
// Mirrors the reference's GPU autotuner (include/openpfc/runtime/common/
// gpu_autotune.hpp:76-333): get_config() returns the cached choice or the
// default, tune() times every candidate (3 warm-up runs, then 10 timed runs,
// here with CUDA events on the caller's stream) and stores the fastest; the cache
// lives in $OPENPFC_GPU_AUTOTUNE_CACHE_DIR (default ".") as
// <device id>_opfc_autotune.json, one file and one in-memory table per device
// (the device current at the call).  OPENPFC_GPU_AUTOTUNE_DISABLE=1 always returns
// defaults; OPENPFC_GPU_AUTOTUNE_MODE = auto | cache_only | fallback_only.
// Where the reference tunes 1D block sizes of finite-difference kernels, the
// candidates here are FFT tile shapes and kernel families.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

namespace opfc {

class AutoTuner {
 public:
  static AutoTuner &instance() {
    static AutoTuner t;
    return t;
  }

  // cached variant index for `key`, or `fallback`
  int get_config(const std::string &key, int fallback) {
    std::lock_guard<std::mutex> lock(mu_);
    refresh();
    if (disabled_ || mode_ == "fallback_only") return fallback;
    const Table &t = table();
    auto it = t.entries.find(key);
    return it == t.entries.end() ? fallback : it->second.first;
  }

  // time `run(v)` for v in [0, n) on `s`; cache and return the fastest.
  // `run` returns 0 on success; failing candidates are skipped.
  int tune(const std::string &key, int n, const std::function<int(int)> &run, cudaStream_t s,
           std::vector<double> *ms_out = nullptr) {
    {
      std::lock_guard<std::mutex> lock(mu_);
      refresh();
    }
    if (disabled_ || mode_ == "fallback_only" || mode_ == "cache_only") return get_config(key, 0);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = -1;
    double best_ms = 1e300;
    if (ms_out) ms_out->assign(n, -1.0);
    for (int v = 0; v < n; ++v) {
      bool ok = true;
      for (int w = 0; w < 3 && ok; ++w) ok = run(v) == 0;
      if (!ok) {
        cudaGetLastError();
        continue;
      }
      cudaEventRecord(e0, s);
      for (int r = 0; r < 10 && ok; ++r) ok = run(v) == 0;
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float t = 0;
      cudaEventElapsedTime(&t, e0, e1);
      if (!ok) continue;
      const double ms = t / 10.0;
      if (ms_out) (*ms_out)[v] = ms;
      if (ms < best_ms) {
        best_ms = ms;
        best = v;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best < 0) return 0;
    std::lock_guard<std::mutex> lock(mu_);
    Table &t = table();
    t.entries[key] = {best, best_ms};
    save(t);
    return best;
  }

 private:
  AutoTuner() { refresh(); }

  // the environment is read on every call, so a process can redirect the cache
  void refresh() {
    const char *d = std::getenv("OPENPFC_GPU_AUTOTUNE_DISABLE");
    disabled_ = d && std::string(d) == "1";
    const char *m = std::getenv("OPENPFC_GPU_AUTOTUNE_MODE");
    mode_ = m ? m : "auto";
    const char *c = std::getenv("OPENPFC_GPU_AUTOTUNE_CACHE_DIR");
    const std::string dir = c ? c : ".";
    if (dir != dir_) {
      dir_ = dir;
      tables_.clear();
    }
  }

  struct Table {
    std::string path;
    std::map<std::string, std::pair<int, double>> entries;
  };

  std::string path() const {
    int dev = 0;
    cudaGetDevice(&dev);
    char bus[64] = "gpu";
    if (cudaDeviceGetPCIBusId(bus, sizeof bus, dev) != cudaSuccess) cudaGetLastError();
    std::string id(bus);
    for (char &ch : id)
      if (ch == ':' || ch == '.') ch = '_';
    return dir_ + "/" + id + "_opfc_autotune.json";
  }

  // the current device's table, read from its file on first use; one entry per
  // line: "key": [variant, ms],
  Table &table() {
    const std::string p = path();
    auto it = tables_.find(p);
    if (it != tables_.end()) return it->second;
    Table &t = tables_[p];
    t.path = p;
    std::ifstream f(p);
    std::string line;
    while (std::getline(f, line)) {
      const auto q0 = line.find('"'), q1 = line.find('"', q0 + 1), b = line.find('[', q1);
      if (q0 == std::string::npos || q1 == std::string::npos || b == std::string::npos) continue;
      int v = 0;
      double ms = 0;
      if (std::sscanf(line.c_str() + b, "[%d, %lf]", &v, &ms) == 2) t.entries[line.substr(q0 + 1, q1 - q0 - 1)] = {v, ms};
    }
    return t;
  }

  static void save(const Table &t) {
    std::ofstream f(t.path);
    if (!f) return;
    f << "{\n";
    size_t i = 0;
    for (const auto &kv : t.entries) {
      f << " \"" << kv.first << "\": [" << kv.second.first << ", " << kv.second.second << "]"
        << (++i < t.entries.size() ? ",\n" : "\n");
    }
    f << "}\n";
  }

  std::mutex mu_;
  bool disabled_ = false;
  std::string mode_, dir_;
  std::map<std::string, Table> tables_;  // by cache file (one per device)
};

}  // namespace opfc
