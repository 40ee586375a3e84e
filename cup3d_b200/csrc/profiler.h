// Per-phase device timing with CUDA events, the role of the reference's
// DeviceProfiler (Utils/DeviceProfiler.cuh:26-108): events are recorded on
// the launching stream around each kernel and resolved only when read, so
// enabling it adds no host synchronisation inside a step.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

namespace cup3d {

struct Profiler {
  bool on = false;
  struct Rec {
    int phase;
    int ev;  // index of the begin event; end event is ev + 1
  };
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<Rec> recs;
  std::vector<std::string> names;
  std::map<std::string, int> ids;
  struct Acc {
    double ms = 0;
    long launches = 0;
  };
  std::vector<Acc> acc;

  int phase_id(const char* name) {
    auto it = ids.find(name);
    if (it != ids.end()) return it->second;
    const int id = int(names.size());
    names.push_back(name);
    ids[name] = id;
    acc.push_back(Acc());
    return id;
  }
  // returns the record index or -1
  int begin(const char* name, cudaStream_t s) {
    if (!on) return -1;
    if (used + 2 > pool.size()) flush();
    if (used + 2 > pool.size()) {
      const size_t add = 1024;
      for (size_t i = 0; i < add; ++i) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return -1;
        pool.push_back(e);
      }
    }
    const int ev = int(used);
    used += 2;
    cudaEventRecord(pool[ev], s);
    recs.push_back({phase_id(name), ev});
    return int(recs.size()) - 1;
  }
  void end(int rec, cudaStream_t s) {
    if (rec < 0) return;
    cudaEventRecord(pool[recs[rec].ev + 1], s);
  }
  // resolves recorded pairs (synchronises on the last event)
  void flush() {
    if (recs.empty()) {
      used = 0;
      return;
    }
    cudaEventSynchronize(pool[recs.back().ev + 1]);
    for (const Rec& r : recs) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, pool[r.ev], pool[r.ev + 1]) == cudaSuccess) {
        acc[r.phase].ms += ms;
        acc[r.phase].launches += 1;
      }
    }
    recs.clear();
    used = 0;
  }
  void reset() {
    flush();
    for (auto& a : acc) a = Acc();
  }
  ~Profiler() {
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
};

// The profiler of the context whose API call is running on this thread.
extern thread_local Profiler* t_prof;

struct ProfScope {
  int rec;
  cudaStream_t s;
  ProfScope(const char* name, cudaStream_t st) : rec(t_prof ? t_prof->begin(name, st) : -1), s(st) {}
  ~ProfScope() {
    if (t_prof) t_prof->end(rec, s);
  }
};

}  // namespace cup3d
