// Internal definition of the device handle (h2dev_handle_t): the device,
// its stream, handle options and the per-launch profiling records.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "h2dev.h"

// Per-launch device timing, recorded only while profiling is enabled on the
// handle: a pair of events around each launch on the handle's stream plus
// the launch's algorithmic FLOP and byte counts.
struct ProfRec {
  const char* name;
  cudaEvent_t a, b;
  double flops, bytes;
};

struct h2dev_handle_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool prof = false;
  int basis_mode = 0;  // 0: Gram + pivoted Cholesky for fixed-rank bases; 1: Householder TSQR everywhere
  std::vector<ProfRec> recs;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  cudaEvent_t take() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  void clear() {
    for (auto& r : recs) {
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    recs.clear();
  }
};

