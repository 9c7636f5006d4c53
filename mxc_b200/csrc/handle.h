// Internal definition of the device handle (h2dev_handle_t): the device,
// its stream, handle options and the per-launch profiling records.
#pragma once

#include <cuda_runtime.h>

#include <utility>
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
  int sampling_mode = 0;  // far-list cap rule for solvers created next (H2DEV_OPT_SAMPLING)
  int basis_mode = 0;  // 0: Gram + pivoted Cholesky for fixed-rank bases; 1: Householder TSQR everywhere
  // One reference held by the caller plus one per live solver: the stream
  // (and the stream-ordered memory freed on it) outlives every solver.
  int refs = 1;
  // Pinned staging buffer for host->device uploads of launch plans, so an
  // upload is stream-ordered and never waits for queued kernels.
  char* stage = nullptr;
  size_t stage_cap = 0, stage_head = 0;
  cudaEvent_t stage_ev = nullptr;  // recorded after the latest copy out of `stage`
  std::vector<std::pair<char*, cudaEvent_t>> stage_retired;
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

