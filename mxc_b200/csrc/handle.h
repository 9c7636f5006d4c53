// Internal definition of the device handle (h2dev_handle_t): the device,
// its stream, handle options and the per-launch profiling records.
#pragma once

#include <cuda_runtime.h>

#include <deque>
#include <string>
#include <unordered_map>
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
  // Side stream (lowest priority; `stream` has the highest) for work that is
  // independent of the main chain inside one call: the near-field apply of
  // an H^2 matvec runs there while the latency-bound upward / far / downward
  // passes run on `stream`.  Every fork (ev_fork) is joined back into
  // `stream` (ev_join) before the call returns, so all memory and cache
  // ordering stays that of `stream`.
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool prof = false;
  // Expired-wait flag of the mbarrier-pipelined kernels (one int in device
  // memory, owned by this handle): set by any k_tc_gemm_ws or k_stream_dtma
  // launched on this handle's streams, read and cleared by check_tc.
  // tc_pending says such a launch was queued since the last check.
  int* d_tc_err = nullptr;
  bool tc_pending = false;
  int sampling_mode = 0;  // far-list cap rule for solvers created next (H2DEV_OPT_SAMPLING)
  bool matrix_free = false;
  bool precond_bf16 = false;
  bool graph_solve = false;
  // Autotuner (H2DEV_OPT_AUTOTUNE): the launch variant chosen for each plan
  // shape bucket (key: plan name, element size, right-hand sides and
  // log2-bucketed task / row / element counts) and the device times each
  // variant took when it was measured.
  bool autotune = true;
  struct TuneRec {
    int choice;
    std::vector<double> ms;
  };
  std::unordered_map<std::string, TuneRec> tune;
  std::vector<std::string> tune_order;  // GMRES solves on this handle run as one captured CUDA graph (H2DEV_OPT_GRAPH_SOLVE)  // FP32 solvers created next apply their substitution from BF16 copies (H2DEV_OPT_PRECOND_BF16)  // operator-mode solvers created next keep no near blocks or couplings (H2DEV_OPT_MATRIX_FREE)
  int basis_mode = 0;  // 0: Gram + pivoted Cholesky for fixed-rank bases; 1: Householder TSQR everywhere
  // One reference held by the caller plus one per live solver: the stream
  // (and the stream-ordered memory freed on it) outlives every solver.
  int refs = 1;
  // Pinned ring buffer for host->device uploads of launch plans, so an
  // upload is stream-ordered and does not wait for queued kernels.  Each
  // copy in flight is a FIFO record (its byte range and an event recorded
  // after it); space is reclaimed as those events complete.
  struct StageRec {
    size_t start, end;
    cudaEvent_t ev;
  };
  char* stage = nullptr;
  size_t stage_cap = 0, stage_head = 0;
  std::deque<StageRec> stage_inflight;
  std::vector<cudaEvent_t> stage_events;  // completed records' events, for reuse
  // Device memory cache: blocks freed by this handle's solvers and
  // temporaries, by size class.  Every block is used only on `stream`, so a
  // block freed in stream order is reusable at once by later work; steady
  // state factorizations then make no driver allocation calls.
  std::unordered_map<size_t, std::vector<void*>> cache;
  size_t cached_bytes = 0;
  size_t live_bytes = 0;  // blocks handed out (solvers, plans, temporaries)
  size_t peak_live_bytes = 0;  // high-water mark of live_bytes since the last reset
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

