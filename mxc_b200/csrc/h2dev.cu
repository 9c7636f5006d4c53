// C ABI and level drivers of the B200-native H^2 solver.
//
// Single process, single device: every box of every level is local, so the
// reference's ColCommMPI reduces to identity collectives and all halo data
// is read in place from HBM (comm-mpi.cpp:198-225 become no-ops).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <future>
#include <thread>
#include <type_traits>
#include <vector>

#include "h2dev.h"
#include "kernels.h"
#include "plan.hpp"

#include "handle.h"

namespace h2b {

static thread_local h2dev_handle_s* g_cur = nullptr;

// Scope of one API call on a handle: makes the handle current for the
// library's allocations and launches, and its device current for the CUDA
// runtime (the caller's current device is restored on exit).
struct CurHandle {
  h2dev_handle_s* prev;
  int prev_dev = -1;
  explicit CurHandle(h2dev_handle_s* h) : prev(g_cur) {
    g_cur = h;
    int d = -1;
    if (h && cudaGetDevice(&d) == cudaSuccess && d != h->device && cudaSetDevice(h->device) == cudaSuccess)
      prev_dev = d;
  }
  ~CurHandle() {
    g_cur = prev;
    if (prev_dev >= 0) cudaSetDevice(prev_dev);
  }
};

struct Prof {
  h2dev_handle_s* h;
  ProfRec r;
  cudaStream_t s = nullptr;
  Prof(const char* name, double flops, double bytes, cudaStream_t on = nullptr)
      : h(g_cur && g_cur->prof ? g_cur : nullptr) {
    if (!h) return;
    s = on ? on : h->stream;
    r.name = name;
    r.flops = flops;
    r.bytes = bytes;
    r.a = h->take();
    r.b = h->take();
    cudaEventRecord(r.a, s);
  }
  ~Prof() {
    if (!h) return;
    cudaEventRecord(r.b, s);
    h->recs.push_back(r);
  }
};

struct H2Error {
  int code;
  std::string msg;
};

static thread_local std::string g_last_error;

static void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    int code = (e == cudaErrorMemoryAllocation) ? H2DEV_ERR_OOM : H2DEV_ERR_CUDA;
    cudaGetLastError();
    throw H2Error{code, std::string(what) + ": " + cudaGetErrorString(e)};
  }
}

static void require(bool ok, const char* what) {
  if (!ok) throw H2Error{H2DEV_ERR_ARG, what};
}

// Host->device copy through the handle's pinned ring (64 MB): the bytes are
// copied into pinned memory at once and the DMA is queued on the handle's
// stream.  When the ring has no room, the call waits for the oldest copy in
// flight to finish; uploads larger than half the ring go in pieces.
constexpr size_t STAGE_BYTES = (size_t)64 << 20;

static void stage_reclaim(h2dev_handle_s* h) {
  while (!h->stage_inflight.empty()) {
    cudaError_t q = cudaEventQuery(h->stage_inflight.front().ev);
    if (q == cudaErrorNotReady) {
      cudaGetLastError();
      return;
    }
    ck(q, "stage event");
    h->stage_events.push_back(h->stage_inflight.front().ev);
    h->stage_inflight.pop_front();
  }
}

static char* stage_reserve(h2dev_handle_s* h, size_t need) {
  if (!h->stage) {
    ck(cudaHostAlloc((void**)&h->stage, STAGE_BYTES, cudaHostAllocDefault), "cudaHostAlloc");
    h->stage_cap = STAGE_BYTES;
    h->stage_head = 0;
  }
  for (;;) {
    stage_reclaim(h);
    if (h->stage_inflight.empty()) h->stage_head = 0;
    const size_t head = h->stage_head, cap = h->stage_cap;
    size_t pos = SIZE_MAX;
    if (h->stage_inflight.empty()) {
      pos = 0;
    } else {
      const size_t tail = h->stage_inflight.front().start;
      if (head > tail) {
        if (cap - head >= need) pos = head;
        else if (tail >= need) pos = 0;
      } else if (head < tail && tail - head >= need) {
        pos = head;
      }
    }
    if (pos != SIZE_MAX) {
      h->stage_head = pos + need;
      return h->stage + pos;
    }
    // No room: wait for the oldest copy in flight.
    ck(cudaEventSynchronize(h->stage_inflight.front().ev), "stage wait");
  }
}

static void stage_copy(h2dev_handle_s* h, void* dst, const void* src, size_t bytes) {
  const size_t piece = STAGE_BYTES / 2;
  for (size_t o = 0; o < bytes; o += piece) {
    const size_t nb = std::min(piece, bytes - o);
    const size_t need = (nb + 255) & ~(size_t)255;
    char* buf = stage_reserve(h, need);
    std::memcpy(buf, static_cast<const char*>(src) + o, nb);
    ck(cudaMemcpyAsync(static_cast<char*>(dst) + o, buf, nb, cudaMemcpyHostToDevice, h->stream), "upload");
    cudaEvent_t ev;
    if (!h->stage_events.empty()) {
      ev = h->stage_events.back();
      h->stage_events.pop_back();
    } else {
      ck(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
    }
    ck(cudaEventRecord(ev, h->stream), "cudaEventRecord");
    h->stage_inflight.push_back(h2dev_handle_s::StageRec{(size_t)(buf - h->stage), (size_t)(buf - h->stage) + need, ev});
  }
}

static void stage_release(h2dev_handle_s* h) {
  for (auto& r : h->stage_inflight) {
    cudaEventSynchronize(r.ev);
    cudaEventDestroy(r.ev);
  }
  h->stage_inflight.clear();
  for (cudaEvent_t e : h->stage_events) cudaEventDestroy(e);
  h->stage_events.clear();
  if (h->stage) cudaFreeHost(h->stage);
  h->stage = nullptr;
  h->stage_cap = h->stage_head = 0;
}

// Size classes of the handle's device-memory cache: four per octave (at
// most 25% rounding), 512 bytes at least.
static size_t cache_class(size_t bytes) {
  size_t b = std::max<size_t>(bytes, 512);
  int p = 63 - __builtin_clzll((unsigned long long)b);
  if (b == ((size_t)1 << p)) return b;
  const size_t step = (size_t)1 << (p - 2);
  return (b + step - 1) / step * step;
}

// Returns every cached block to the driver (after the stream drains).
static void cache_trim(h2dev_handle_s* h) {
  if (h->cached_bytes == 0) return;
  cudaStreamSynchronize(h->stream);
  for (auto& kv : h->cache)
    for (void* p : kv.second) cudaFree(p);
  h->cache.clear();
  h->cached_bytes = 0;
}

static void* cache_alloc(h2dev_handle_s* h, size_t cls) {
  auto it = h->cache.find(cls);
  if (it != h->cache.end() && !it->second.empty()) {
    void* p = it->second.back();
    it->second.pop_back();
    h->cached_bytes -= cls;
    h->live_bytes += cls;
    h->peak_live_bytes = std::max(h->peak_live_bytes, h->live_bytes);
    return p;
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, cls);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    cache_trim(h);
    e = cudaMalloc(&p, cls);
  }
  ck(e, "cudaMalloc");
  h->live_bytes += cls;
  h->peak_live_bytes = std::max(h->peak_live_bytes, h->live_bytes);
  return p;
}

static void cache_free(h2dev_handle_s* h, void* p, size_t cls) {
  h->cache[cls].push_back(p);
  h->cached_bytes += cls;
  h->live_bytes -= cls;
}

// Device array.  Inside an API call (a current handle) memory comes from the
// handle's cache and goes back to it when released; all its users are on the
// handle's stream, so temporaries need no synchronisation before they go.
template <typename T>
struct DVec {
  T* p = nullptr;
  size_t n = 0;
  h2dev_handle_s* owner = nullptr;  // cache the block came from (none: plain cudaMalloc)
  size_t cls = 0;
  DVec() = default;
  DVec(const DVec&) = delete;
  DVec& operator=(const DVec&) = delete;
  DVec(DVec&& o) noexcept : p(o.p), n(o.n), owner(o.owner), cls(o.cls) { o.p = nullptr; o.n = 0; }
  DVec& operator=(DVec&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; owner = o.owner; cls = o.cls;
      o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  ~DVec() { release(); }
  void release() {
    if (p) {
      if (owner)
        cache_free(owner, p, cls);
      else
        cudaFree(p);
    }
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count == n && p) return;
    release();
    owner = g_cur;
    if (count) {
      if (owner) {
        cls = cache_class(count * sizeof(T));
        p = static_cast<T*>(cache_alloc(owner, cls));
      } else {
        ck(cudaMalloc((void**)&p, count * sizeof(T)), "cudaMalloc");
      }
    }
    n = count;
  }
  void zero(cudaStream_t st) {
    if (n) ck(cudaMemsetAsync(p, 0, n * sizeof(T), st), "cudaMemsetAsync");
  }
  void upload(const std::vector<T>& v) {
    alloc(v.size());
    if (v.empty()) return;
    if (owner && g_cur == owner)
      stage_copy(g_cur, p, v.data(), v.size() * sizeof(T));
    else {
      // From pageable memory cudaMemcpy may return before its DMA lands;
      // wait for it so that work on any stream sees the data.
      ck(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
      ck(cudaStreamSynchronize(cudaStreamLegacy), "upload sync");
    }
  }
  std::vector<T> download(cudaStream_t st) const {
    std::vector<T> v(n);
    if (n) {
      ck(cudaStreamSynchronize(st), "sync");
      ck(cudaMemcpy(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost), "download");
    }
    return v;
  }
};

// Process-wide choice of the apply kernel for skinny plans (handle option
// H2DEV_OPT_SKINNY_TILED, used to compare the two kernels).
static bool g_force_tiled = false;
static bool force_tiled() { return g_force_tiled; }
// Process-wide mode of the FP32 contractions (H2DEV_OPT_TENSOR_CORES):
// 0 SIMT, 1 tcgen05 with the 3-term TF32 split, 2 tcgen05 single TF32.
static int g_tensor_cores = 1;

// Throws when a tensor-core GEMM launched on this handle since the last
// check reported an expired wait (then its output is incomplete).  Reads and
// clears the handle's flag; synchronises the handle's streams only when such
// a GEMM was queued.
static void check_tc(h2dev_handle_s* h) {
  if (!h || !h->tc_pending) return;
  int flag = 0;
  ck(cudaStreamSynchronize(h->stream2), "sync");
  ck(cudaStreamSynchronize(h->stream), "sync");
  ck(cudaMemcpy(&flag, h->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost), "tensor-core GEMM status");
  h->tc_pending = false;
  if (flag) {
    ck(cudaMemset(h->d_tc_err, 0, sizeof(int)), "tensor-core GEMM status");
    throw H2Error{H2DEV_ERR_CUDA,
                  "tensor-core GEMM or bulk-copy apply: an mbarrier wait expired (the result is incomplete)"};
  }
}

// Largest row count of a generation task list (one CTA per 256 rows).
static i64 gen_max_rows(const std::vector<GenTask>& gt) {
  i64 m = 0;
  for (const auto& t : gt) m = std::max<i64>(m, t.m);
  return m;
}

// The current handle's error word for the bulk-copy staging of the
// generation kernel (checked with the other mbarrier-pipelined kernels').
static int* gen_err() {
  if (!g_cur) return nullptr;
  g_cur->tc_pending = true;
  return g_cur->d_tc_err;
}

// ------------------------------------------------------------------ autotuner
// The first time a plan of a given shape bucket runs on a handle (outside
// any stream capture), every launch variant it admits is timed on the
// plan's own data -- twice each, keeping the second time, with CUDA events
// on the launching stream -- and the fastest is recorded for the bucket;
// later plans of the bucket (every factorization of a serving system, every
// step of a benchmark) reuse the choice without timing.  Variants differ
// only in how rows are tiled over CTAs, so every variant gives the same
// result bit for bit.
static std::string tune_key(const char* name, int esize, int nr, double tasks, double rows, double elems) {
  auto b = [](double v) { return v <= 1. ? 0 : (int)std::ceil(std::log2(v)); };
  char buf[160];
  snprintf(buf, sizeof(buf), "%s/e%d/n%d/t%d/r%d/a%d", name, esize, nr, b(tasks), b(rows), b(elems));
  return buf;
}

static bool stream_capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

// Returns the variant to run for `key` (0 when tuning is off or impossible),
// timing `nvar` variants through run_variant(v) when the bucket is new.
template <typename F>
static int tuned_variant(const std::string& key, int nvar, cudaStream_t st, F run_variant) {
  h2dev_handle_s* h = g_cur;
  if (!h || !h->autotune || nvar < 2) return 0;
  auto it = h->tune.find(key);
  if (it != h->tune.end()) return it->second.choice;
  if (stream_capturing(st) || h->prof) return 0;
  h2dev_handle_s::TuneRec rec;
  rec.ms.assign(nvar, 0.);
  cudaEvent_t a = nullptr, b = nullptr;
  ck(cudaEventCreate(&a), "event");
  ck(cudaEventCreate(&b), "event");
  for (int v = 0; v < nvar; v++)
    for (int rep = 0; rep < 2; rep++) {
      ck(cudaEventRecord(a, st), "event");
      run_variant(v);
      ck(cudaEventRecord(b, st), "event");
      ck(cudaEventSynchronize(b), "event");
      float ms = 0.f;
      ck(cudaEventElapsedTime(&ms, a, b), "event");
      rec.ms[v] = ms;
    }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  rec.choice = 0;
  for (int v = 1; v < nvar; v++)
    if (rec.ms[v] < rec.ms[rec.choice]) rec.choice = v;
  h->tune[key] = rec;
  h->tune_order.push_back(key);
  return rec.choice;
}

// Host-built list of segmented-GEMM tasks, uploaded once and replayed.
template <typename T>
struct GemmPlan {
  std::vector<GemmTask<T>> tasks;
  std::vector<GemmEntry<T>> ents;
  DVec<GemmTask<T>> d_tasks;
  DVec<GemmEntry<T>> d_ents;
  DVec<TileRef> d_tiles;
  int ntiles = 0;
  int shape = GEMM_BIG;
  int tc_mode = 0;  // GEMM_TC: 1 three-term TF32 split, 2 single TF32
  const char* name = "seg_gemm";
  double flops = 0., bytes = 0.;  // algorithmic work of one run
  bool skinny_nn = false;          // use k_skinny_nn instead of the tiled kernel
  int nr = 0;
  DVec<int2> d_rtiles, d_rtiles_w;  // row tiles of the 128- and 256-row streaming variants
  // Autotuned tilings of the streaming path: 0 = per-task rule (256-row
  // tiles where they pad no more than 128-row ones), 1 = all 128-row, 2 =
  // all 256-row tiles.
  DVec<int2> d_alt_n, d_alt_w;
  std::string tkey;
  mutable int variant = -1;
  // Only plans that overwrite their outputs (every beta zero) are timed:
  // repeating one leaves the same result, so tuning runs are harmless.
  bool idempotent = false;
  // FP64 streaming plans whose A columns all start on 16-byte boundaries run
  // the bulk-copy kernel.
  bool bulk_ok = false;
  DVec<T> parts_buf;               // partial results of split tasks
  DVec<SumTask<T>> d_sums;
  int nsums = 0, sum_maxmn = 0;
  double sum_bytes = 0.;
  void add_task(T* C, i64 ldc, int m, int n, T beta) {
    GemmTask<T> t;
    t.C = C; t.ldc = ldc; t.m = m; t.n = n; t.beta = beta;
    t.e0 = t.e1 = (int)ents.size();
    tasks.push_back(t);
  }
  void add_entry(const T* A, i64 lda, int opA, const T* B, i64 ldb, int opB, int k, T alpha) {
    if (k <= 0) return;
    GemmEntry<T> e;
    e.A = A; e.B = B; e.lda = lda; e.ldb = ldb; e.k = k; e.opA = opA; e.opB = opB; e.alpha = alpha;
    ents.push_back(e);
    tasks.back().e1 = (int)ents.size();
  }
  void finalize() {
    int maxn = 0;
    for (auto& t : tasks) maxn = std::max(maxn, t.n);
    shape = maxn <= 16 ? GEMM_SKINNY : GEMM_BIG;
    if (std::is_same<T, float>::value && shape == GEMM_BIG && g_tensor_cores) {
      shape = GEMM_TC;
      tc_mode = g_tensor_cores;
    }
    bool nn = true;
    for (const auto& e : ents) nn = nn && e.opA == 0 && e.opB == 0;
    skinny_nn = nn && maxn <= 16 && !force_tiled();
    nr = maxn;
    // Decided on the tasks as given: split_tasks() moves a task's beta to
    // its ordered sum and gives the parts beta zero.
    idempotent = true;
    for (const auto& t : tasks) idempotent = idempotent && t.beta == T(0);
    if (skinny_nn) split_tasks();
    if (skinny_nn) {
      // A task takes 256-row tiles when they leave no more padding rows
      // than 128-row tiles would, else 128-row tiles (two launches back to
      // back; padding rows are zero-filled copies whose tensor-core work is
      // skipped, but a mostly empty CTA still walks every stage).
      std::vector<int2> rt[2], alt[2];
      double rows = 0., elems = 0.;
      for (int ti = 0; ti < (int)tasks.size(); ti++) {
        const auto& t = tasks[ti];
        if (t.m <= 0 || t.n <= 0) continue;
        if (t.e0 == t.e1 && t.beta == T(1)) continue;
        const int n1 = skinny_rows_per_cta(0), n2 = skinny_rows_per_cta(1);
        const int wide = ((t.m + n2 - 1) / n2) * n2 == ((t.m + n1 - 1) / n1) * n1 ? 1 : 0;
        const int rb = skinny_rows_per_cta(wide);
        for (int a = 0; a < (t.m + rb - 1) / rb; a++) rt[wide].push_back(make_int2(ti, a));
        for (int w = 0; w < 2; w++)
          for (int a = 0; a < (t.m + skinny_rows_per_cta(w) - 1) / skinny_rows_per_cta(w); a++)
            alt[w].push_back(make_int2(ti, a));
        rows += t.m;
        for (int e = t.e0; e < t.e1; e++) elems += (double)t.m * ents[e].k;
      }
      d_rtiles.upload(rt[0]);
      d_rtiles_w.upload(rt[1]);
      d_alt_n.upload(alt[0]);
      d_alt_w.upload(alt[1]);
      tkey = tune_key(name, (int)sizeof(T), nr, (double)tasks.size(), rows, elems);
      bulk_ok = sizeof(T) == 8 && nr > 4;
      for (const auto& e : ents)
        bulk_ok = bulk_ok && (reinterpret_cast<uintptr_t>(e.A) & 15) == 0 && (e.lda & 1) == 0;
    }
    int bm = shape == GEMM_TC ? tc_gemm_tile() : gemm_tile_m(shape);
    int bn = shape == GEMM_TC ? tc_gemm_tile() : gemm_tile_n(shape);
    std::vector<TileRef> tiles;
    for (int ti = 0; ti < (int)tasks.size(); ti++) {
      const auto& t = tasks[ti];
      if (t.m <= 0 || t.n <= 0) continue;
      if (t.e0 == t.e1 && t.beta == T(1)) continue;  // nothing to do
      for (int a = 0; a < (t.m + bm - 1) / bm; a++)
        for (int b = 0; b < (t.n + bn - 1) / bn; b++) tiles.push_back(TileRef{ti, a, b});
    }
    ntiles = (int)tiles.size();
    flops = bytes = 0.;
    for (const auto& t : tasks) {
      if (t.m <= 0 || t.n <= 0) continue;
      bytes += (double)t.m * t.n * sizeof(T) * (t.beta == T(0) ? 1. : 2.);
      for (int e = t.e0; e < t.e1; e++) {
        flops += 2. * t.m * t.n * ents[e].k;
        bytes += ((double)t.m * ents[e].k + (double)ents[e].k * t.n) * sizeof(T);
      }
    }
    bytes += sum_bytes;
    d_tasks.upload(tasks);
    d_ents.upload(ents);
    d_tiles.upload(tiles);
    tasks.clear();
    tasks.shrink_to_fit();
    ents.clear();
    ents.shrink_to_fit();
  }
  // Spreads tasks with many entries over several CTAs: a task whose A
  // elements exceed an even share of the plan's total is cut at entry
  // boundaries into parts that write m x n partials; k_sum_parts adds them in
  // order into the task's C afterwards.  Upper tree levels have few boxes
  // with many large couplings, so without this a few CTAs would stream most
  // of the bytes.
  void split_tasks() {
    double total = 0.;
    for (const auto& t : tasks)
      for (int e = t.e0; e < t.e1; e++) total += (double)t.m * ents[e].k;
    // Plans with fewer row tiles than about four CTAs per SM (the upper
    // tree levels: U^T x, U y and the ULV substitution blocks of few large
    // boxes) are latency-bound on the streaming rate of single CTAs: there
    // an entry longer than a part is first cut along k into entries of a
    // multiple of 16 columns of A (rows of B; these plans are all NN), so
    // one-entry tasks spread over several CTAs too.  Larger plans keep
    // whole entries (partials would only add traffic).
    double rowtiles = 0.;
    for (const auto& t : tasks) rowtiles += (t.m + 127) / 128;
    constexpr double kCtaTarget = 4. * 148.;
    const bool cut_k = rowtiles < kCtaTarget;
    const double cap = cut_k ? std::max(total / kCtaTarget, 16384.) : std::max(total / 4096., 65536.);
    if (cut_k) {
      std::vector<GemmEntry<T>> cut;
      cut.reserve(ents.size());
      for (auto& t : tasks) {
        const int e0 = (int)cut.size();
        for (int e = t.e0; e < t.e1; e++) {
          const GemmEntry<T>& en = ents[e];
          const int mcta = std::min(t.m, 256);  // rows one CTA streams
          if (t.m <= 0 || (double)mcta * en.k <= cap || en.opA || en.opB) {
            cut.push_back(en);
            continue;
          }
          const int kc = std::max(16, (int)(cap / mcta) / 16 * 16);
          for (int k0 = 0; k0 < en.k; k0 += kc) {
            GemmEntry<T> piece = en;
            piece.A = en.A + (i64)k0 * en.lda;
            piece.B = en.B + k0;
            piece.k = std::min(kc, en.k - k0);
            cut.push_back(piece);
          }
        }
        t.e0 = e0;
        t.e1 = (int)cut.size();
      }
      ents.swap(cut);
    }
    std::vector<GemmTask<T>> out;
    struct Pending { int first; int parts; GemmTask<T> orig; i64 off; };
    std::vector<Pending> pend;
    i64 scratch = 0;
    for (const auto& t : tasks) {
      // Part weight: A elements one CTA streams (rows capped at a 256-row
      // tile when entries were cut, else the whole task's rows).
      const double mw = cut_k ? std::min(t.m, 256) : t.m;
      double w = 0.;
      for (int e = t.e0; e < t.e1; e++) w += mw * ents[e].k;
      if (w <= cap || t.e1 - t.e0 < 2 || t.m <= 0 || t.n <= 0) {
        out.push_back(t);
        continue;
      }
      Pending pd;
      pd.first = (int)out.size();
      pd.orig = t;
      pd.off = scratch;
      pd.parts = 0;
      int e = t.e0;
      while (e < t.e1) {
        GemmTask<T> part = t;
        part.e0 = e;
        double wp = 0.;
        while (e < t.e1 && (wp == 0. || wp + mw * ents[e].k <= cap)) {
          wp += mw * ents[e].k;
          e++;
        }
        part.e1 = e;
        part.beta = T(0);
        part.ldc = t.m;
        part.C = nullptr;  // set once the scratch exists
        out.push_back(part);
        pd.parts++;
      }
      scratch += (i64)pd.parts * t.m * t.n;
      pend.push_back(pd);
    }
    if (pend.empty()) return;
    parts_buf.alloc(scratch);
    std::vector<SumTask<T>> sums;
    for (const auto& pd : pend) {
      const i64 mn = (i64)pd.orig.m * pd.orig.n;
      for (int p = 0; p < pd.parts; p++) out[pd.first + p].C = parts_buf.p + pd.off + p * mn;
      SumTask<T> st_;
      st_.dst = pd.orig.C;
      st_.ldd = pd.orig.ldc;
      st_.src = parts_buf.p + pd.off;
      st_.m = pd.orig.m;
      st_.n = pd.orig.n;
      st_.parts = pd.parts;
      st_.beta = pd.orig.beta;
      sums.push_back(st_);
      sum_maxmn = std::max(sum_maxmn, (int)mn);
      sum_bytes += (double)(pd.parts + 1) * mn * sizeof(T);
    }
    tasks.swap(out);
    nsums = (int)sums.size();
    d_sums.upload(sums);
  }

  void run_skinny(int v, cudaStream_t st) const {
    const DVec<int2>& w = v == 0 ? d_rtiles_w : d_alt_w;
    const DVec<int2>& n = v == 0 ? d_rtiles : d_alt_n;
    int* be = (bulk_ok && g_cur) ? g_cur->d_tc_err : nullptr;
    if (be) g_cur->tc_pending = true;
    if (v != 1) ck(launch_skinny_nn<T>(nr, 1, d_tasks.p, d_ents.p, w.p, (int)w.n, st, be), "skinny_nn");
    if (v != 2) ck(launch_skinny_nn<T>(nr, 0, d_tasks.p, d_ents.p, n.p, (int)n.n, st, be), "skinny_nn");
    if (nsums) ck(launch_sum_parts<T>(d_sums.p, nsums, sum_maxmn, st), "sum_parts");
  }

  // Picks the streaming tiling (timing the variants if the bucket is new).
  void tune(cudaStream_t st) const {
    if (!skinny_nn || variant >= 0) return;
    if (!idempotent) {
      variant = 0;
      return;
    }
    const int v = tuned_variant(tkey, 3, st, [&](int x) { run_skinny(x, st); });
    if (!stream_capturing(st)) variant = v;
  }

  void run(cudaStream_t st) const {
    tune(st);
    Prof p(name, flops, bytes, st);
    if (skinny_nn) {
      run_skinny(variant < 0 ? 0 : variant, st);
    } else if (shape == GEMM_TC) {
      if constexpr (std::is_same<T, float>::value) {
        require(g_cur != nullptr, "tensor-core GEMM outside an API call");
        ck(launch_tc_gemm(d_tasks.p, d_ents.p, d_tiles.p, ntiles, tc_mode == 1 ? 1 : 0, g_cur->d_tc_err, st),
           "tc_gemm");
        g_cur->tc_pending = true;
      }
    } else if (std::is_same<T, double>::value && shape == GEMM_BIG && g_tensor_cores) {
      if constexpr (std::is_same<T, double>::value)
        ck(launch_dgemm(d_tasks.p, d_ents.p, d_tiles.p, ntiles, st), "dgemm");
    } else {
      ck(launch_seg_gemm<T>(shape, d_tasks.p, d_ents.p, d_tiles.p, ntiles, st), "seg_gemm");
    }
  }
};

// Host-built matrix-free apply plan (k_mf.cu): tasks over point sets,
// uploaded once per right-hand-side count and replayed.
struct MfPlan {
  std::vector<MfTask> tasks;
  std::vector<MfEntry> ents;
  std::vector<int2> tiles;
  DVec<MfTask> d_tasks;
  DVec<MfEntry> d_ents;
  DVec<int2> d_tiles;
  int nr = 0;
  const char* name = "mf_apply";
  double flops = 0., bytes = 0.;
  // Autotuned rows per thread (at most 4 right-hand sides): variant 0 = 2
  // rows, 1 = 1 row per thread; with more, variant 1 is the tensor-core
  // kernel over 32-row tiles.
  std::vector<int2> tiles1;
  DVec<int2> d_tiles1;
  std::string tkey;
  mutable int variant = -1;
  void add_task(const double* pts, int m, double* C, i64 ldc, double beta) {
    MfTask t;
    t.pts = pts; t.m = m; t.C = C; t.ldc = ldc; t.beta = beta;
    t.e0 = t.e1 = (int)ents.size();
    tasks.push_back(t);
  }
  void add_entry(const double* pts, int k, const double* B, i64 ldb, double alpha) {
    if (k <= 0) return;
    MfEntry e;
    e.pts = pts; e.k = k; e.B = B; e.ldb = ldb; e.alpha = alpha;
    ents.push_back(e);
    tasks.back().e1 = (int)ents.size();
    // 2 nr multiply-adds per pair (the kernel evaluation is extra work);
    // bytes: the entry's points and right-hand-side rows.
    flops += 2. * nr * (double)tasks.back().m * k;
    bytes += (24. + 8. * nr) * k;
  }
  void finalize() {
    const int bm = mf_rows_per_cta(2), bm1 = nr > 4 ? mf_dmma_rows_per_cta() : mf_rows_per_cta(1);
    tiles.clear();
    tiles1.clear();
    double rows = 0.;
    for (size_t t = 0; t < tasks.size(); t++) {
      bytes += (24. + 8. * nr) * tasks[t].m;
      rows += tasks[t].m;
      for (int r = 0; r < tasks[t].m; r += bm) tiles.push_back(make_int2((int)t, r / bm));
      for (int r = 0; r < tasks[t].m; r += bm1) tiles1.push_back(make_int2((int)t, r / bm1));
    }
    d_tasks.upload(tasks);
    d_ents.upload(ents);
    d_tiles.upload(tiles);
    d_tiles1.upload(tiles1);
    tkey = tune_key(name, 8, nr, (double)tasks.size(), rows, flops / (2. * nr));
  }
  void launch(const KernelParams& kp, int v, cudaStream_t st) const {
    if (v == 1)
      ck(launch_mf_apply(kp, nr, 1, d_tasks.p, d_ents.p, d_tiles1.p, (int)tiles1.size(), st), name);
    else
      ck(launch_mf_apply(kp, nr, 2, d_tasks.p, d_ents.p, d_tiles.p, (int)tiles.size(), st), name);
  }
  void tune(const KernelParams& kp, cudaStream_t st) const {
    if (variant >= 0) return;
    if (nr > 4) {  // one kernel (tensor cores, 128-row tiles): nothing to choose
      variant = 1;
      return;
    }
    const int v = tuned_variant(tkey, 2, st, [&](int x) { launch(kp, x, st); });  // beta 0: repeatable
    if (!stream_capturing(st)) variant = v;
  }
  void run(const KernelParams& kp, cudaStream_t st) const {
    tune(kp, st);
    Prof p(name, flops, bytes, st);
    launch(kp, variant < 0 ? (nr > 4 ? 1 : 0) : variant, st);
  }
};

// BF16 substitution plan: the tasks of one FP32 GemmPlan with each entry's
// block packed to BF16 (per-block power-of-two scale), applied by
// k_stream_bf16.
struct BfPlan {
  std::vector<GemmTask<float>> tasks;
  std::vector<BfEntry> ents;
  std::vector<int2> tiles;
  DVec<GemmTask<float>> d_tasks;
  DVec<BfEntry> d_ents;
  DVec<int2> d_tiles;
  int nr = 0;
  double flops = 0., bytes = 0.;
  // Split tasks (as GemmPlan::split_tasks): partials in parts_buf, summed
  // in order into the task's output by k_sum_parts.
  DVec<float> parts_buf;
  DVec<SumTask<float>> d_sums;
  int nsums = 0, sum_maxmn = 0;
  void finalize() {
    split();
    const int bm = bf16_rows_per_cta();
    tiles.clear();
    for (size_t t = 0; t < tasks.size(); t++)
      for (int r = 0; r < tasks[t].m; r += bm) tiles.push_back(make_int2((int)t, r / bm));
    d_tasks.upload(tasks);
    d_ents.upload(ents);
    d_tiles.upload(tiles);
  }
  // Plans with fewer 256-row tiles than about four CTAs per SM (the upper
  // tree levels: few large boxes) cut their entries along k into pieces of
  // a multiple of 32 columns and spread each task over several CTAs.
  void split() {
    double rowtiles = 0., total = 0.;
    for (const auto& t : tasks) {
      rowtiles += (t.m + 255) / 256;
      for (int e = t.e0; e < t.e1; e++) total += (double)std::min(t.m, 256) * ents[e].k;
    }
    constexpr double kCtaTarget = 4. * 148.;
    if (rowtiles >= kCtaTarget || tasks.empty()) return;
    const double cap = std::max(total / kCtaTarget, 16384.);
    std::vector<GemmTask<float>> out;
    std::vector<BfEntry> cut;
    std::vector<SumTask<float>> sums;
    i64 scratch = 0;
    std::vector<std::pair<size_t, i64>> scr;  // (first part index in out, scratch offset) per split task
    for (const auto& t : tasks) {
      const int mw = std::min(t.m, 256);
      // pieces of this task's entries
      std::vector<BfEntry> pcs;
      for (int e = t.e0; e < t.e1; e++) {
        const BfEntry& en = ents[e];
        if (en.k <= 0) continue;
        const int kc = std::max(32, (int)(cap / mw) / 32 * 32);
        for (int k0 = 0; k0 < en.k; k0 += kc) {
          BfEntry p = en;
          p.A = en.A + (i64)k0 * en.lda;
          p.B = en.B + k0;
          p.k = std::min(kc, en.k - k0);
          pcs.push_back(p);
        }
      }
      double w = 0.;
      for (const auto& p : pcs) w += (double)mw * p.k;
      if (w <= cap || pcs.size() < 2 || t.m <= 0 || t.n <= 0) {
        GemmTask<float> nt = t;
        nt.e0 = (int)cut.size();
        cut.insert(cut.end(), pcs.begin(), pcs.end());
        nt.e1 = (int)cut.size();
        out.push_back(nt);
        continue;
      }
      const size_t first = out.size();
      int parts = 0;
      size_t q = 0;
      while (q < pcs.size()) {
        GemmTask<float> part = t;
        part.e0 = (int)cut.size();
        double wp = 0.;
        while (q < pcs.size() && (wp == 0. || wp + (double)mw * pcs[q].k <= cap)) {
          wp += (double)mw * pcs[q].k;
          cut.push_back(pcs[q++]);
        }
        part.e1 = (int)cut.size();
        part.beta = 0.f;
        part.ldc = t.m;
        part.C = nullptr;  // set once the scratch exists
        out.push_back(part);
        parts++;
      }
      SumTask<float> sm;
      sm.dst = t.C;
      sm.ldd = t.ldc;
      sm.src = nullptr;
      sm.m = t.m;
      sm.n = t.n;
      sm.parts = parts;
      sm.beta = t.beta;
      sums.push_back(sm);
      scr.emplace_back(first, scratch);
      scratch += (i64)parts * t.m * t.n;
      sum_maxmn = std::max(sum_maxmn, t.m * t.n);
      bytes += (double)(parts + 1) * t.m * t.n * sizeof(float);
    }
    if (sums.empty()) return;
    parts_buf.alloc(scratch);
    for (size_t i = 0; i < sums.size(); i++) {
      const i64 mn = (i64)sums[i].m * sums[i].n;
      sums[i].src = parts_buf.p + scr[i].second;
      for (int p = 0; p < sums[i].parts; p++) out[scr[i].first + p].C = parts_buf.p + scr[i].second + p * mn;
    }
    tasks.swap(out);
    ents.swap(cut);
    nsums = (int)sums.size();
    d_sums.upload(sums);
  }
  void run(cudaStream_t st) const {
    Prof p("bf16_precond", flops, bytes, st);
    ck(launch_stream_bf16(nr, d_tasks.p, d_ents.p, d_tiles.p, (int)tiles.size(), st), "bf16_precond");
    if (nsums) ck(launch_sum_parts<float>(d_sums.p, nsums, sum_maxmn, st), "sum_parts");
  }
};

template <typename T>
struct CopyPlan {
  std::vector<CopyEntry<T>> ents;
  DVec<CopyEntry<T>> d;
  int n = 0;
  void add(const T* src, i64 lds, T* dst, i64 ldd, int m, int nn, int trans = 0) {
    if (m <= 0 || nn <= 0) return;
    CopyEntry<T> e;
    e.src = src; e.dst = dst; e.lds = lds; e.ldd = ldd; e.m = m; e.n = nn; e.trans = trans;
    ents.push_back(e);
  }
  void finalize() {
    n = (int)ents.size();
    bytes = 0.;
    for (const auto& e : ents) bytes += 2. * e.m * e.n * sizeof(T);
    d.upload(ents);
    ents.clear();
    ents.shrink_to_fit();
  }
  double bytes = 0.;
  void run(cudaStream_t st) const {
    Prof p("batched_copy", 0., bytes);
    ck(launch_batched_copy<T>(d.p, n, st), "batched_copy");
  }
};

}  // namespace h2b

namespace h2b {

template <typename T>
struct Level {
  int l = 0;
  i64 nodes = 0, gbegin = 0;
  std::vector<i64> arow, acol, crow, ccol, diag;
  std::vector<i64> dims, ranks, xoff, zoff, qoff, aoff, coff;
  // Leading dimension of box i's coupling blocks C_ij (rank_i x rank_j at
  // coff): rank_i rounded up to 4, so that every column starts on a
  // 32-byte boundary and the streaming applies copy whole 16-byte vectors.
  std::vector<i64> cld;
  i64 lenX = 0, lenZ = 0, maxM = 0;
  DVec<i64> d_dims, d_ranks, d_xoff, d_qoff;
  DVec<double> pts;  // lenX x 3, skeleton-first after the basis
  DVec<T> Q, R, A, C;
  std::vector<i64> na_off, na_ld;  // destination of each near block's ss part in the parent A
  // factorization results
  DVec<T> B, invT;
  std::vector<i64> boff, ioff;
  DVec<int> ipiv, info;
  int info_count = 0;
  // Transposed copies for the multi-RHS applies, so every apply streams
  // its matrix as stored: Qt = Q[:, :rank]^T (rank x M per box at qtoff,
  // leading dimension rank rounded up to 4) for the upward pass,
  // Rt = (factor's R slot)^T (M x M at qoff) for the ULV forward
  // substitution.
  DVec<T> Qt, Rt;
  std::vector<i64> qtoff;
  // per-nrhs vectors
  DVec<T> vX, vZ, vW;
};

template <typename T>
void batched_gemm(int64_t batch, int64_t nterms, int64_t m, int64_t n, int64_t k, int opA, int opB,
                         double alpha, const T* A, int64_t lda, int64_t sA, const T* B, int64_t ldb, int64_t sB,
                         double beta, T* C, int64_t ldc, int64_t sC, cudaStream_t st) {
  GemmPlan<T> g;
  g.name = "batched_gemm";
  for (int64_t b = 0; b < batch; b++) {
    g.add_task(C + b * sC, ldc, (int)m, (int)n, (T)beta);
    for (int64_t t = 0; t < nterms; t++)
      g.add_entry(A + (b * nterms + t) * sA, lda, opA, B + (b * nterms + t) * sB, ldb, opB, (int)k, (T)alpha);
  }
  g.finalize();
  g.run(st);
  check_tc(g_cur);
}


struct SolveGraph;  // a captured, instantiated GMRES solve kept for replay (gmres_graph)

static uint64_t next_solver_uid() {
  static std::atomic<uint64_t> n{0};
  return ++n;
}

class SolverBase {
 public:
  virtual ~SolverBase() {}
  // Identity for caches (never reused) and a generation bumped whenever the
  // solver's plans, per-nrhs vectors or factors change: a captured solve is
  // replayed only while both solvers' generations are those it captured.
  uint64_t uid = next_solver_uid();
  uint64_t gen = 0;
  std::shared_ptr<SolveGraph> solve_graph;
  virtual i64 lenX() const = 0;
  virtual i64 nlevels() const = 0;
  virtual void matvec(i64 nrhs, double* dX, i64 ldx) = 0;
  virtual void factorize(int* info) = 0;
  virtual void precondition(i64 nrhs, double* dX, i64 ldx) = 0;
  // Builds the per-nrhs vectors and the matvec / substitution plans now, so
  // that later applies only launch (required before a graph capture).
  virtual void prepare(i64 nrhs) = 0;
  virtual void level_dims(i64 l, i64* dims, i64* ranks) const = 0;
  virtual i64 export_size(i64 l, int what) const = 0;
  virtual void export_to(i64 l, int what, double* out) = 0;
  h2dev_handle_s* h = nullptr;
  // Helmholtz: the solver holds the real symmetric form S of the complex
  // matrix K over two unknowns per body (KERNEL_HELMHOLTZ), S conj(x) = K x.
  // The entry points conjugate their vectors so that callers see K itself.
  bool complex_form = false;
};

struct BuildArgs {
  KernelParams kp;
  double epi;
  i64 rank, leveled_rank, levels, nbodies, samples;
  double theta;
  std::vector<Cell> cells;
  const double* bodies;
};

template <typename T>
class Solver : public SolverBase {
 public:
  KernelParams kp;
  double epi = 0.;
  bool fix_rank = false;
  i64 rank = 0, leveled_rank = 0, levels = 0, N = 0, samples = 0;
  std::vector<Cell> cells;
  DVec<double> bodies;
  std::vector<Level<T>> L;
  bool factored = false;
  // Matrix-free operator (H2DEV_OPT_MATRIX_FREE, ID mode, FP64): the leaf
  // near blocks and the couplings are evaluated inside the matvec, never
  // stored, and the upper-level near blocks (read only by a factorization)
  // are not assembled.
  bool matrix_free = false;
  MfPlan mf_leaf, mf_far;
  int sampling_mode = 0;                 // 0: strided, 1: level-geometric far-list cap
  std::vector<std::vector<i64>> gstart;  // per cell: first range of each level group
  // per-nrhs state
  i64 cur_nrhs = -1;
  DVec<T> vin, vout;
  GemmPlan<T> mv_leaf, mv_far, mv_qw;  // leaf: near field (A_ij x_j); qw: + U W at the leaves
  std::vector<GemmPlan<T>> mv_up, mv_down;
  std::vector<GemmPlan<T>> pc_fx, pc_fz, pc_bx, pc_by;
  // BF16 substitution (H2DEV_OPT_PRECOND_BF16, FP32 solvers): packed
  // copies of the streamed blocks and the plans that read them.
  bool precond_bf16 = false;
  DVec<__nv_bfloat16> bf_pool;
  DVec<float> bf_scales;
  std::vector<BfPlan> bf_fx, bf_fz, bf_bx, bf_by;
  std::vector<CopyPlan<T>> pc_fcopy, pc_bcopy;
  bool mv_built = false, pc_built = false;

  cudaStream_t st() const { return h->stream; }
  i64 lenX() const override { return N; }
  i64 nlevels() const override { return levels; }

  void build(const BuildArgs& a) {
    kp = a.kp;
    epi = a.epi;
    fix_rank = (a.epi == 0.);
    rank = a.rank;
    leveled_rank = a.leveled_rank;
    levels = a.levels;
    N = a.nbodies;
    samples = a.samples;
    sampling_mode = h->sampling_mode;
    matrix_free = h->matrix_free && !fix_rank && std::is_same<T, double>::value;
    precond_bf16 = h->precond_bf16 && std::is_same<T, float>::value;
    cells = a.cells;
    {
      std::vector<double> hb(a.bodies, a.bodies + 3 * N);
      bodies.upload(hb);
    }
    PairCSR nearL = build_pair_csr('N', cells, a.theta);
    PairCSR farL = build_pair_csr('F', cells, a.theta);
    PairCSR sampL = fix_rank ? build_pair_csr('F', cells, 0.) : farL;

    // Far-body ranges per cell: the parent's list then the cell's own far
    // boxes (h-matrix.cpp:83-98, 122-127); the root has none.
    i64 ncells = (i64)cells.size();
    std::vector<std::vector<std::pair<i64, i64>>> ranges(ncells);
    gstart.assign(ncells, std::vector<i64>());
    for (i64 c = 1; c < ncells; c++) {
      i64 parent = (c - 1) / 2;
      ranges[c] = ranges[parent];
      gstart[c] = gstart[parent];
      gstart[c].push_back((i64)ranges[parent].size());
      for (i64 k = sampL.row[c]; k < sampL.row[c + 1]; k++) {
        i64 x = sampL.col[k];
        ranges[c].emplace_back(cells[x].body[0], cells[x].body[1]);
      }
    }
    if (ncells) ranges[0].clear();

    L.resize(levels + 1);
    for (i64 l = 0; l <= levels; l++) {
      Level<T>& lv = L[l];
      lv.l = (int)l;
      lv.gbegin = ((i64)1 << l) - 1;
      lv.nodes = (i64)1 << l;
      i64 g0 = lv.gbegin, g1 = g0 + lv.nodes;
      lv.arow.assign(lv.nodes + 1, 0);
      lv.crow.assign(lv.nodes + 1, 0);
      for (i64 i = 0; i < lv.nodes; i++) {
        for (i64 k = nearL.row[g0 + i]; k < nearL.row[g0 + i + 1]; k++) lv.acol.push_back(nearL.col[k] - g0);
        for (i64 k = farL.row[g0 + i]; k < farL.row[g0 + i + 1]; k++) lv.ccol.push_back(farL.col[k] - g0);
        lv.arow[i + 1] = (i64)lv.acol.size();
        lv.crow[i + 1] = (i64)lv.ccol.size();
      }
      (void)g1;
      lv.diag.assign(lv.nodes, -1);
      for (i64 i = 0; i < lv.nodes; i++)
        for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++)
          if (lv.acol[k] == i) lv.diag[i] = k;
      lv.na_off.assign(lv.acol.size(), -1);
      lv.na_ld.assign(lv.acol.size(), 0);
    }
    // Sample lists of every level, leaves first, on one background thread
    // (each level's list is itself built by up to 8 threads), so that the
    // host computes level l-1's lists while the device works on level l.
    // The futures are taken (or, on an error, drained) before this returns.
    std::thread ahead;
    std::vector<std::promise<LevelSamples>> prom;
    if (sampling_mode != 2) {
      prom.resize(levels + 1);
      sample_ahead.resize(levels + 1);
      for (i64 l = 0; l <= levels; l++) sample_ahead[l] = prom[l].get_future();
      ahead = std::thread([this, &prom, &ranges]() {
        for (i64 l = levels; l >= 0; l--) {
          try {
            prom[l].set_value(level_samples(l, ranges));
          } catch (...) {
            prom[l].set_exception(std::current_exception());
          }
        }
      });
    }
    struct Join {
      std::thread& t;
      std::vector<std::future<LevelSamples>>& f;
      ~Join() {
        if (t.joinable()) t.join();
        f.clear();
      }
    } join{ahead, sample_ahead};
    for (i64 l = levels; l >= 0; l--) construct_level(l, ranges);
    if (fix_rank) {
      // The host-side rank rule must agree with the ranks the device chose
      // (plans and offsets were sized from it).
      for (i64 l = 0; l <= levels; l++)
        if (L[l].d_ranks.n) require(L[l].d_ranks.download(st()) == L[l].ranks, "fixed-rank rule disagrees with the device");
    }
    check_tc(h);
  }

  double level_epi(i64 l) const {
    return fix_rank ? (double)((levels - l) * leveled_rank + rank) : epi;
  }

  // h2matrix.cpp:72-249 for one level.
  // Ranks of fixed-rank bases (epi >= 1), by the rule k_basis_finish
  // applies on the device: min(K, M, floor(epi)) with K the box's sample
  // rows (0 when K or M is 0).  Knowing them on the host spares the level a
  // device-to-host synchronisation before its completion plans are built.
  static std::vector<i64> fixed_rank_rule(const std::vector<i64>& dims, const std::vector<i64>& krows, double e) {
    std::vector<i64> r(dims.size(), 0);
    const i64 cap = (i64)std::floor(e);
    for (size_t i = 0; i < dims.size(); i++) {
      if (dims[i] == 0 || krows[i] == 0) continue;
      r[i] = std::min(std::min(krows[i], dims[i]), cap);
    }
    return r;
  }

  // Far-sample index lists of one level (strided or level-geometric cap):
  // every box's list concatenated in box order, and the per-box counts;
  // host work that depends only on the tree, so build() computes all levels
  // ahead on a background thread while the device constructs the levels
  // below.
  struct LevelSamples {
    std::vector<int> sidx;
    std::vector<i64> cnt;
  };
  std::vector<std::future<LevelSamples>> sample_ahead;

  LevelSamples level_samples(i64 l, const std::vector<std::vector<std::pair<i64, i64>>>& ranges) const {
    const i64 nodes = (i64)1 << l, g0 = nodes - 1;
    LevelSamples out;
    out.cnt.assign(nodes, 0);
    const int nth = (int)std::max<i64>(1, std::min<i64>({8, (i64)std::thread::hardware_concurrency(), nodes / 16}));
    std::vector<std::vector<int>> part(nth);
    auto work = [&](int t) {
      std::vector<int> tmp;
      for (i64 i = nodes * t / nth; i < nodes * (t + 1) / nth; i++) {
        if (sampling_mode == 1)
          sample_far_list_geometric(ranges[g0 + i], gstart[g0 + i], samples, tmp);
        else
          sample_far_list(ranges[g0 + i], samples, tmp);
        part[t].insert(part[t].end(), tmp.begin(), tmp.end());
        out.cnt[i] = (i64)tmp.size();
      }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nth; t++) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    size_t tot = 0;
    for (auto& v : part) tot += v.size();
    out.sidx.reserve(tot);
    for (auto& v : part) out.sidx.insert(out.sidx.end(), v.begin(), v.end());
    return out;
  }

  LevelSamples take_samples(i64 l, const std::vector<std::vector<std::pair<i64, i64>>>& ranges) {
    if ((i64)sample_ahead.size() > l && sample_ahead[l].valid()) return sample_ahead[l].get();
    return level_samples(l, ranges);
  }

  void construct_level(i64 l, const std::vector<std::vector<std::pair<i64, i64>>>& ranges) {
    Level<T>& lv = L[l];
    Level<T>* low = (l < levels) ? &L[l + 1] : nullptr;
    const i64 nodes = lv.nodes;
    const i64 g0 = lv.gbegin;
    lv.dims.assign(nodes, 0);
    for (i64 i = 0; i < nodes; i++)
      lv.dims[i] = low ? low->ranks[2 * i] + low->ranks[2 * i + 1] : cells[g0 + i].body[1] - cells[g0 + i].body[0];
    lv.xoff.assign(nodes + 1, 0);
    lv.qoff.assign(nodes + 1, 0);
    for (i64 i = 0; i < nodes; i++) {
      lv.xoff[i + 1] = lv.xoff[i] + lv.dims[i];
      lv.qoff[i + 1] = lv.qoff[i] + lv.dims[i] * lv.dims[i];
      lv.maxM = std::max(lv.maxM, lv.dims[i]);
    }
    require(lv.maxM <= 2048, "box dimension above 2048 is not supported");
    lv.lenX = lv.xoff[nodes];
    i64 nA = (i64)lv.acol.size();
    lv.aoff.assign(nA + 1, 0);
    for (i64 i = 0; i < nodes; i++)
      for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) lv.aoff[k + 1] = lv.aoff[k] + lv.dims[i] * lv.dims[lv.acol[k]];
    lv.d_dims.upload(lv.dims);
    lv.d_xoff.upload(lv.xoff);
    lv.d_qoff.upload(lv.qoff);
    lv.pts.alloc(3 * lv.lenX);
    lv.Q.alloc(lv.qoff[nodes]);
    lv.R.alloc(lv.qoff[nodes]);
    lv.A.alloc(matrix_free ? 0 : lv.aoff[nA]);
    lv.Q.zero(st());
    lv.R.zero(st());
    lv.A.zero(st());
    lv.ranks.assign(nodes, 0);

    if (lv.lenX > 0) {
      if (!low) {
        ck(cudaMemcpyAsync(lv.pts.p, bodies.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, st()), "pts");
        ck(launch_set_identity<T>(lv.Q.p, lv.d_qoff.p, lv.d_dims.p, (int)nodes, st()), "identity");
        std::vector<GenTask> gt;
        for (i64 i = 0; i < nodes; i++)
          for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) {
            i64 j = lv.acol[k];
            GenTask t;
            t.bi = bodies.p + 3 * cells[g0 + i].body[0];
            t.bj = bodies.p + 3 * cells[g0 + j].body[0];
            t.m = (int)lv.dims[i];
            t.n = (int)lv.dims[j];
            t.out_off = lv.aoff[k];
            t.ld = lv.dims[i];
            gt.push_back(t);
          }
        if (matrix_free) gt.clear();
        DVec<GenTask> dg;
        dg.upload(gt);
        if (!gt.empty()) {
          Prof pf("gen_near_blocks", 0., (double)lv.aoff[nA] * sizeof(T));
          // FP64 blocks use the std::hypot-exact distance (bit-exact with the
          // reference); FP32 blocks the rsqrt path, rounded to FP32 anyway.
          ck(launch_gen_blocks<T>(kp, dg.p, (int)gt.size(), gen_max_rows(gt), lv.A.p, st(), sizeof(T) == 4 ? 1 : 0,
                                  gen_err()),
             "gen near");
        }
      } else {
        CopyPlan<double> pcopy;
        CopyPlan<T> qcopy, acopy;
        for (i64 i = 0; i < nodes; i++) {
          const i64 M = lv.dims[i];
          i64 offy = 0;
          for (i64 y = 2 * i; y <= 2 * i + 1; y++) {
            const i64 ny = low->ranks[y];
            pcopy.add(low->pts.p + 3 * low->xoff[y], 3 * ny, lv.pts.p + 3 * (lv.xoff[i] + offy), 3 * ny, (int)(3 * ny), 1);
            qcopy.add(low->R.p + low->qoff[y], low->dims[y], lv.Q.p + lv.qoff[i] + offy + offy * M, M, (int)ny, (int)ny);
            if (M > 0)
              for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) {
                i64 j = lv.acol[k];
                i64 offx = 0;
                for (i64 x = 2 * j; x <= 2 * j + 1; x++) {
                  const i64 nx = low->ranks[x];
                  i64 lowN = -1, lowC = -1;
                  for (i64 q = low->arow[y]; q < low->arow[y + 1]; q++)
                    if (low->acol[q] == x) lowN = q;
                  if (lowN < 0)
                    for (i64 q = low->crow[y]; q < low->crow[y + 1]; q++)
                      if (low->ccol[q] == x) lowC = q;
                  if (lowN >= 0) {
                    low->na_off[lowN] = lv.aoff[k] + offy + offx * M;
                    low->na_ld[lowN] = M;
                  } else if (lowC >= 0 && !matrix_free) {
                    acopy.add(low->C.p + low->coff[lowC], low->cld[y], lv.A.p + lv.aoff[k] + offy + offx * M, M, (int)ny, (int)nx);
                  }
                  offx += nx;
                }
              }
            offy += ny;
          }
        }
        pcopy.finalize();
        qcopy.finalize();
        acopy.finalize();
        pcopy.run(st());
        qcopy.run(st());
        acopy.run(st());
      }

      // Shared basis of every box (compute_basis, h2matrix.cpp:195-200).
      // Far-sample lists of all boxes, built by up to 8 host threads over
      // contiguous box ranges and concatenated in box order.
      std::vector<int> sidx;
      std::vector<i64> soff(nodes + 1, 0), krows(nodes, 0);
      // Sketch mode (H2DEV_OPT_SAMPLING = 2): every far body, as ranges of
      // the tree-sorted body array per box (start, running count).
      const bool sketch = sampling_mode == 2;
      std::vector<i64> roff, rstart, rend;
      if (sketch) {
        // samples <= 0: every far body.  samples > 0: the far boxes of this
        // level and the two above it in full (they hold the numerical rank)
        // plus `samples` strided bodies of the farther list, whose
        // interactions are smooth -- the whole far field's accuracy at a
        // cost that no longer grows with N.
        roff.assign(nodes + 1, 0);
        std::vector<int> tmp;
        for (i64 i = 0; i < nodes; i++) {
          const auto& rl = ranges[g0 + i];
          const auto& gs = gstart[g0 + i];
          size_t cut = 0;
          if (samples > 0 && gs.size() >= 3) cut = (size_t)gs[gs.size() - 3];
          i64 cnt = 0;
          for (size_t q = cut; q < rl.size(); q++) {
            cnt += rl[q].second - rl[q].first;
            rstart.push_back(rl[q].first);
            rend.push_back(cnt);
          }
          if (cut > 0) {
            std::vector<std::pair<i64, i64>> farther(rl.begin(), rl.begin() + cut);
            sample_far_list(farther, samples, tmp);
            for (int b : tmp) {
              cnt += 1;
              rstart.push_back(b);
              rend.push_back(cnt);
            }
          }
          roff[i + 1] = (i64)rstart.size();
          soff[i + 1] = soff[i] + cnt;
          krows[i] = std::min<i64>(lv.dims[i], cnt);
        }
      } else {
        // Computed ahead by the background thread started in build() (or
        // here, when none runs).
        LevelSamples ls = take_samples(l, ranges);
        for (i64 i = 0; i < nodes; i++) {
          soff[i + 1] = soff[i] + ls.cnt[i];
          krows[i] = std::min<i64>(lv.dims[i], ls.cnt[i]);
        }
        sidx.swap(ls.sidx);
      }
      DVec<int> d_sidx, d_perm, d_nonzero;
      DVec<i64> d_soff, d_krows;
      DVec<double> d_maxpiv;
      d_sidx.upload(sidx);
      d_soff.upload(soff);
      d_krows.upload(krows);
      d_perm.alloc(lv.lenX);
      d_nonzero.alloc(nodes);
      d_maxpiv.alloc(nodes);
      lv.d_ranks.alloc(nodes);
      const double e = level_epi(l);
      const bool orth = 1. <= e;
      i64 cap = -1;
      if (e >= 1.) cap = (i64)std::floor(e);
      if (orth && h->basis_mode == 0 && !sketch) {
        basis_gram(lv, low == nullptr, soff, d_sidx, d_krows, d_perm, d_maxpiv, d_nonzero, e, cap);
      } else {
        DVec<T> Rws;
        Rws.alloc(lv.qoff[nodes]);
        Rws.zero(st());
        {
          double fl = 0.;
          for (i64 i = 0; i < nodes; i++) {
            double S = (double)(soff[i + 1] - soff[i]), Md = (double)lv.dims[i];
            fl += S >= Md ? 2. * S * Md * Md - 2. / 3. * Md * Md * Md : 2. * Md * S * S - 2. / 3. * S * S * S;
          }
          if (sketch) {
            // Y = Omega XF over the whole far list (k_sketch.cu), or XF
            // itself where the list has at most M bodies.
            const int tm = sketch_tile_rows(), tn = sketch_tile_cols();
            std::vector<int4> tiles;
            double sfl = 0.;
            for (i64 i = 0; i < nodes; i++) {
              const i64 M = lv.dims[i], S = soff[i + 1] - soff[i];
              if (M == 0 || S == 0) continue;
              const i64 rows = std::min(M, S);
              for (i64 a = 0; a < (rows + tm - 1) / tm; a++)
                for (i64 c = 0; c < (M + tn - 1) / tn; c++) tiles.push_back(make_int4((int)i, (int)a, (int)c, 0));
              if (S > M) sfl += 2. * (double)M * (double)M * (double)S;
            }
            DVec<i64> d_roff, d_rstart, d_rend;
            DVec<int4> d_tiles;
            d_roff.upload(roff);
            d_rstart.upload(rstart);
            d_rend.upload(rend);
            d_tiles.upload(tiles);
            Prof pf("sketch", sfl, 24. * (double)soff[nodes]);
            ck(launch_sketch<T>(kp, bodies.p, lv.pts.p, lv.d_xoff.p, lv.d_dims.p, lv.d_qoff.p, d_roff.p, d_rstart.p,
                                d_rend.p, d_tiles.p, (int)tiles.size(), Rws.p, st()),
               "sketch");
          } else {
            Prof pf("sample_tsqr", fl, (double)sidx.size() * 28.);
            ck(launch_sample_tsqr<T>(kp, bodies.p, lv.pts.p, lv.d_xoff.p, lv.d_dims.p, d_sidx.p, d_soff.p, Rws.p,
                                     lv.d_qoff.p, (int)nodes, (int)lv.maxM, st()),
               "sample_tsqr");
          }
        }
        {
          double fl = 0.;
          for (i64 i = 0; i < nodes; i++) {
            double K = (double)krows[i], Md = (double)lv.dims[i];
            double st_ = std::min(K, Md);
            if (cap >= 0) st_ = std::min(st_, (double)cap);
            fl += 4. * K * Md * st_ - 2. * (K + Md) * st_ * st_ + 4. / 3. * st_ * st_ * st_;
          }
          Prof pf("cpqr", fl, 0.);
          ck(launch_cpqr<T>(lv.d_dims.p, d_krows.p, Rws.p, lv.d_qoff.p, d_perm.p, lv.d_xoff.p, d_maxpiv.p,
                            d_nonzero.p, cap, (int)nodes, (int)lv.maxM, st()),
             "cpqr");
        }
        DVec<T> taus;
        if (orth) taus.alloc(std::max<i64>(1, lv.lenX));
        {
          Prof pfin("basis_finish", 0., (double)lv.qoff[nodes] * sizeof(T) * 3.);
          ck(launch_basis_finish<T>(lv.d_dims.p, d_krows.p, Rws.p, lv.Q.p, lv.R.p, lv.d_qoff.p, d_perm.p,
                                    lv.d_xoff.p, d_maxpiv.p, d_nonzero.p, lv.pts.p, lv.d_ranks.p, e, orth ? 1 : 0,
                                    low ? 0 : 1, (int)nodes, (int)lv.maxM, st(), orth ? taus.p : nullptr),
             "basis_finish");
        }
        if (orth) blocked_orth_qr<T>(lv, Rws.p, lv.Q.p, lv.R.p, taus.p, fixed_rank_rule(lv.dims, krows, e), low == nullptr);
      }
      lv.ranks = orth ? fixed_rank_rule(lv.dims, krows, e) : lv.d_ranks.download(st());
    } else {
      lv.d_ranks.alloc(nodes);
      lv.d_ranks.zero(st());
    }

    lv.zoff.assign(nodes + 1, 0);
    for (i64 i = 0; i < nodes; i++) lv.zoff[i + 1] = lv.zoff[i] + lv.ranks[i];
    lv.lenZ = lv.zoff[nodes];
    i64 nC = (i64)lv.ccol.size();
    lv.coff.assign(nC + 1, 0);
    lv.cld.assign(nodes, 0);
    for (i64 i = 0; i < nodes; i++) {
      lv.cld[i] = (lv.ranks[i] + 3) / 4 * 4;
      for (i64 k = lv.crow[i]; k < lv.crow[i + 1]; k++) lv.coff[k + 1] = lv.coff[k] + lv.cld[i] * lv.ranks[lv.ccol[k]];
    }
    lv.C.alloc(matrix_free ? 0 : lv.coff[nC]);
    if (lv.lenZ > 0 && nC > 0 && !matrix_free) {
      // Couplings (h2matrix.cpp:222-242): K(S_y, S_x) on the skeletons,
      // scaled by R_y on the left and R_x^T on the right in orthogonal mode.
      const bool orth = 1. <= level_epi(l);
      DVec<T> K;
      T* kout = lv.C.p;
      if (orth) {
        K.alloc(lv.coff[nC]);
        kout = K.p;
      }
      std::vector<GenTask> gt;
      for (i64 i = 0; i < nodes; i++)
        for (i64 k = lv.crow[i]; k < lv.crow[i + 1]; k++) {
          i64 x = lv.ccol[k];
          GenTask t;
          t.bi = lv.pts.p + 3 * lv.xoff[i];
          t.bj = lv.pts.p + 3 * lv.xoff[x];
          t.m = (int)lv.ranks[i];
          t.n = (int)lv.ranks[x];
          t.out_off = lv.coff[k];
          t.ld = lv.cld[i];
          gt.push_back(t);
        }
      DVec<GenTask> dg;
      dg.upload(gt);
      {
        Prof pf("gen_couplings", 0., (double)lv.coff[nC] * sizeof(T));
        ck(launch_gen_blocks<T>(kp, dg.p, (int)gt.size(), gen_max_rows(gt), kout, st(), sizeof(T) == 4 ? 1 : 0,
                                gen_err()),
           "gen couplings");
      }
      if (orth) {
        DVec<T> T1;
        T1.alloc(lv.coff[nC]);
        GemmPlan<T> g1, g2;
        for (i64 i = 0; i < nodes; i++)
          for (i64 k = lv.crow[i]; k < lv.crow[i + 1]; k++) {
            i64 x = lv.ccol[k];
            int ry = (int)lv.ranks[i], rx = (int)lv.ranks[x];
            const i64 ld = lv.cld[i];
            g1.add_task(T1.p + lv.coff[k], ld, ry, rx, T(0));
            g1.add_entry(lv.R.p + lv.qoff[i], lv.dims[i], 0, K.p + lv.coff[k], ld, 0, ry, T(1));
            g2.add_task(lv.C.p + lv.coff[k], ld, ry, rx, T(0));
            g2.add_entry(T1.p + lv.coff[k], ld, 0, lv.R.p + lv.qoff[x], lv.dims[x], 1, rx, T(1));
          }
        g1.name = g2.name = "gemm_coupling";
        g1.finalize();
        g2.finalize();
        g1.run(st());
        g2.run(st());
      }
    }
  }

  // Fixed-rank orthogonal mode: far-sample block XF generated into HBM in
  // bounded chunks, Gram matrix G = XF^T XF by the segmented GEMM (FP64),
  // pivoted Cholesky of G (the pivots and R rows of ColPivHouseholderQR in
  // exact arithmetic, h2matrix.cpp:21-32), then the same ID / completion step
  // as the Householder path, in FP64, converted to T at the end.
  void basis_gram(Level<T>& lv, bool leaf, const std::vector<i64>& soff, DVec<int>& d_sidx, DVec<i64>& d_krows,
                  DVec<int>& d_perm, DVec<double>& d_maxpiv, DVec<int>& d_nonzero, double e, i64 cap) {
    const i64 nodes = lv.nodes;
    std::vector<i64> gram_krows(nodes);
    for (i64 i = 0; i < nodes; i++) gram_krows[i] = std::min<i64>(lv.dims[i], soff[i + 1] - soff[i]);
    DVec<double> spts, G, XF, Rws;
    spts.alloc(std::max<i64>(3, 3 * soff[nodes]));
    ck(launch_gather_points(bodies.p, d_sidx.p, soff[nodes], spts.p, st()), "gather samples");
    G.alloc(lv.qoff[nodes]);
    const i64 cap_elems = (i64)1 << 28;
    std::vector<std::pair<i64, i64>> chunks;
    i64 maxchunk = 1;
    for (i64 i0 = 0; i0 < nodes;) {
      i64 used = 0, i1 = i0;
      while (i1 < nodes) {
        i64 sz = (soff[i1 + 1] - soff[i1]) * lv.dims[i1];
        if (used > 0 && used + sz > cap_elems) break;
        used += sz;
        i1++;
      }
      chunks.emplace_back(i0, i1);
      maxchunk = std::max(maxchunk, used);
      i0 = i1;
    }
    XF.alloc(maxchunk);
    const int gt_w = gram_tile();
    for (auto& ch : chunks) {
      std::vector<GenTask> gt;
      std::vector<GramTask> gm;
      std::vector<int4> tiles;
      double gfl = 0.;
      i64 o = 0;
      for (i64 i = ch.first; i < ch.second; i++) {
        const i64 S = soff[i + 1] - soff[i], M = lv.dims[i];
        if (M == 0) continue;
        if (S == 0) {
          ck(cudaMemsetAsync(G.p + lv.qoff[i], 0, sizeof(double) * M * M, st()), "gram zero");
          continue;
        }
        GenTask t;
        t.bi = spts.p + 3 * soff[i];
        t.bj = lv.pts.p + 3 * lv.xoff[i];
        t.m = (int)S;
        t.n = (int)M;
        t.out_off = o;
        t.ld = S;
        gt.push_back(t);
        GramTask g;
        g.X = XF.p + o;
        g.ld = S;
        g.S = (int)S;
        g.M = (int)M;
        g.G = G.p + lv.qoff[i];
        g.ldg = M;
        const int tn = (int)((M + gt_w - 1) / gt_w);
        for (int a = 0; a < tn; a++)
          for (int b = a; b < tn; b++) tiles.push_back(make_int4((int)gm.size(), a, b, 0));
        gm.push_back(g);
        gfl += (double)S * M * (M + 1);  // symmetric rank-S product
        o += S * M;
      }
      if (gt.empty()) continue;
      DVec<GenTask> dg;
      dg.upload(gt);
      {
        Prof pf("gen_samples", 0., 8. * o);
        ck(launch_gen_blocks<double>(kp, dg.p, (int)gt.size(), gen_max_rows(gt), XF.p, st(), 1, gen_err()),
           "gen samples");
      }
      DVec<GramTask> dgm;
      DVec<int4> dtl;
      dgm.upload(gm);
      dtl.upload(tiles);
      {
        Prof pf("gram", gfl, 8. * o);
        ck(launch_gram(dgm.p, dtl.p, (int)tiles.size(), st()), "gram");
      }
    }
    Rws.alloc(lv.qoff[nodes]);
    Rws.zero(st());
    {
      // Blocked pivoted Cholesky: panels of 32 pivots per box, each followed
      // by one batched rank-32 update of every trailing Gram matrix.
      const int nb = 32;
      std::vector<i64> steps(nodes, 0);
      i64 maxsteps = 0;
      double fl = 0.;
      for (i64 i = 0; i < nodes; i++) {
        i64 K = std::min<i64>(lv.dims[i], soff[i + 1] - soff[i]);
        steps[i] = cap >= 0 ? std::min<i64>(K, cap) : K;
        maxsteps = std::max(maxsteps, steps[i]);
        double Md = (double)lv.dims[i], sd = (double)steps[i];
        fl += 2. * (Md * Md * sd - Md * sd * sd + sd * sd * sd / 3.);
      }
      DVec<i64> d_steps;
      DVec<double> state;
      d_steps.upload(steps);
      state.alloc(3 * nodes);
      // The trailing-update plans depend only on the sizes: all are built
      // (and uploaded) before the first panel, so the device does not wait
      // for host planning between panels.
      std::vector<GemmPlan<double>> ups;
      ups.reserve((size_t)std::max<i64>(0, (maxsteps - 1) / nb));
      for (i64 k0 = 0; k0 + nb < maxsteps; k0 += nb) {
        const i64 k1 = k0 + nb;
        ups.emplace_back();
        GemmPlan<double>& up = ups.back();
        up.name = "gemm_pivchol_update";
        for (i64 i = 0; i < nodes; i++) {
          const i64 M = lv.dims[i];
          if (steps[i] <= k1 || M <= k1) continue;
          double* Rb = Rws.p + lv.qoff[i];
          up.add_task(G.p + lv.qoff[i] + k1 + k1 * M, M, (int)(M - k1), (int)(M - k1), 1.);
          up.add_entry(Rb + k0 * M + k1, M, 0, Rb + k0 * M + k1, M, 1, nb, -1.);
        }
        up.finalize();
      }
      Prof pf("pivchol", fl, 0.);
      for (i64 k0 = 0, p = 0; k0 < maxsteps; k0 += nb, p++) {
        ck(launch_pivchol_panel(lv.d_dims.p, d_steps.p, G.p, Rws.p, lv.d_qoff.p, d_perm.p, lv.d_xoff.p, state.p,
                                (int)k0, nb, (int)nodes, (int)lv.maxM, st()),
           "pivchol panel");
        if (k0 + nb >= maxsteps) break;
        ups[p].run(st());
      }
    }
    DVec<double> taus;
    taus.alloc(std::max<i64>(1, lv.lenX));
    if (std::is_same<T, double>::value) {
      {
        Prof pfin("basis_finish", 0., (double)lv.qoff[nodes] * 24.);
        ck(launch_basis_finish<double>(lv.d_dims.p, d_krows.p, Rws.p, reinterpret_cast<double*>(lv.Q.p),
                                       reinterpret_cast<double*>(lv.R.p), lv.d_qoff.p, d_perm.p, lv.d_xoff.p,
                                       d_maxpiv.p, d_nonzero.p, lv.pts.p, lv.d_ranks.p, e, 1, leaf ? 1 : 0,
                                       (int)nodes, (int)lv.maxM, st(), taus.p),
           "basis_finish");
      }
      blocked_orth_qr<double>(lv, Rws.p, reinterpret_cast<double*>(lv.Q.p), reinterpret_cast<double*>(lv.R.p),
                              taus.p, fixed_rank_rule(lv.dims, gram_krows, e), leaf);
    } else {
      DVec<double> Qd, Rd;
      Qd.alloc(lv.qoff[nodes]);
      Rd.alloc(lv.qoff[nodes]);
      Rd.zero(st());
      ck(launch_convert<T, double>(lv.Q.p, Qd.p, lv.qoff[nodes], st()), "convert");
      {
        Prof pfin("basis_finish", 0., (double)lv.qoff[nodes] * 24.);
        ck(launch_basis_finish<double>(lv.d_dims.p, d_krows.p, Rws.p, Qd.p, Rd.p, lv.d_qoff.p, d_perm.p,
                                       lv.d_xoff.p, d_maxpiv.p, d_nonzero.p, lv.pts.p, lv.d_ranks.p, e, 1,
                                       leaf ? 1 : 0, (int)nodes, (int)lv.maxM, st(), taus.p),
           "basis_finish");
      }
      blocked_orth_qr<double>(lv, Rws.p, Qd.p, Rd.p, taus.p, fixed_rank_rule(lv.dims, gram_krows, e), leaf);
      ck(launch_convert<double, T>(Qd.p, lv.Q.p, lv.qoff[nodes], st()), "convert");
      ck(launch_convert<double, T>(Rd.p, lv.R.p, lv.qoff[nodes], st()), "convert");
    }
  }

  // Orthogonal completion (h2matrix.cpp:43-49) for every box with
  // 0 < rank < M, after the finish kernel left U_ID = P [I; T^T] in R's slot
  // and Q_in (upper triangular) in Q: W = Q_in U_ID (M x rank, ld M), a
  // blocked Householder QR of W (panels factored in shared memory, the
  // trailing columns updated by three batched GEMMs per panel,
  // A -= V (T^T (V^T A))), R = triu(W[:rank, :rank]) and
  // Q = H_0 ... H_{rank-1} in compact-WY form.
  template <typename U>
  void blocked_orth_qr(Level<T>& lv, U* W, U* Q, U* R, U* taus, const std::vector<i64>& ranks, bool leaf) {
    std::vector<i64> box;
    i64 maxM = 0, maxr = 0, ysz = 0;
    for (i64 i = 0; i < lv.nodes; i++) {
      const i64 M = lv.dims[i], r = ranks[i];
      if (!(0 < r && r < M)) continue;
      box.push_back(i);
      maxM = std::max(maxM, M);
      maxr = std::max(maxr, r);
    }
    if (box.empty()) return;
    int nb = 32;
    while (nb > 1 && sizeof(U) * ((size_t)maxM * nb + 2 * nb + (size_t)nb * nb) > 190 * 1024) nb--;
    for (i64 i : box) ysz += (i64)nb * ranks[i];
    {
      double fl = 0.;
      for (i64 i : box) fl += leaf ? 0. : (double)lv.dims[i] * lv.dims[i] * ranks[i];
      if (leaf) {
        CopyPlan<U> cp;
        for (i64 i : box) cp.add(R + lv.qoff[i], lv.dims[i], W + lv.qoff[i], lv.dims[i], (int)lv.dims[i], (int)ranks[i]);
        cp.finalize();
        cp.run(st());
      } else {
        GemmPlan<U> g;
        g.name = "gemm_qr";
        for (i64 i : box) {
          const i64 M = lv.dims[i];
          g.add_task(W + lv.qoff[i], M, (int)M, (int)ranks[i], U(0));
          g.add_entry(Q + lv.qoff[i], M, 0, R + lv.qoff[i], M, 0, (int)M, U(1));
        }
        g.finalize();
        g.run(st());
      }
    }
    DVec<U> Vp, Tp, Y, Y2;
    Vp.alloc((i64)box.size() * maxM * nb);
    Tp.alloc((i64)box.size() * nb * nb);
    Y.alloc(ysz);
    Y2.alloc(ysz);
    for (i64 k0 = 0; k0 < maxr; k0 += nb) {
      std::vector<QrPanelTask<U>> pt;
      GemmPlan<U> gy, gt, ga;
      gy.name = gt.name = ga.name = "gemm_qr";
      i64 yo = 0;
      int maxm = 0;
      double fl = 0.;
      for (size_t z = 0; z < box.size(); z++) {
        const i64 i = box[z], M = lv.dims[i], r = ranks[i];
        if (k0 >= r) continue;
        const int w = (int)std::min<i64>(nb, r - k0), m = (int)(M - k0);
        U* vp = Vp.p + (i64)z * maxM * nb;
        U* tp = Tp.p + (i64)z * nb * nb;
        QrPanelTask<U> t;
        t.W = W + lv.qoff[i];
        t.Vp = vp;
        t.Tp = tp;
        t.taus = taus + lv.xoff[i];
        t.M = (int)M;
        t.k0 = (int)k0;
        t.nb = w;
        pt.push_back(t);
        maxm = std::max(maxm, m);
        fl += 2. * m * w * w;
        const i64 n2 = r - k0 - w;
        if (n2 <= 0) continue;
        U* At = W + lv.qoff[i] + k0 + (k0 + w) * M;
        gy.add_task(Y.p + yo, w, w, (int)n2, U(0));
        gy.add_entry(vp, m, 1, At, M, 0, m, U(1));
        gt.add_task(Y2.p + yo, w, w, (int)n2, U(0));
        gt.add_entry(tp, w, 1, Y.p + yo, w, 0, w, U(1));
        ga.add_task(At, M, m, (int)n2, U(1));
        ga.add_entry(vp, m, 0, Y2.p + yo, w, 0, w, U(-1));
        yo += (i64)w * n2;
      }
      DVec<QrPanelTask<U>> dpt;
      dpt.upload(pt);
      {
        Prof pf("qr_panel", fl, 0.);
        ck(launch_qr_panel<U>(dpt.p, (int)pt.size(), maxm, nb, st()), "qr_panel");
      }
      if (yo > 0) {
        gy.finalize();
        gt.finalize();
        ga.finalize();
        gy.run(st());
        gt.run(st());
        ga.run(st());
      }
    }
    std::vector<QrExtractTask<U>> et;
    for (i64 i : box) {
      QrExtractTask<U> t;
      t.W = W + lv.qoff[i];
      t.R = R + lv.qoff[i];
      t.Q = Q + lv.qoff[i];
      t.M = (int)lv.dims[i];
      t.rank = (int)ranks[i];
      et.push_back(t);
    }
    DVec<QrExtractTask<U>> det;
    det.upload(et);
    {
      Prof pf("qr_extract", 0., 0.);
      ck(launch_qr_extract<U>(det.p, (int)et.size(), st()), "qr_extract");
    }
    wy_form_q<U>(lv, W, Q, taus, ranks);
  }

  // Q = H_0 ... H_{r-1} = I - V T V^T for every box whose orthogonal basis
  // was completed by a Householder QR (0 < rank < M): S = V^T V and the two
  // products are batched GEMMs over the level, T comes from k_wy_t.  W holds
  // the explicit V (M x rank, column-major at the box's qoff), Q the identity.
  template <typename U>
  void wy_form_q(Level<T>& lv, U* W, U* Q, U* taus, const std::vector<i64>& ranks) {
    std::vector<i64> so(1, 0), wo(1, 0);
    std::vector<i64> box;
    int maxr = 0;
    for (i64 i = 0; i < lv.nodes; i++) {
      const i64 M = lv.dims[i], r = ranks[i];
      if (!(0 < r && r < M)) continue;
      box.push_back(i);
      so.push_back(so.back() + r * r);
      wo.push_back(wo.back() + r * M);
      maxr = std::max<int>(maxr, (int)r);
    }
    if (box.empty()) return;
    DVec<U> Sb, Tb, W2;
    Sb.alloc(so.back());
    Tb.alloc(so.back());
    W2.alloc(wo.back());
    GemmPlan<U> gs, gw, gq;
    gs.name = gw.name = gq.name = "gemm_wy";
    std::vector<WyTask<U>> wt;
    for (size_t z = 0; z < box.size(); z++) {
      const i64 i = box[z], M = lv.dims[i];
      const int r = (int)ranks[i];
      U* Wi = W + lv.qoff[i];
      gs.add_task(Sb.p + so[z], r, r, r, U(0));
      gs.add_entry(Wi, M, 1, Wi, M, 0, (int)M, U(1));
      WyTask<U> t;
      t.S = Sb.p + so[z];
      t.taus = taus + lv.xoff[i];
      t.Tm = Tb.p + so[z];
      t.r = r;
      wt.push_back(t);
      gw.add_task(W2.p + wo[z], r, r, (int)M, U(0));
      gw.add_entry(Tb.p + so[z], r, 0, Wi, M, 1, r, U(1));
      gq.add_task(Q + lv.qoff[i], M, (int)M, (int)M, U(1));
      gq.add_entry(Wi, M, 0, W2.p + wo[z], r, 0, r, U(-1));
    }
    gs.finalize();
    gw.finalize();
    gq.finalize();
    DVec<WyTask<U>> dwt;
    dwt.upload(wt);
    gs.run(st());
    {
      Prof pf("wy_t", 0., 0.);
      ck(launch_wy_t<U>(dwt.p, (int)wt.size(), maxr, st()), "wy_t");
    }
    gw.run(st());
    gq.run(st());
  }

  // ------------------------------------------------------------ vectors
  void ensure_vectors(i64 nrhs) {
    if (nrhs == cur_nrhs) return;
    for (auto& lv : L) {
      lv.vX.alloc(std::max<i64>(1, lv.lenX * nrhs));
      lv.vZ.alloc(std::max<i64>(1, lv.lenZ * nrhs));
      lv.vW.alloc(std::max<i64>(1, lv.lenZ * nrhs));
    }
    vin.alloc(std::max<i64>(1, N * nrhs));
    vout.alloc(std::max<i64>(1, N * nrhs));
    cur_nrhs = nrhs;
    mv_built = false;
    pc_built = false;
    gen++;
  }

  // H^2 matvec plans (h2matrix.cpp:251-344) for the current nrhs.
  // Multi-RHS H^2 matvec plans (h2matrix.cpp:303-344): upward pass
  // Z_l = Q_l^T X_l (from the transposed copies), one launch for the far
  // couplings of every level W_l = sum_j C_ij Z_j (all levels read finished
  // upward results and write their own W), then the downward pass
  // W_{l+1} += Q_l W_l level by level and the leaf Y = Q W + sum_j A_ij X_j.
  void build_matvec(i64 nrhs) {
    const int nr = (int)nrhs;
    gen++;
    mv_up.clear();
    mv_down.clear();
    mv_up.resize(levels + 1);
    mv_down.resize(levels + 1);
    {
      CopyPlan<T> tp;
      for (i64 l = 0; l <= levels; l++) {
        Level<T>& lv = L[l];
        lv.qtoff.assign(lv.nodes + 1, 0);
        // Leading dimension rank_i rounded up to 4 (32-byte column starts).
        for (i64 i = 0; i < lv.nodes; i++) lv.qtoff[i + 1] = lv.qtoff[i] + (lv.ranks[i] + 3) / 4 * 4 * lv.dims[i];
        lv.Qt.alloc(std::max<i64>(1, lv.qtoff[lv.nodes]));
        for (i64 i = 0; i < lv.nodes; i++)
          tp.add(lv.Q.p + lv.qoff[i], lv.dims[i], lv.Qt.p + lv.qtoff[i], (lv.ranks[i] + 3) / 4 * 4, (int)lv.ranks[i],
                 (int)lv.dims[i], 1);
      }
      tp.finalize();
      tp.run(st());
    }
    for (i64 l = levels; l >= 0; l--) {
      Level<T>& lv = L[l];
      const T* X = (l == levels) ? vin.p : L[l + 1].vZ.p;
      const i64 ldx = lv.lenX;
      GemmPlan<T>& g = mv_up[l];
      g.name = "gemm_matvec_up";
      for (i64 i = 0; i < lv.nodes; i++) {
        int M = (int)lv.dims[i], r = (int)lv.ranks[i];
        if (r == 0) continue;
        g.add_task(lv.vZ.p + lv.zoff[i], lv.lenZ, r, nr, T(0));
        g.add_entry(lv.Qt.p + lv.qtoff[i], (r + 3) / 4 * 4, 0, X + lv.xoff[i], ldx, 0, M, T(1));
      }
      g.finalize();
    }
    if (matrix_free) build_mf_plans(nr);
    mv_far = GemmPlan<T>();
    mv_far.name = "gemm_matvec_far";
    for (i64 l = 0; l <= levels && !matrix_free; l++) {
      Level<T>& lv = L[l];
      for (i64 i = 0; i < lv.nodes; i++) {
        int r = (int)lv.ranks[i];
        if (r == 0) continue;
        mv_far.add_task(lv.vW.p + lv.zoff[i], lv.lenZ, r, nr, T(0));
        for (i64 k = lv.crow[i]; k < lv.crow[i + 1]; k++) {
          i64 j = lv.ccol[k];
          mv_far.add_entry(lv.C.p + lv.coff[k], lv.cld[i], 0, lv.vZ.p + lv.zoff[j], lv.lenZ, 0, (int)lv.ranks[j], T(1));
        }
      }
    }
    mv_far.finalize();
    for (i64 l = 0; l < levels; l++) {
      Level<T>& lv = L[l];
      GemmPlan<T>& d = mv_down[l];
      d.name = "gemm_matvec_down";
      Level<T>& nx = L[l + 1];  // Y_l lives in W_{l+1}
      for (i64 i = 0; i < lv.nodes; i++) {
        int M = (int)lv.dims[i], r = (int)lv.ranks[i];
        d.add_task(nx.vW.p + lv.xoff[i], nx.lenZ, M, nr, T(1));
        d.add_entry(lv.Q.p + lv.qoff[i], M, 0, lv.vW.p + lv.zoff[i], lv.lenZ, 0, r, T(1));
      }
      d.finalize();
    }
    {
      Level<T>& lv = L[levels];
      GemmPlan<T>& g = mv_leaf;
      g = GemmPlan<T>();
      g.name = "gemm_matvec_near";
      GemmPlan<T>& q = mv_qw;
      q = GemmPlan<T>();
      q.name = "gemm_matvec_down";
      for (i64 i = 0; i < lv.nodes; i++) {
        int M = (int)lv.dims[i], r = (int)lv.ranks[i];
        if (!matrix_free) {
          g.add_task(vout.p + lv.xoff[i], lv.lenX, M, nr, T(0));
          for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) {
            i64 j = lv.acol[k];
            g.add_entry(lv.A.p + lv.aoff[k], M, 0, vin.p + lv.xoff[j], lv.lenX, 0, (int)lv.dims[j], T(1));
          }
        }
        q.add_task(vout.p + lv.xoff[i], lv.lenX, M, nr, T(1));
        q.add_entry(lv.Q.p + lv.qoff[i], M, 0, lv.vW.p + lv.zoff[i], lv.lenZ, 0, r, T(1));
      }
      g.finalize();
      q.finalize();
    }
    mv_built = true;
  }

  // Matrix-free near field (leaf boxes, tree-order bodies, as the stored
  // blocks are generated) and couplings (skeleton bodies of every level).
  void build_mf_plans(int nr) {
    if constexpr (std::is_same<T, double>::value) {
      mf_far = MfPlan();
      mf_far.name = "mf_matvec_far";
      mf_far.nr = nr;
      for (i64 l = 0; l <= levels; l++) {
        Level<T>& lv = L[l];
        for (i64 i = 0; i < lv.nodes; i++) {
          const int r = (int)lv.ranks[i];
          if (r == 0) continue;
          mf_far.add_task(lv.pts.p + 3 * lv.xoff[i], r, lv.vW.p + lv.zoff[i], lv.lenZ, 0.);
          for (i64 k = lv.crow[i]; k < lv.crow[i + 1]; k++) {
            const i64 j = lv.ccol[k];
            mf_far.add_entry(lv.pts.p + 3 * lv.xoff[j], (int)lv.ranks[j], lv.vZ.p + lv.zoff[j], lv.lenZ, 1.);
          }
        }
      }
      mf_far.finalize();
      mf_leaf = MfPlan();
      mf_leaf.name = "mf_matvec_near";
      mf_leaf.nr = nr;
      Level<T>& lv = L[levels];
      const i64 g0 = lv.gbegin;
      for (i64 i = 0; i < lv.nodes; i++) {
        const int M = (int)lv.dims[i];
        mf_leaf.add_task(bodies.p + 3 * cells[g0 + i].body[0], M, vout.p + lv.xoff[i], lv.lenX, 0.);
        for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) {
          const i64 j = lv.acol[k];
          mf_leaf.add_entry(bodies.p + 3 * cells[g0 + j].body[0], (int)lv.dims[j], vin.p + lv.xoff[j], lv.lenX, 1.);
        }
      }
      mf_leaf.finalize();
    }
  }
  void run_near(cudaStream_t s) {
    if (matrix_free)
      mf_leaf.run(kp, s);
    else
      mv_leaf.run(s);
  }
  void run_far(cudaStream_t s) {
    if (matrix_free)
      mf_far.run(kp, s);
    else
      mv_far.run(s);
  }

  void stage_in(i64 nrhs, const double* dX, i64 ldx) {
    Prof pf("stage_convert", 0., (8. + sizeof(T)) * N * nrhs);
    if (ldx == N) {
      ck(launch_convert<double, T>(dX, vin.p, N * nrhs, st()), "convert in");
    } else {
      for (i64 c = 0; c < nrhs; c++) ck(launch_convert<double, T>(dX + c * ldx, vin.p + c * N, N, st()), "convert in");
    }
  }
  void stage_out(i64 nrhs, double* dX, i64 ldx) {
    Prof pf("stage_convert", 0., (8. + sizeof(T)) * N * nrhs);
    if (ldx == N) {
      ck(launch_convert<T, double>(vout.p, dX, N * nrhs, st()), "convert out");
    } else {
      for (i64 c = 0; c < nrhs; c++) ck(launch_convert<T, double>(vout.p + c * N, dX + c * ldx, N, st()), "convert out");
    }
  }

  void prepare(i64 nrhs) override {
    ensure_vectors(nrhs);
    if (!mv_built) build_matvec(nrhs);
    if (factored && !pc_built) build_precondition(nrhs);
    // Autotuning decisions are taken now, outside any capture (the timed
    // runs write only this solver's internal vectors).
    for (auto& g : mv_up) g.tune(st());
    for (auto& g : mv_down) g.tune(st());
    mv_far.tune(st());
    mv_leaf.tune(st());
    mv_qw.tune(st());
    if (matrix_free) {
      mf_far.tune(kp, st());
      mf_leaf.tune(kp, st());
    }
    if (factored)
      for (auto* v : {&pc_fx, &pc_fz, &pc_bx, &pc_by})
        for (auto& g : *v) g.tune(st());
  }

  void matvec(i64 nrhs, double* dX, i64 ldx) override {
    require(nrhs > 0 && ldx >= N, "matvec: bad nrhs/ld");
    ensure_vectors(nrhs);
    if (!mv_built) build_matvec(nrhs);
    stage_in(nrhs, dX, ldx);
    // The near field (reads the input, writes the output) does not depend on
    // the upward / far / downward chain: it runs on the side stream while the
    // chain's small upper-level launches run on the main one (serialised
    // while per-launch profiling is on, so each launch is timed alone).
    // The leaf U W term is added after both, so the result does not depend
    // on the overlap.
    const bool fork = h->stream2 && !h->prof;
    if (fork) {
      ck(cudaEventRecord(h->ev_fork, st()), "fork");
      ck(cudaStreamWaitEvent(h->stream2, h->ev_fork, 0), "fork");
      run_near(h->stream2);
      ck(cudaEventRecord(h->ev_join, h->stream2), "join");
    }
    for (i64 l = levels; l >= 0; l--) mv_up[l].run(st());
    run_far(st());
    for (i64 l = 0; l < levels; l++) mv_down[l].run(st());
    if (fork) {
      ck(cudaStreamWaitEvent(st(), h->ev_join, 0), "join");
    } else {
      run_near(st());
    }
    mv_qw.run(st());
    stage_out(nrhs, dX, ldx);
  }

  // ------------------------------------------------------------ factor
  // h2matrix.cpp:346-425 for one level (factorizeCopyNext, 427-446, is copy_next).
  void factor_level(i64 l) {
    Level<T>& lv = L[l];
    const i64 nodes = lv.nodes;
    if (lv.lenX == 0) {
      lv.info_count = 0;
      return;
    }
    std::vector<i64>& D = lv.dims;
    std::vector<i64>& Rk = lv.ranks;
    DVec<T> T1;
    T1.alloc(lv.qoff[nodes]);
    lv.boff.assign(nodes + 1, 0);
    lv.ioff.assign(nodes + 1, 0);
    std::vector<i64> poff(nodes + 1, 0);
    for (i64 i = 0; i < nodes; i++) {
      i64 Mr = D[i] - Rk[i];
      lv.boff[i + 1] = lv.boff[i] + Mr * D[i];
      lv.ioff[i + 1] = lv.ioff[i] + Mr * Mr;
      poff[i + 1] = poff[i] + Mr;
    }
    lv.B.alloc(std::max<i64>(1, lv.boff[nodes]));
    // Global LU scratch only for redundant blocks too large for the solve
    // kernel's shared memory; released at the end of the level.
    i64 maxMr = 0;
    for (i64 i = 0; i < nodes; i++) maxMr = std::max(maxMr, D[i] - Rk[i]);
    const bool lu_in_smem = (double)sizeof(T) * maxMr * (maxMr + 1) + 8. * maxMr + 16. <= 200. * 1024.;
    lv.invT.alloc(lu_in_smem ? 1 : std::max<i64>(1, lv.ioff[nodes]));
    lv.ipiv.alloc(std::max<i64>(1, poff[nodes]));
    lv.info.alloc(nodes);
    lv.info.zero(st());
    T* A = lv.A.p;
    T* Q = lv.Q.p;
    T* V = lv.R.p;  // V stored transposed: V^T column-major
    // Steps 1-2: A_ii <- U^T A_ii U.
    GemmPlan<T> s1, s2, s6, s7, s8;
    CopyPlan<T> c3, c8;
    for (i64 i = 0; i < nodes; i++) {
      const int M = (int)D[i];
      if (M == 0) continue;
      T* Aii = A + lv.aoff[lv.diag[i]];
      s1.add_task(T1.p + lv.qoff[i], M, M, M, T(0));
      s1.add_entry(Aii, M, 0, Q + lv.qoff[i], M, 0, M, T(1));
      s2.add_task(Aii, M, M, M, T(0));
      s2.add_entry(Q + lv.qoff[i], M, 1, T1.p + lv.qoff[i], M, 0, M, T(1));
    }
    s1.name = "gemm_factor";
    s1.finalize();
    s2.name = "gemm_factor";
    s2.finalize();
    s1.run(st());
    s2.run(st());
    // Step 3: V^T[:, :Ms] = U_s.  Steps 4-5: PartialPivLU of A_rr and
    // V_r = A_rr^{-1} U_r^T by its triangular solves (h2matrix.cpp:377-379);
    // V_r is stored as V^T[:, Ms:], row r of V_r contiguous, as U_r^T is in
    // Q[:, Ms:].
    std::vector<LuSolveTask<T>> lt;
    for (i64 i = 0; i < nodes; i++) {
      const int M = (int)D[i], Ms = (int)Rk[i], Mr = M - Ms;
      if (M == 0) continue;
      c3.add(Q + lv.qoff[i], M, V + lv.qoff[i], M, M, Ms);
      LuSolveTask<T> t;
      t.A = A + lv.aoff[lv.diag[i]] + Ms + (i64)Ms * M;
      t.lda = M;
      t.n = Mr;
      t.B = Q + lv.qoff[i] + (i64)Ms * M;
      t.ldb = M;
      t.m = M;
      t.X = V + lv.qoff[i] + (i64)Ms * M;
      t.ldx = M;
      t.work = lu_in_smem ? nullptr : lv.invT.p + lv.ioff[i];
      t.ipiv = lv.ipiv.p + poff[i];
      t.info = lv.info.p + i;
      lt.push_back(t);
    }
    c3.finalize();
    c3.run(st());
    {
      DVec<LuSolveTask<T>> dl;
      dl.upload(lt);
      double fl = 0.;
      for (const auto& t : lt) fl += 2. / 3. * (double)t.n * t.n * t.n + 2. * (double)t.n * t.n * t.m;
      Prof pf("lu_solve", fl, 0.);
      int maxn = 0;
      for (const auto& x : lt) maxn = std::max(maxn, x.n);
      ck(launch_lu_solve<T>(dl.p, (int)lt.size(), maxn, st()), "lu_solve");
    }
    // Steps 6-8.
    for (i64 i = 0; i < nodes; i++) {
      const int M = (int)D[i], Ms = (int)Rk[i], Mr = M - Ms;
      if (M == 0 || Mr == 0) continue;
      T* Aii = A + lv.aoff[lv.diag[i]];
      if (Ms > 0) {
        s6.add_task(Aii + Ms, M, Mr, Ms, T(0));
        s6.add_entry(V + lv.qoff[i] + (i64)Ms * M, M, 1, T1.p + lv.qoff[i], M, 0, M, T(1));
        s7.add_task(Aii, M, Ms, Ms, T(1));
        s7.add_entry(Aii + (i64)Ms * M, M, 0, Aii + Ms, M, 0, Mr, T(-1));
      }
      c8.add(Aii + Ms, M, lv.B.p + lv.boff[i], Mr, Mr, Ms);
      s8.add_task(lv.B.p + lv.boff[i] + (i64)Ms * Mr, Mr, Mr, Mr, T(0));
      s8.add_entry(V + lv.qoff[i] + (i64)Ms * M, M, 1, Q + lv.qoff[i] + (i64)Ms * M, M, 0, M, T(1));
    }
    s6.name = "gemm_factor";
    s6.finalize();
    s7.name = "gemm_factor";
    s7.finalize();
    s8.name = "gemm_factor";
    s8.finalize();
    c8.finalize();
    s6.run(st());
    s7.run(st());
    c8.run(st());
    s8.run(st());
    // Step 9: off-diagonal transforms A_ij <- V_i A_ij U_j, in chunks of
    // bounded scratch.
    {
      std::vector<i64> offd;
      for (i64 i = 0; i < nodes; i++)
        for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++)
          if (k != lv.diag[i]) offd.push_back(k);
      std::vector<i64> rowof(lv.acol.size());
      for (i64 i = 0; i < nodes; i++)
        for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) rowof[k] = i;
      const i64 cap = (i64)1 << 27;  // elements of scratch per chunk
      size_t p = 0;
      DVec<T> T2;
      while (p < offd.size()) {
        i64 used = 0;
        size_t q = p;
        while (q < offd.size()) {
          i64 k = offd[q];
          i64 sz = D[rowof[k]] * D[lv.acol[k]];
          if (used > 0 && used + sz > cap) break;
          used += sz;
          q++;
        }
        T2.alloc(std::max<i64>(used, 1));
        GemmPlan<T> a, b;
        i64 o = 0;
        for (size_t z = p; z < q; z++) {
          i64 k = offd[z];
          i64 i = rowof[k], j = lv.acol[k];
          int Mi = (int)D[i], Nj = (int)D[j];
          if (Mi == 0 || Nj == 0) continue;
          T* Aij = A + lv.aoff[k];
          a.add_task(T2.p + o, Mi, Mi, Nj, T(0));
          a.add_entry(Aij, Mi, 0, Q + lv.qoff[j], Nj, 0, Nj, T(1));
          // Only the skeleton rows (ss, sr) and the rs block are formed: the
          // redundant-redundant block of an off-diagonal A_ij is never read
          // afterwards (Schur updates read ss / sr / rs, the substitution sr
          // and rs, the parent level ss), as the reference ULV drops that fill.
          const int Ms = (int)Rk[i], Ns = (int)Rk[j];
          if (Ms > 0) {
            b.add_task(Aij, Mi, Ms, Nj, T(0));
            b.add_entry(V + lv.qoff[i], Mi, 1, T2.p + o, Mi, 0, Mi, T(1));
          }
          if (Mi > Ms && Ns > 0) {
            b.add_task(Aij + Ms, Mi, Mi - Ms, Ns, T(0));
            b.add_entry(V + lv.qoff[i] + (i64)Ms * Mi, Mi, 1, T2.p + o, Mi, 0, Mi, T(1));
          }
          o += (i64)Mi * Nj;
        }
        a.name = b.name = "gemm_factor";
        a.finalize();
        b.finalize();
        a.run(st());
        b.run(st());
        p = q;
      }
      // Steps 10-11: neighbour Schur updates of the skeleton blocks.
      GemmPlan<T> s10, s11a, s11b;
      std::vector<i64> t3off(lv.acol.size() + 1, 0);
      for (i64 i = 0; i < nodes; i++)
        for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) {
          i64 j = lv.acol[k];
          i64 add = (k != lv.diag[i]) ? Rk[i] * (D[j] - Rk[j]) : 0;
          t3off[k + 1] = t3off[k] + add;
        }
      DVec<T> T3;
      T3.alloc(std::max<i64>(1, t3off.back()));
      for (i64 i = 0; i < nodes; i++) {
        const int M = (int)D[i], Ms = (int)Rk[i], Mr = M - Ms;
        if (Ms == 0) continue;
        T* Aii = A + lv.aoff[lv.diag[i]];
        bool any = false;
        for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) {
          if (k == lv.diag[i]) continue;
          i64 j = lv.acol[k];
          const int N = (int)D[j], Ns = (int)Rk[j], Nr = N - Ns;
          T* Aij = A + lv.aoff[k];
          if (Ns > 0) {
            s10.add_task(Aij, M, Ms, Ns, T(1));
            s10.add_entry(Aii + (i64)Ms * M, M, 0, Aij + Ms, M, 0, Mr, T(-1));
            s10.add_entry(Aij + (i64)Ns * M, M, 0, lv.B.p + lv.boff[j], Nr, 0, Nr, T(-1));
          }
          if (Nr > 0) {
            s11a.add_task(T3.p + t3off[k], Ms, Ms, Nr, T(0));
            s11a.add_entry(Aij + (i64)Ns * M, M, 0, lv.B.p + lv.boff[j] + (i64)Ns * Nr, Nr, 0, Nr, T(1));
            any = true;
          }
        }
        if (any) {
          s11b.add_task(Aii, M, Ms, Ms, T(1));
          for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) {
            if (k == lv.diag[i]) continue;
            i64 j = lv.acol[k];
            const int N = (int)D[j], Ns = (int)Rk[j], Nr = N - Ns;
            if (Nr > 0) s11b.add_entry(T3.p + t3off[k], Ms, 0, A + lv.aoff[k] + (i64)Ns * M, M, 1, Nr, T(-1));
          }
        }
      }
      s10.name = "gemm_factor";
    s10.finalize();
      s11a.name = "gemm_factor";
    s11a.finalize();
      s11b.name = "gemm_factor";
    s11b.finalize();
      s11a.run(st());
      s10.run(st());
      s11b.run(st());
    }
    lv.invT.release();
  }

  void copy_next(i64 l) {
    Level<T>& lv = L[l];
    Level<T>& up = L[l - 1];
    CopyPlan<T> cp;
    for (i64 i = 0; i < lv.nodes; i++)
      for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) {
        i64 j = lv.acol[k];
        int Ms = (int)lv.ranks[i], Ns = (int)lv.ranks[j];
        if (Ms > 0 && Ns > 0 && lv.na_off[k] >= 0)
          cp.add(lv.A.p + lv.aoff[k], lv.dims[i], up.A.p + lv.na_off[k], lv.na_ld[k], Ms, Ns);
      }
    cp.finalize();
    cp.run(st());
  }

  void factorize(int* info) override {
    require(!factored, "factorize: already factored");
    if (matrix_free)
      throw H2Error{H2DEV_ERR_STATE, "factorize: a matrix-free operator stores no near blocks to factor"};
    for (i64 l = levels; l >= 0; l--) {
      factor_level(l);
      if (l > 0) copy_next(l);
    }
    check_tc(h);
    // Singular-block counts per level, read once after the last level.
    for (i64 l = 0; l <= levels; l++) {
      std::vector<int> inf = L[l].info.download(st());
      L[l].info_count = 0;
      for (int v : inf) L[l].info_count += v;
      info[l] = L[l].info_count;
    }
    factored = true;
    pc_built = false;
    gen++;
  }

  // ULV substitution plans (h2matrix.cpp:448-537).
  void build_precondition(i64 nrhs) {
    const int nr = (int)nrhs;
    gen++;
    pc_fx.clear(); pc_fz.clear(); pc_bx.clear(); pc_by.clear(); pc_fcopy.clear(); pc_bcopy.clear();
    pc_fx.resize(levels + 1); pc_fz.resize(levels + 1); pc_bx.resize(levels + 1); pc_by.resize(levels + 1);
    pc_fcopy.resize(levels + 1); pc_bcopy.resize(levels + 1);
    {
      CopyPlan<T> tp;
      for (i64 l = 0; l <= levels; l++) {
        Level<T>& lv = L[l];
        lv.Rt.alloc(std::max<i64>(1, lv.qoff[lv.nodes]));
        for (i64 i = 0; i < lv.nodes; i++)
          tp.add(lv.R.p + lv.qoff[i], lv.dims[i], lv.Rt.p + lv.qoff[i], lv.dims[i], (int)lv.dims[i], (int)lv.dims[i], 1);
      }
      tp.finalize();
      tp.run(st());
    }
    for (i64 l = 0; l <= levels; l++) {
      Level<T>& lv = L[l];
      const T* Yin = (l == levels) ? vin.p : L[l + 1].vZ.p;
      T* Yout = (l == levels) ? vout.p : L[l + 1].vW.p;
      const i64 ldx = lv.lenX, ldz = lv.lenZ;
      T* X = lv.vX.p;
      T* Z = lv.vZ.p;
      T* W = lv.vW.p;
      for (i64 i = 0; i < lv.nodes; i++) {
        const int M = (int)lv.dims[i], Ms = (int)lv.ranks[i], Mr = M - Ms;
        if (M == 0) continue;
        // forward: X = V Y; Z = X_s - sum_j A_ij[:Ms, Ns:] X_j[Ns:]
        pc_fx[l].add_task(X + lv.xoff[i], ldx, M, nr, T(0));
        pc_fx[l].add_entry(lv.Rt.p + lv.qoff[i], M, 0, Yin + lv.xoff[i], ldx, 0, M, T(1));
        if (Ms > 0) {
          pc_fcopy[l].add(X + lv.xoff[i], ldx, Z + lv.zoff[i], ldz, Ms, nr);
          pc_fz[l].add_task(Z + lv.zoff[i], ldz, Ms, nr, T(1));
          for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) {
            i64 j = lv.acol[k];
            const int Nj = (int)lv.dims[j], Ns = (int)lv.ranks[j], Nr = Nj - Ns;
            if (Nr > 0)
              pc_fz[l].add_entry(lv.A.p + lv.aoff[k] + (i64)Ns * M, M, 0, X + lv.xoff[j] + Ns, ldx, 0, Nr, T(-1));
          }
        }
        // backward: X_s = W; X_r -= sum_j A_ij[Ms:, :Ns] W_j; Y = U X
        if (Ms > 0) pc_bcopy[l].add(W + lv.zoff[i], ldz, X + lv.xoff[i], ldx, Ms, nr);
        if (Mr > 0) {
          pc_bx[l].add_task(X + lv.xoff[i] + Ms, ldx, Mr, nr, T(1));
          for (i64 k = lv.arow[i]; k < lv.arow[i + 1]; k++) {
            i64 j = lv.acol[k];
            const int Ns = (int)lv.ranks[j];
            if (Ns > 0) pc_bx[l].add_entry(lv.A.p + lv.aoff[k] + Ms, M, 0, W + lv.zoff[j], ldz, 0, Ns, T(-1));
          }
        }
        const i64 ldy = (l == levels) ? N : L[l + 1].lenZ;
        pc_by[l].add_task(Yout + lv.xoff[i], ldy, M, nr, T(0));
        pc_by[l].add_entry(lv.Q.p + lv.qoff[i], M, 0, X + lv.xoff[i], ldx, 0, M, T(1));
      }
      pc_fx[l].name = pc_fz[l].name = pc_bx[l].name = pc_by[l].name = "gemm_precond";
      if (precond_bf16) continue;  // the BF16 plans below replace them
      pc_fx[l].finalize(); pc_fz[l].finalize(); pc_bx[l].finalize(); pc_by[l].finalize();
    }
    for (i64 l = 0; l <= levels; l++) {
      pc_fcopy[l].finalize();
      pc_bcopy[l].finalize();
    }
    if (precond_bf16) build_bf16_plans(nr);
    pc_built = true;
  }

  // Packs every block the substitution plans stream into one BF16 pool
  // (columns padded to multiples of 8 elements, so each block and column
  // starts on a 16-byte boundary) and builds the BF16 plans over it.
  void build_bf16_plans(int nr) {
    if constexpr (std::is_same<T, float>::value) {
      std::vector<GemmPlan<T>>* srcs[4] = {&pc_fx, &pc_fz, &pc_bx, &pc_by};
      std::vector<BfPlan>* dsts[4] = {&bf_fx, &bf_fz, &bf_bx, &bf_by};
      i64 total = 0, nblk = 0;
      for (auto* sp : srcs)
        for (auto& g : *sp)
          for (const auto& t : g.tasks)
            for (int e = t.e0; e < t.e1; e++) {
              total += (i64)((t.m + 7) / 8 * 8) * g.ents[e].k;
              nblk++;
            }
      bf_pool.alloc(std::max<i64>(8, total));
      bf_scales.alloc(std::max<i64>(1, nblk));
      std::vector<BfPackTask> packs;
      i64 off = 0, sb = 0;
      for (int q = 0; q < 4; q++) {
        dsts[q]->clear();
        dsts[q]->resize(levels + 1);
        for (i64 l = 0; l <= levels; l++) {
          const GemmPlan<T>& g = (*srcs[q])[l];
          BfPlan& b = (*dsts[q])[l];
          b.nr = nr;
          for (const auto& t : g.tasks) {
            GemmTask<float> bt = t;
            bt.e0 = (int)b.ents.size();
            const i64 ldd = (t.m + 7) / 8 * 8;
            for (int e = t.e0; e < t.e1; e++) {
              const GemmEntry<float>& en = g.ents[e];
              if (en.k <= 0) continue;
              BfPackTask pk;
              pk.src = en.A;
              pk.lds = en.lda;
              pk.m = t.m;
              pk.k = en.k;
              pk.dst = bf_pool.p + off;
              pk.ldd = ldd;
              pk.scale = bf_scales.p + sb;
              packs.push_back(pk);
              BfEntry be;
              be.A = pk.dst;
              be.lda = ldd;
              be.B = en.B;
              be.ldb = en.ldb;
              be.k = en.k;
              be.alpha = en.alpha;
              be.scale = pk.scale;
              b.ents.push_back(be);
              b.flops += 2. * nr * (double)t.m * en.k;
              b.bytes += 2. * (double)t.m * en.k + 4. * (double)nr * en.k;
              off += ldd * en.k;
              sb++;
            }
            bt.e1 = (int)b.ents.size();
            b.bytes += 8. * (double)nr * t.m;
            b.tasks.push_back(bt);
          }
          b.finalize();
        }
      }
      DVec<BfPackTask> dp;
      dp.upload(packs);
      Prof pf("bf16_pack", 0., 6. * (double)off);
      ck(launch_bf16_pack(dp.p, (int)packs.size(), st()), "bf16_pack");
    }
  }

  void precondition(i64 nrhs, double* dX, i64 ldx) override {
    if (!factored) throw H2Error{H2DEV_ERR_STATE, "solve_precondition before factorize"};
    require(nrhs > 0 && ldx >= N, "precondition: bad nrhs/ld");
    ensure_vectors(nrhs);
    if (!pc_built) build_precondition(nrhs);
    stage_in(nrhs, dX, ldx);
    if constexpr (std::is_same<T, float>::value) {
      if (precond_bf16) {
        for (i64 l = levels; l >= 0; l--) {
          bf_fx[l].run(st());
          pc_fcopy[l].run(st());
          bf_fz[l].run(st());
        }
        for (i64 l = 0; l <= levels; l++) {
          pc_bcopy[l].run(st());
          bf_bx[l].run(st());
          bf_by[l].run(st());
        }
        stage_out(nrhs, dX, ldx);
        return;
      }
    }
    for (i64 l = levels; l >= 0; l--) {
      pc_fx[l].run(st());
      pc_fcopy[l].run(st());
      pc_fz[l].run(st());
    }
    for (i64 l = 0; l <= levels; l++) {
      pc_bcopy[l].run(st());
      pc_bx[l].run(st());
      pc_by[l].run(st());
    }
    stage_out(nrhs, dX, ldx);
  }

  void level_dims(i64 l, i64* dims, i64* ranks) const override {
    require(l >= 0 && l <= levels, "level out of range");
    for (i64 i = 0; i < L[l].nodes; i++) {
      if (dims) dims[i] = L[l].dims[i];
      if (ranks) ranks[i] = L[l].ranks[i];
    }
  }

  i64 export_size(i64 l, int what) const override {
    require(l >= 0 && l <= levels, "level out of range");
    const Level<T>& lv = L[l];
    switch (what) {
      case H2DEV_EXPORT_S: return 3 * lv.lenX;
      case H2DEV_EXPORT_Q:
      case H2DEV_EXPORT_R: return lv.qoff.back();
      case H2DEV_EXPORT_A: return matrix_free ? 0 : lv.aoff.back();
      case H2DEV_EXPORT_C: {
        if (matrix_free) return 0;
        i64 n = 0;  // packed: each block rank_i x rank_j with leading dimension rank_i
        for (i64 i = 0; i < lv.nodes; i++)
          for (i64 k = lv.crow[i]; k < lv.crow[i + 1]; k++) n += lv.ranks[i] * lv.ranks[lv.ccol[k]];
        return n;
      }
    }
    require(false, "export: unknown container");
    return 0;
  }

  void export_to(i64 l, int what, double* out) override {
    i64 n = export_size(l, what);
    if (n == 0) return;
    const Level<T>& lv = L[l];
    if (what == H2DEV_EXPORT_S) {
      ck(cudaStreamSynchronize(st()), "sync");
      ck(cudaMemcpy(out, lv.pts.p, sizeof(double) * n, cudaMemcpyDeviceToHost), "export");
      return;
    }
    const T* src = what == H2DEV_EXPORT_Q ? lv.Q.p : what == H2DEV_EXPORT_R ? lv.R.p : what == H2DEV_EXPORT_A ? lv.A.p : lv.C.p;
    const i64 stored = what == H2DEV_EXPORT_C ? lv.coff.back() : n;
    DVec<double> tmp;
    tmp.alloc(stored);
    ck(launch_convert<T, double>(src, tmp.p, stored, st()), "export convert");
    ck(cudaStreamSynchronize(st()), "sync");
    if (what != H2DEV_EXPORT_C) {
      ck(cudaMemcpy(out, tmp.p, sizeof(double) * n, cudaMemcpyDeviceToHost), "export");
      return;
    }
    // Couplings are stored with leading dimension cld[i] >= rank_i: repack.
    std::vector<double> h(stored);
    ck(cudaMemcpy(h.data(), tmp.p, sizeof(double) * stored, cudaMemcpyDeviceToHost), "export");
    i64 o = 0;
    for (i64 i = 0; i < lv.nodes; i++)
      for (i64 k = lv.crow[i]; k < lv.crow[i + 1]; k++) {
        const i64 ri = lv.ranks[i], rj = lv.ranks[lv.ccol[k]];
        for (i64 c = 0; c < rj; c++)
          for (i64 r = 0; r < ri; r++) out[o++] = h[lv.coff[k] + r + c * lv.cld[i]];
      }
  }
};

// ------------------------------------------------------------------ GMRES
// solver.cpp:144-201 with one independent GMRES per right-hand side.  The
// control flow is on the device (k_vec.cu: k_gmres_init / cycle_begin /
// estimate / cycle_end): which columns are active, when a cycle's Arnoldi
// loop may stop early, the residual history.  Launched step by step (the
// host reads one flag after each Arnoldi step when early exit is on, and the
// active flags after each cycle), or, with the handle's graph option, the
// whole solve is captured once as a CUDA graph -- a WHILE node over restart
// cycles, an IF node around each Arnoldi step -- and runs as one launch with
// no host round trip until the end.
struct GmresState {
  i64 N = 0, nrhs = 0, inner = 0, outer = 0, vstride = 0;
  int ldh = 0, nch = 0;
  double tol = 0.;
  int early = 0;
  // Complex GMRES (Helmholtz): vectors of N / 2 complex entries (interleaved),
  // complex H and y; the operator and preconditioner act on the real form,
  // so a vector is conjugated before each matvec and after each
  // preconditioner solve (S conj(x) = K x, S_M^-1 y = conj(M^-1 y)).
  int cplx = 0;
  // With early exit: residual by recurrence.  A v_i is kept for every
  // Arnoldi vector (AV) and the cycle's starting residual (Rr), so the new
  // residual is Rr - AV y without a matvec; the true residual B - A X is
  // computed only to certify a column below tol (or on its last cycle), and
  // a column that fails it continues from the true residual.
  int rec = 0;
  DVec<double> V, w, R, Bc, X, H, y, beta, nrm2, partial, normb, rvec, resh, AV, Rr;
  DVec<int> act, it, ctl;  // ctl: used, stop, cycles, another cycle, need true residual
};

static void gmres_prologue(SolverBase& M, GmresState& g, cudaStream_t st) {
  const int nr = (int)g.nrhs;
  ck(launch_gmres_cycle_begin(g.ctl.p, (int)g.inner, st), "cycle begin");
  if (g.rec) ck(cudaMemcpyAsync(g.Rr.p, g.R.p, sizeof(double) * g.vstride, cudaMemcpyDeviceToDevice, st), "Rr=R");
  M.precondition(g.nrhs, g.R.p, g.N);
  if (g.cplx) ck(launch_conj_interleaved(g.R.p, g.N, g.N, nr, st), "conj");
  ck(launch_dots(g.R.p, 0, 1, g.R.p, g.N, nr, g.partial.p, g.nch, g.nrm2.p, st), "dots");
  ck(launch_scale_by_norm(g.R.p, g.V.p, g.nrm2.p, g.beta.p, 1, g.N, nr, st), "v0");
  ck(cudaMemsetAsync(g.H.p, 0, sizeof(double) * g.H.n, st), "H=0");
}

static void gmres_step(SolverBase& A, SolverBase& M, GmresState& g, i64 i, cudaStream_t st) {
  const int nr = (int)g.nrhs, kv = (int)i + 1;
  const int cw = g.cplx ? 2 : 1;  // doubles per H entry
  const i64 hstride = (i64)cw * g.ldh * g.inner;
  ck(cudaMemcpyAsync(g.w.p, g.V.p + i * g.vstride, sizeof(double) * g.vstride, cudaMemcpyDeviceToDevice, st), "w=v");
  if (g.cplx) ck(launch_conj_interleaved(g.w.p, g.N, g.N, nr, st), "conj");
  A.matvec(g.nrhs, g.w.p, g.N);
  if (g.rec)
    ck(cudaMemcpyAsync(g.AV.p + i * g.vstride, g.w.p, sizeof(double) * g.vstride, cudaMemcpyDeviceToDevice, st),
       "AV");
  M.precondition(g.nrhs, g.w.p, g.N);
  if (g.cplx) ck(launch_conj_interleaved(g.w.p, g.N, g.N, nr, st), "conj");
  double* hcol = g.H.p + (i64)cw * i * g.ldh;  // H[:, i] of rhs c at hcol + c * hstride
  {
    Prof pf("gmres_dots", 2. * g.N * kv * nr, 8. * (kv + 1) * g.N * nr);
    if (g.cplx)
      ck(launch_cdots_strided(g.V.p, g.vstride, kv, g.w.p, g.N / 2, nr, g.partial.p, cdots_chunks(g.N / 2), hcol,
                              hstride, st),
         "dots");
    else
      ck(launch_dots_strided(g.V.p, g.vstride, kv, g.w.p, g.N, nr, g.partial.p, g.nch, hcol, hstride, st), "dots");
  }
  {
    Prof pf("gmres_gs_update", 2. * g.N * kv * nr, 8. * (kv + 2) * g.N * nr);
    if (g.cplx)
      ck(launch_cgs_update(g.w.p, g.V.p, g.vstride, hcol, hstride, kv, g.N / 2, nr, -1.0, nullptr, st), "gs");
    else
      ck(launch_gs_update(g.w.p, g.V.p, g.vstride, hcol, hstride, kv, g.N, nr, -1.0, nullptr, st), "gs");
  }
  ck(launch_dots(g.w.p, 0, 1, g.w.p, g.N, nr, g.partial.p, g.nch, g.nrm2.p, st), "dots");
  // H[i + 1][i] = ||w|| (real; its imaginary part stays zero from the cycle's memset)
  ck(launch_scale_by_norm(g.w.p, g.V.p + (i + 1) * g.vstride, g.nrm2.p, hcol + cw * (i + 1), hstride, g.N, nr, st),
     "scale");
  if (g.early) {
    if (g.cplx)
      ck(launch_cgmres_estimate(g.H.p, g.ldh, (int)g.inner, (int)i, g.beta.p, g.normb.p, g.act.p, nr, g.tol,
                                g.ctl.p, st),
         "estimate");
    else
      ck(launch_gmres_estimate(g.H.p, g.ldh, (int)g.inner, (int)i, g.beta.p, g.normb.p, g.act.p, nr, g.tol,
                               g.ctl.p, st),
         "estimate");
  }
}

// rvec = || B - A X || / || B || per column (the reference's restart
// residual, solver.cpp:192-200).
static void gmres_true_residual(SolverBase& A, GmresState& g, cudaStream_t st) {
  const int nr = (int)g.nrhs;
  ck(cudaMemcpyAsync(g.R.p, g.X.p, sizeof(double) * g.vstride, cudaMemcpyDeviceToDevice, st), "R=X");
  if (g.cplx) ck(launch_conj_interleaved(g.R.p, g.N, g.N, nr, st), "conj");
  A.matvec(g.nrhs, g.R.p, g.N);
  ck(launch_axpby(g.R.p, g.Bc.p, -1.0, 1.0, g.vstride, st), "R=B-AX");
  ck(launch_dots(g.R.p, 0, 1, g.R.p, g.N, nr, g.partial.p, g.nch, g.nrm2.p, st), "dots");
  ck(launch_residual_norm_finish(g.nrm2.p, g.normb.p, g.rvec.p, nr, st), "resid");
}

// child: a stream for capturing the true-residual IF node (graph mode).
static void gmres_epilogue(SolverBase& A, GmresState& g, int graph, cudaGraphConditionalHandle hw, cudaStream_t st,
                           cudaStream_t child = nullptr) {
  const int nr = (int)g.nrhs;
  if (g.cplx) {
    ck(launch_cgmres_ls(g.H.p, g.ldh, (int)g.inner, g.beta.p, g.y.p, nr, st, g.ctl.p), "ls");
    ck(launch_cgs_update(g.X.p, g.V.p, g.vstride, g.y.p, 2 * g.inner, (int)g.inner, g.N / 2, nr, 1.0, g.act.p, st,
                         g.ctl.p),
       "x update");
  } else {
    ck(launch_gmres_ls(g.H.p, g.ldh, (int)g.inner, g.beta.p, g.y.p, nr, st, g.ctl.p), "ls");
    ck(launch_gs_update(g.X.p, g.V.p, g.vstride, g.y.p, g.inner, (int)g.inner, g.N, nr, 1.0, g.act.p, st, g.ctl.p),
       "x update");
  }
  if (!g.rec) {
    gmres_true_residual(A, g, st);
  } else {
    // R = Rr - AV y (the columns that are done keep whatever R holds)
    ck(cudaMemcpyAsync(g.R.p, g.Rr.p, sizeof(double) * g.vstride, cudaMemcpyDeviceToDevice, st), "R=Rr");
    if (g.cplx)
      ck(launch_cgs_update(g.R.p, g.AV.p, g.vstride, g.y.p, 2 * g.inner, (int)g.inner, g.N / 2, nr, -1.0, g.act.p, st,
                           g.ctl.p),
         "R update");
    else
      ck(launch_gs_update(g.R.p, g.AV.p, g.vstride, g.y.p, g.inner, (int)g.inner, g.N, nr, -1.0, g.act.p, st,
                          g.ctl.p),
         "R update");
    ck(launch_dots(g.R.p, 0, 1, g.R.p, g.N, nr, g.partial.p, g.nch, g.nrm2.p, st), "dots");
    ck(launch_residual_norm_finish(g.nrm2.p, g.normb.p, g.rvec.p, nr, st), "resid");
    ck(launch_gmres_need_true(g.rvec.p, g.act.p, g.it.p, (int)g.outer, nr, g.tol, g.ctl.p, st), "need true");
    if (graph) {
      h2dev_handle_s* h = A.h;
      cudaStreamCaptureStatus cs;
      cudaGraph_t bg = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t ndeps = 0;
      ck(cudaStreamGetCaptureInfo(st, &cs, nullptr, &bg, &deps, &ndeps), "capture info");
      cudaGraphConditionalHandle hc;
      ck(cudaGraphConditionalHandleCreate(&hc, bg, 0, 0), "conditional handle");
      ck(launch_graph_condition(hc, g.ctl.p + 4, 0, st), "certify condition");
      ck(cudaStreamGetCaptureInfo(st, &cs, nullptr, &bg, &deps, &ndeps), "capture info");
      cudaGraphNodeParams ip = {};
      ip.type = cudaGraphNodeTypeConditional;
      ip.conditional.handle = hc;
      ip.conditional.type = cudaGraphCondTypeIf;
      ip.conditional.size = 1;
      cudaGraphNode_t inode;
      ck(cudaGraphAddNode(&inode, bg, deps, ndeps, &ip), "if node");
      ck(cudaStreamUpdateCaptureDependencies(st, &inode, 1, cudaStreamSetCaptureDependencies), "capture deps");
      h->stream = child;
      ck(cudaStreamBeginCaptureToGraph(child, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                       cudaStreamCaptureModeRelaxed),
         "certify capture");
      gmres_true_residual(A, g, child);
      cudaGraph_t done = nullptr;
      ck(cudaStreamEndCapture(child, &done), "certify capture end");
      h->stream = st;
    } else {
      std::vector<int> c5 = g.ctl.download(st);
      if (c5[4]) gmres_true_residual(A, g, st);
    }
  }
  ck(launch_gmres_cycle_end(g.rvec.p, g.act.p, g.it.p, g.resh.p, (int)g.outer, g.tol, nr, g.ctl.p, st),
     "cycle end");
  if (graph) ck(launch_graph_condition(hw, g.ctl.p + 3, 0, st), "cycle condition");
}

// The whole solve as one graph: init kernel, then WHILE(another cycle)
// { prologue; [IF(not stopped) { Arnoldi step i }] for i < inner; epilogue }.
// A conditional handle belongs to one node, so each IF node has its own,
// set from the stop flag by a small kernel just before it.  Library launches
// go to h->stream, pointed at each body's capture stream in turn; the matvec
// keeps its near field on that stream while capturing (no side-stream fork),
// so the bodies hold kernels, copies and memsets only.
// A captured solve and the state buffers its nodes point at, kept on the
// operator's solver and replayed while the key (both solvers' identities and
// generations, the shape and the tolerance) still matches.
struct SolveGraph {
  uint64_t m_uid = 0, m_gen = 0, a_gen = 0;
  i64 nrhs = 0, inner = 0, outer = 0;
  int early = 0;
  double tol = 0.;
  GmresState g;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool matches(const SolverBase& A, const SolverBase& M, i64 nr, i64 in, i64 out, int ea, double t) const {
    return exec && m_uid == M.uid && m_gen == M.gen && a_gen == A.gen && nrhs == nr && inner == in && outer == out &&
           early == ea && tol == t;
  }
  ~SolveGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

static void gmres_graph(SolverBase& A, SolverBase& M, GmresState& g, SolveGraph& out) {
  h2dev_handle_s* h = A.h;
  cudaStream_t s0 = h->stream;
  cudaStream_t side = h->stream2;
  cudaStream_t sb = nullptr, ss = nullptr;
  // Restores the handle and releases the capture streams and graphs on every
  // exit; captures still open (after an error) are ended first, innermost
  // first, so no stream is destroyed mid-capture.
  struct Scope {
    h2dev_handle_s* h;
    cudaStream_t s0, side, sb = nullptr, ss = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~Scope() {
      for (cudaStream_t s : {ss, sb, s0}) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (s && cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
          cudaGraph_t junk = nullptr;
          cudaStreamEndCapture(s, &junk);
          if (junk && s == s0) cudaGraphDestroy(junk);
        }
      }
      cudaGetLastError();
      h->stream = s0;
      h->stream2 = side;
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      if (sb) cudaStreamDestroy(sb);
      if (ss) cudaStreamDestroy(ss);
    }
  } scope{h, s0, side};
  h->stream2 = nullptr;
  ck(cudaStreamCreateWithFlags(&sb, cudaStreamNonBlocking), "stream");
  scope.sb = sb;
  ck(cudaStreamCreateWithFlags(&ss, cudaStreamNonBlocking), "stream");
  scope.ss = ss;
  ck(cudaStreamBeginCapture(s0, cudaStreamCaptureModeRelaxed), "capture");
  cudaGraph_t g0 = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  cudaStreamCaptureStatus cs;
  ck(cudaStreamGetCaptureInfo(s0, &cs, nullptr, &g0, &deps, &ndeps), "capture info");
  cudaGraphConditionalHandle hw;
  ck(cudaGraphConditionalHandleCreate(&hw, g0, 0, 0), "conditional handle");
  ck(launch_gmres_init(g.act.p, g.it.p, g.resh.p, (int)g.outer, g.tol, (int)g.nrhs, g.ctl.p, s0), "init");
  ck(launch_graph_condition(hw, g.ctl.p + 3, 0, s0), "cycle condition");
  ck(cudaStreamGetCaptureInfo(s0, &cs, nullptr, &g0, &deps, &ndeps), "capture info");
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = hw;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  ck(cudaGraphAddNode(&wnode, g0, deps, ndeps, &wp), "while node");
  ck(cudaStreamUpdateCaptureDependencies(s0, &wnode, 1, cudaStreamSetCaptureDependencies), "capture deps");
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  h->stream = sb;
  ck(cudaStreamBeginCaptureToGraph(sb, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed), "body capture");
  gmres_prologue(M, g, sb);
  for (i64 i = 0; i < g.inner; i++) {
    cudaGraphConditionalHandle hi;
    ck(cudaGraphConditionalHandleCreate(&hi, body, 0, 0), "conditional handle");
    ck(launch_graph_condition(hi, g.ctl.p + 1, 1, sb), "step condition");  // step i runs unless stopped
    cudaGraph_t bg = nullptr;
    ck(cudaStreamGetCaptureInfo(sb, &cs, nullptr, &bg, &deps, &ndeps), "capture info");
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = hi;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode;
    ck(cudaGraphAddNode(&inode, bg, deps, ndeps, &ip), "if node");
    ck(cudaStreamUpdateCaptureDependencies(sb, &inode, 1, cudaStreamSetCaptureDependencies), "capture deps");
    h->stream = ss;
    ck(cudaStreamBeginCaptureToGraph(ss, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                     cudaStreamCaptureModeRelaxed),
       "step capture");
    gmres_step(A, M, g, i, ss);
    cudaGraph_t done = nullptr;
    ck(cudaStreamEndCapture(ss, &done), "step capture end");
    h->stream = sb;
  }
  gmres_epilogue(A, g, 1, hw, sb, ss);
  cudaGraph_t bdone = nullptr;
  ck(cudaStreamEndCapture(sb, &bdone), "body capture end");
  h->stream = s0;
  ck(cudaStreamEndCapture(s0, &scope.graph), "capture end");
  ck(cudaGraphInstantiate(&scope.exec, scope.graph, 0), "graph instantiate");
  out.graph = scope.graph;
  out.exec = scope.exec;
  scope.graph = nullptr;
  scope.exec = nullptr;
}

static void gmres_alloc(GmresState& g, cudaStream_t st) {
  const i64 nrhs = g.nrhs, inner = g.inner, outer = g.outer;
  g.V.alloc((size_t)(inner + 1) * g.vstride);
  g.w.alloc(g.vstride);
  g.R.alloc(g.vstride);
  g.Bc.alloc(g.vstride);
  g.X.alloc(g.vstride);
  const size_t cw = g.cplx ? 2 : 1;
  g.H.alloc(cw * g.ldh * inner * nrhs);
  g.y.alloc(cw * inner * nrhs);
  g.beta.alloc(nrhs);
  g.nrm2.alloc(nrhs);
  g.normb.alloc(nrhs);
  g.rvec.alloc(nrhs);
  g.resh.alloc((size_t)(outer + 1) * nrhs);
  g.act.alloc(nrhs);
  g.it.alloc(nrhs);
  g.ctl.alloc(5);
  if (g.rec) {
    g.AV.alloc((size_t)inner * g.vstride);
    g.Rr.alloc(g.vstride);
  }
  g.partial.alloc(cw * g.nch * (inner + 1) * nrhs);
  g.y.zero(st);
}

static int gmres(SolverBase& A, SolverBase& M, double tol, i64 nrhs, double* dX, const double* dB, i64 ld, i64 inner,
                 i64 outer, int early_exit, double* resid, i64* iters) {
  require(A.lenX() == M.lenX(), "gmres: A and M sizes differ");
  require(A.complex_form == M.complex_form, "gmres: operator and preconditioner kernels differ in kind");
  require(inner >= 1 && inner <= 16 && outer >= 0 && nrhs >= 1, "gmres: inner must be in [1,16]");
  cudaStream_t st = A.h->stream;
  const int nr = (int)nrhs;
  const int early = early_exit ? 1 : 0;
  const bool use_graph = A.h->graph_solve && !A.h->prof && A.h == M.h;
  // Graph path: the solve is captured once per (operator, preconditioner,
  // shape, tolerance) and replayed by later calls -- a serving system solving
  // batch after batch pays the capture once.  Everything a capture must not
  // do (plan builds, uploads, allocations, autotuning) happens in prepare().
  std::shared_ptr<SolveGraph> sg;
  GmresState local;
  GmresState* gp = &local;
  if (use_graph) {
    A.prepare(nrhs);
    M.prepare(nrhs);
    if (A.solve_graph && A.solve_graph->matches(A, M, nrhs, inner, outer, early, tol)) {
      sg = A.solve_graph;
    } else {
      A.solve_graph.reset();
      sg = std::make_shared<SolveGraph>();
      sg->m_uid = M.uid;
      sg->m_gen = M.gen;
      sg->a_gen = A.gen;
      sg->nrhs = nrhs;
      sg->inner = inner;
      sg->outer = outer;
      sg->early = early;
      sg->tol = tol;
    }
    gp = &sg->g;
  }
  GmresState& g = *gp;
  if (!g.V.p) {
    g.N = A.lenX();
    g.nrhs = nrhs;
    g.inner = inner;
    g.outer = outer;
    g.ldh = (int)inner + 1;
    g.vstride = g.N * nrhs;
    g.tol = tol;
    g.early = early;
    g.cplx = A.complex_form ? 1 : 0;
    g.rec = early;
    g.nch = dots_chunks(g.N);
    gmres_alloc(g, st);
  }
  g.resh.zero(st);
  for (i64 c = 0; c < nrhs; c++) {
    ck(cudaMemcpyAsync(g.Bc.p + c * g.N, dB + c * ld, sizeof(double) * g.N, cudaMemcpyDeviceToDevice, st), "copy B");
    ck(cudaMemcpyAsync(g.X.p + c * g.N, dX + c * ld, sizeof(double) * g.N, cudaMemcpyDeviceToDevice, st), "copy X");
  }
  ck(launch_dots(g.Bc.p, 0, 1, g.Bc.p, g.N, nr, g.partial.p, g.nch, g.nrm2.p, st), "dots");
  {
    std::vector<double> n2 = g.nrm2.download(st), hn(nrhs);
    for (i64 c = 0; c < nrhs; c++) {
      hn[c] = std::sqrt(n2[c]);
      if (hn[c] == 0.) hn[c] = 1.;
    }
    g.normb.upload(hn);
  }
  // The reference starts from the given X with R = B (not B - A X) in its
  // first cycle (solver.cpp:157); the initial guess is zero in every caller.
  ck(cudaMemcpyAsync(g.R.p, g.Bc.p, sizeof(double) * g.vstride, cudaMemcpyDeviceToDevice, st), "R=B");
  if (use_graph) {
    if (!sg->exec) gmres_graph(A, M, g, *sg);
    A.solve_graph = sg;
    A.h->tc_pending = true;  // the graph may hold mbarrier-pipelined kernels
    ck(cudaGraphLaunch(sg->exec, st), "graph launch");
    ck(cudaStreamSynchronize(st), "sync");
  } else {
    ck(launch_gmres_init(g.act.p, g.it.p, g.resh.p, (int)outer, tol, nr, g.ctl.p, st), "init");
    bool any = 0 < outer && tol <= 1.;
    while (any) {
      gmres_prologue(M, g, st);
      for (i64 i = 0; i < inner; i++) {
        gmres_step(A, M, g, i, st);
        if (g.early) {
          int stop = 0;
          ck(cudaStreamSynchronize(st), "sync");
          ck(cudaMemcpy(&stop, g.ctl.p + 1, sizeof(int), cudaMemcpyDeviceToHost), "stop flag");
          if (stop) break;
        }
      }
      gmres_epilogue(A, g, 0, 0, st);
      std::vector<int> c4 = g.ctl.download(st);
      any = c4[3] != 0;
    }
  }
  for (i64 c = 0; c < nrhs; c++)
    ck(cudaMemcpyAsync(dX + c * ld, g.X.p + c * g.N, sizeof(double) * g.N, cudaMemcpyDeviceToDevice, st), "copy X out");
  std::vector<double> res = g.resh.download(st);
  std::vector<int> it = g.it.download(st);
  ck(cudaGetLastError(), "gmres");
  check_tc(A.h);
  check_tc(M.h);
  bool conv = true;
  for (i64 c = 0; c < nrhs; c++) {
    require(it[c] >= 0 && it[c] <= outer, "gmres: cycle count out of range (device control state)");
    for (i64 k = 0; k <= outer; k++) resid[c * (outer + 1) + k] = res[c * (outer + 1) + k];
    if (iters) iters[c] = it[c];
    if (!(res[c * (outer + 1) + it[c]] < tol)) conv = false;
  }
  return conv ? H2DEV_OK : H2DEV_ERR_NOCONV;
}

}  // namespace h2b

struct h2dev_solver_s {
  std::unique_ptr<h2b::SolverBase> impl;
};

using namespace h2b;

#define H2_API_BEGIN try {
#define H2_API_END                                \
  }                                               \
  catch (const H2Error& e) {                      \
    g_last_error = e.msg;                         \
    return e.code;                                \
  }                                               \
  catch (const std::bad_alloc&) {                 \
    g_last_error = "host allocation failed";      \
    return H2DEV_ERR_OOM;                         \
  }                                               \
  catch (const std::exception& e) {               \
    g_last_error = e.what();                      \
    return H2DEV_ERR_ARG;                         \
  }

static KernelParams make_kp(int kernel, double singularity, double alpha) {
  require(kernel == H2DEV_KERNEL_LAPLACE || kernel == H2DEV_KERNEL_YUKAWA || kernel == H2DEV_KERNEL_QUADRATIC ||
              kernel == H2DEV_KERNEL_HELMHOLTZ,
          "unknown kernel");
  require(singularity != 0., "singularity must be nonzero");
  KernelParams kp;
  kp.kind = kernel;
  kp.diag = 1. / singularity;
  kp.alpha = alpha;
  return kp;
}

extern "C" {

const char* h2dev_last_error_message(void) { return g_last_error.c_str(); }

int h2_uniform_unit_cube_rnd(double* bodies, int64_t nbodies, double diameter, int64_t dim, unsigned seed) {
  H2_API_BEGIN
  require(bodies && nbodies >= 0, "bad arguments");
  uniform_unit_cube_rnd(bodies, nbodies, diameter, dim, seed);
  return H2DEV_OK;
  H2_API_END
}

int h2_uniform_rhs(double* x, int64_t n) {
  H2_API_BEGIN
  require(x && n >= 0, "bad arguments");
  uniform_rhs(x, n);
  return H2DEV_OK;
  H2_API_END
}

int64_t h2_levels_for(int64_t nbodies, int64_t leaf) {
  if (nbodies <= 0 || leaf <= 0) return -1;
  leaf = nbodies < leaf ? nbodies : leaf;
  return (int64_t)std::log2((double)nbodies / leaf);
}

int h2_build_tree(double* bodies, int64_t nbodies, int64_t levels, int64_t* cell_child, int64_t* cell_body,
                  double* cell_R, double* cell_C) {
  H2_API_BEGIN
  require(bodies && nbodies > 0 && levels >= 0 && levels < 40, "bad arguments");
  require(((int64_t)1 << levels) <= nbodies, "more leaves than bodies");
  int64_t ncells = ((int64_t)2 << levels) - 1;
  std::vector<Cell> cells(ncells);
  build_binary_tree(cells.data(), bodies, nbodies, levels);
  for (int64_t c = 0; c < ncells; c++) {
    for (int k = 0; k < 2; k++) {
      if (cell_child) cell_child[2 * c + k] = cells[c].child[k];
      if (cell_body) cell_body[2 * c + k] = cells[c].body[k];
    }
    for (int k = 0; k < 3; k++) {
      if (cell_R) cell_R[3 * c + k] = cells[c].R[k];
      if (cell_C) cell_C[3 * c + k] = cells[c].C[k];
    }
  }
  return H2DEV_OK;
  H2_API_END
}

int h2_build_tree_capped(double* bodies, int64_t nbodies, int64_t levels, int64_t leaf_min, int64_t leaf_max,
                         int64_t* cell_child, int64_t* cell_body, double* cell_R, double* cell_C) {
  H2_API_BEGIN
  require(bodies && nbodies > 0 && levels >= 0 && levels < 40, "bad arguments");
  require(leaf_min >= 1 && leaf_min <= leaf_max, "need 1 <= leaf_min <= leaf_max");
  require(leaf_min * ((int64_t)1 << levels) <= nbodies && nbodies <= leaf_max * ((int64_t)1 << levels),
          "leaf_min * 2^levels <= nbodies <= leaf_max * 2^levels does not hold");
  int64_t ncells = ((int64_t)2 << levels) - 1;
  std::vector<Cell> cells(ncells);
  build_binary_tree_capped(cells.data(), bodies, nbodies, levels, leaf_min, leaf_max);
  for (int64_t c = 0; c < ncells; c++) {
    for (int k = 0; k < 2; k++) {
      if (cell_child) cell_child[2 * c + k] = cells[c].child[k];
      if (cell_body) cell_body[2 * c + k] = cells[c].body[k];
    }
    for (int k = 0; k < 3; k++) {
      if (cell_R) cell_R[3 * c + k] = cells[c].R[k];
      if (cell_C) cell_C[3 * c + k] = cells[c].C[k];
    }
  }
  return H2DEV_OK;
  H2_API_END
}

int h2_pair_csr(char kind, int64_t ncells, const int64_t* cell_child, const int64_t* cell_body, const double* cell_R,
                const double* cell_C, double theta, int64_t* row, int64_t* col, int64_t cap, int64_t* nnz) {
  H2_API_BEGIN
  require(ncells > 0 && cell_child && cell_body && cell_R && cell_C && row && nnz, "bad arguments");
  require(kind == 'N' || kind == 'n' || kind == 'F' || kind == 'f', "kind must be N or F");
  std::vector<Cell> cells(ncells);
  for (int64_t c = 0; c < ncells; c++) {
    for (int k = 0; k < 2; k++) {
      cells[c].child[k] = cell_child[2 * c + k];
      cells[c].body[k] = cell_body[2 * c + k];
    }
    for (int k = 0; k < 3; k++) {
      cells[c].R[k] = cell_R[3 * c + k];
      cells[c].C[k] = cell_C[3 * c + k];
    }
  }
  PairCSR csr = build_pair_csr(kind, cells, theta);
  for (int64_t i = 0; i <= ncells; i++) row[i] = csr.row[i];
  *nnz = (int64_t)csr.col.size();
  if (col && cap >= *nnz)
    for (size_t k = 0; k < csr.col.size(); k++) col[k] = csr.col[k];
  return H2DEV_OK;
  H2_API_END
}

int h2dev_handle_create(int device, h2dev_handle_t* out) {
  H2_API_BEGIN
  require(out != nullptr, "null out");
  ck(cudaSetDevice(device), "cudaSetDevice");
  auto* h = new h2dev_handle_s();
  h->device = device;
  int least = 0, greatest = 0;
  ck(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priority range");
  cudaError_t e = cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking, greatest);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&h->stream2, cudaStreamNonBlocking, least);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->d_tc_err, 256);
  if (e == cudaSuccess) e = cudaMemset(h->d_tc_err, 0, sizeof(int));
  if (e != cudaSuccess) {
    if (h->d_tc_err) cudaFree(h->d_tc_err);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->stream2) cudaStreamDestroy(h->stream2);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    ck(e, "cudaStreamCreate");
  }
  *out = h;
  return H2DEV_OK;
  H2_API_END
}

// Drops one reference; the last one frees the stream, events and staging.
static void handle_release(h2dev_handle_s* h) {
  if (!h || --h->refs > 0) return;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  stage_release(h);
  h->clear();
  for (cudaEvent_t e : h->pool) cudaEventDestroy(e);
  if (h->t0) cudaEventDestroy(h->t0);
  if (h->t1) cudaEventDestroy(h->t1);
  cache_trim(h);
  cudaStreamSynchronize(h->stream2);
  cudaEventDestroy(h->ev_fork);
  cudaEventDestroy(h->ev_join);
  cudaStreamDestroy(h->stream2);
  cudaStreamDestroy(h->stream);
  cudaFree(h->d_tc_err);
  delete h;
}

int h2dev_handle_destroy(h2dev_handle_t h) {
  H2_API_BEGIN
  handle_release(h);
  return H2DEV_OK;
  H2_API_END
}

int h2dev_handle_memory(h2dev_handle_t h, int64_t* live_bytes, int64_t* cached_bytes) {
  H2_API_BEGIN
  require(h != nullptr, "null handle");
  if (live_bytes) *live_bytes = (int64_t)h->live_bytes;
  if (cached_bytes) *cached_bytes = (int64_t)h->cached_bytes;
  return H2DEV_OK;
  H2_API_END
}

int h2dev_handle_memory_peak(h2dev_handle_t h, int64_t* peak_live_bytes, int reset) {
  H2_API_BEGIN
  require(h != nullptr && peak_live_bytes != nullptr, "null argument");
  *peak_live_bytes = (int64_t)h->peak_live_bytes;
  if (reset) h->peak_live_bytes = h->live_bytes;
  return H2DEV_OK;
  H2_API_END
}

int h2dev_handle_trim(h2dev_handle_t h) {
  H2_API_BEGIN
  require(h != nullptr, "null handle");
  ck(cudaSetDevice(h->device), "cudaSetDevice");
  cache_trim(h);
  return H2DEV_OK;
  H2_API_END
}

int h2dev_handle_synchronize(h2dev_handle_t h) {
  H2_API_BEGIN
  require(h != nullptr, "null handle");
  ck(cudaStreamSynchronize(h->stream), "sync");
  return H2DEV_OK;
  H2_API_END
}

int h2dev_solver_create(h2dev_handle_t h, int kernel, double singularity, double alpha, double epi, int64_t rank,
                        int64_t leveled_rank, int64_t ncells, const int64_t* cell_child, const int64_t* cell_body,
                        const double* cell_R, const double* cell_C, double theta, const double* bodies,
                        int64_t nbodies, int64_t levels, int64_t samples, int precision, h2dev_solver_t* out) {
  H2_API_BEGIN
  require(h && out && cell_child && cell_body && cell_R && cell_C && bodies, "null argument");
  require(levels >= 0 && ncells == ((int64_t)2 << levels) - 1, "ncells must be 2^(levels+1)-1");
  require(nbodies > 0 && epi >= 0., "bad sizes");
  require(precision == H2DEV_FP64 || precision == H2DEV_FP32, "precision");
  ck(cudaSetDevice(h->device), "cudaSetDevice");
  CurHandle ch(h);
  BuildArgs a;
  a.kp = make_kp(kernel, singularity, alpha);
  a.epi = epi;
  a.rank = rank;
  a.leveled_rank = leveled_rank;
  a.levels = levels;
  a.nbodies = nbodies;
  a.samples = samples;
  a.theta = theta;
  a.bodies = bodies;
  a.cells.resize(ncells);
  for (int64_t c = 0; c < ncells; c++) {
    for (int k = 0; k < 2; k++) {
      a.cells[c].child[k] = cell_child[2 * c + k];
      a.cells[c].body[k] = cell_body[2 * c + k];
    }
    for (int k = 0; k < 3; k++) {
      a.cells[c].R[k] = cell_R[3 * c + k];
      a.cells[c].C[k] = cell_C[3 * c + k];
    }
  }
  require(a.cells[0].body[0] == 0 && a.cells[0].body[1] == nbodies, "root cell must span all bodies");
  // Helmholtz: body i becomes unknowns 2i (real part) and 2i + 1 (imaginary
  // part) of the real form, tagged in bit 0 of x; every cell keeps its
  // geometry and owns the unknowns of its bodies; ranks and far samples
  // count real unknowns, two per complex degree of freedom.
  std::vector<double> helm_bodies;
  const bool helm = kernel == H2DEV_KERNEL_HELMHOLTZ;
  if (helm) {
    require(nbodies < ((int64_t)1 << 40), "too many bodies");
    helm_bodies.resize((size_t)6 * nbodies);
    for (int64_t i = 0; i < nbodies; i++) {
      int64_t xb;
      std::memcpy(&xb, &bodies[3 * i], sizeof(xb));
      for (int t = 0; t < 2; t++) {
        const int64_t xt = (xb & ~(int64_t)1) | t;
        std::memcpy(&helm_bodies[6 * i + 3 * t], &xt, sizeof(xt));
        helm_bodies[6 * i + 3 * t + 1] = bodies[3 * i + 1];
        helm_bodies[6 * i + 3 * t + 2] = bodies[3 * i + 2];
      }
    }
    a.bodies = helm_bodies.data();
    a.nbodies = 2 * nbodies;
    a.rank = 2 * rank;
    a.leveled_rank = 2 * leveled_rank;
    a.samples = samples > 0 ? 2 * samples : samples;
    for (auto& c : a.cells) {
      c.body[0] *= 2;
      c.body[1] *= 2;
    }
  }
  std::unique_ptr<h2dev_solver_s> s(new h2dev_solver_s());
  if (precision == H2DEV_FP64) {
    auto* p = new Solver<double>();
    s->impl.reset(p);
    p->h = h;
    p->build(a);
  } else {
    auto* p = new Solver<float>();
    s->impl.reset(p);
    p->h = h;
    p->build(a);
  }
  s->impl->complex_form = helm;
  h->refs++;
  *out = s.release();
  return H2DEV_OK;
  H2_API_END
}

int h2dev_solver_destroy(h2dev_solver_t s) {
  H2_API_BEGIN
  if (s) {
    h2dev_handle_s* h = s->impl ? s->impl->h : nullptr;
    if (h) {
      cudaSetDevice(h->device);
      CurHandle ch(h);
      delete s;
      cudaStreamSynchronize(h->stream);
    } else {
      delete s;
    }
    handle_release(h);
  }
  return H2DEV_OK;
  H2_API_END
}

int h2dev_solver_shape(h2dev_solver_t s, int64_t* levels, int64_t* lenX) {
  H2_API_BEGIN
  require(s && s->impl, "null solver");
  if (levels) *levels = s->impl->nlevels();
  if (lenX) *lenX = s->impl->lenX();
  return H2DEV_OK;
  H2_API_END
}

int h2dev_solver_level_dims(h2dev_solver_t s, int64_t level, int64_t* dims, int64_t* ranks) {
  H2_API_BEGIN
  require(s && s->impl, "null solver");
  s->impl->level_dims(level, dims, ranks);
  return H2DEV_OK;
  H2_API_END
}

static void with_device_copy(h2dev_handle_s* h, int64_t n, int64_t nrhs, double* X, int64_t ld,
                             const std::function<void(double*)>& fn) {
  DVec<double> d;
  d.alloc((size_t)n * nrhs);
  ck(cudaMemcpy2DAsync(d.p, sizeof(double) * n, X, sizeof(double) * ld, sizeof(double) * n, nrhs,
                       cudaMemcpyHostToDevice, h->stream),
     "H2D");
  fn(d.p);
  ck(cudaMemcpy2DAsync(X, sizeof(double) * ld, d.p, sizeof(double) * n, sizeof(double) * n, nrhs,
                       cudaMemcpyDeviceToHost, h->stream),
     "D2H");
  ck(cudaStreamSynchronize(h->stream), "sync");
}

int h2dev_matvec(h2dev_solver_t s, int64_t nrhs, double* X, int64_t ldx) {
  H2_API_BEGIN
  require(s && s->impl && X, "null argument");
  SolverBase* p = s->impl.get();
  CurHandle ch(p->h);
  require(nrhs > 0 && ldx >= p->lenX(), "bad nrhs/ld");
  with_device_copy(p->h, p->lenX(), nrhs, X, ldx, [&](double* d) {
    if (p->complex_form) ck(launch_conj_interleaved(d, p->lenX(), p->lenX(), (int)nrhs, p->h->stream), "conj");
    p->matvec(nrhs, d, p->lenX());
  });
  check_tc(p->h);
  return H2DEV_OK;
  H2_API_END
}

int h2dev_matvec_device(h2dev_solver_t s, int64_t nrhs, double* dX, int64_t ldx) {
  H2_API_BEGIN
  require(s && s->impl && dX, "null argument");
  CurHandle ch(s->impl->h);
  if (s->impl->complex_form)
    ck(launch_conj_interleaved(dX, s->impl->lenX(), ldx, (int)nrhs, s->impl->h->stream), "conj");
  s->impl->matvec(nrhs, dX, ldx);
  check_tc(s->impl->h);
  return H2DEV_OK;
  H2_API_END
}

int h2dev_factorize(h2dev_solver_t s, int* info_per_level) {
  H2_API_BEGIN
  require(s && s->impl, "null solver");
  CurHandle ch(s->impl->h);
  std::vector<int> info(s->impl->nlevels() + 1, 0);
  s->impl->factorize(info.data());
  int any = 0;
  for (size_t l = 0; l < info.size(); l++) {
    if (info_per_level) info_per_level[l] = info[l];
    any |= info[l] != 0;
  }
  return any ? H2DEV_ERR_SINGULAR : H2DEV_OK;
  H2_API_END
}

int h2dev_solve_precondition(h2dev_solver_t s, int64_t nrhs, double* X, int64_t ldx) {
  H2_API_BEGIN
  require(s && s->impl && X, "null argument");
  SolverBase* p = s->impl.get();
  CurHandle ch(p->h);
  require(nrhs > 0 && ldx >= p->lenX(), "bad nrhs/ld");
  with_device_copy(p->h, p->lenX(), nrhs, X, ldx, [&](double* d) {
    p->precondition(nrhs, d, p->lenX());
    if (p->complex_form) ck(launch_conj_interleaved(d, p->lenX(), p->lenX(), (int)nrhs, p->h->stream), "conj");
  });
  check_tc(p->h);
  return H2DEV_OK;
  H2_API_END
}

int h2dev_solve_precondition_device(h2dev_solver_t s, int64_t nrhs, double* dX, int64_t ldx) {
  H2_API_BEGIN
  require(s && s->impl && dX, "null argument");
  CurHandle ch(s->impl->h);
  s->impl->precondition(nrhs, dX, ldx);
  if (s->impl->complex_form)
    ck(launch_conj_interleaved(dX, s->impl->lenX(), ldx, (int)nrhs, s->impl->h->stream), "conj");
  check_tc(s->impl->h);
  return H2DEV_OK;
  H2_API_END
}

int h2dev_solve_gmres_device(h2dev_solver_t A, h2dev_solver_t M, double tol, int64_t nrhs, double* dX,
                             const double* dB, int64_t ld, int64_t inner, int64_t outer, int early_exit,
                             double* resid, int64_t* iters) {
  H2_API_BEGIN
  require(A && A->impl && M && M->impl && dX && dB && resid, "null argument");
  require(ld >= A->impl->lenX(), "bad ld");
  require(A->impl->complex_form == M->impl->complex_form, "operator and preconditioner kernels differ in kind");
  CurHandle ch(A->impl->h);
  // Helmholtz: complex GMRES on K x = B (vectors conjugated around each
  // real-form matvec and preconditioner solve inside).
  return gmres(*A->impl, *M->impl, tol, nrhs, dX, dB, ld, inner, outer, early_exit, resid, iters);
  H2_API_END
}

int h2dev_solve_gmres(h2dev_solver_t A, h2dev_solver_t M, double tol, int64_t nrhs, double* X, const double* B,
                      int64_t ld, int64_t inner, int64_t outer, int early_exit, double* resid, int64_t* iters) {
  H2_API_BEGIN
  require(A && A->impl && M && M->impl && X && B && resid, "null argument");
  SolverBase* a = A->impl.get();
  CurHandle ch(a->h);
  const int64_t n = a->lenX();
  require(nrhs > 0 && ld >= n, "bad nrhs/ld");
  require(a->complex_form == M->impl->complex_form, "operator and preconditioner kernels differ in kind");
  cudaStream_t st = a->h->stream;
  DVec<double> dX, dB;
  dX.alloc((size_t)n * nrhs);
  dB.alloc((size_t)n * nrhs);
  ck(cudaMemcpy2DAsync(dX.p, sizeof(double) * n, X, sizeof(double) * ld, sizeof(double) * n, nrhs,
                       cudaMemcpyHostToDevice, st), "H2D");
  ck(cudaMemcpy2DAsync(dB.p, sizeof(double) * n, B, sizeof(double) * ld, sizeof(double) * n, nrhs,
                       cudaMemcpyHostToDevice, st), "H2D");
  int rc = gmres(*a, *M->impl, tol, nrhs, dX.p, dB.p, n, inner, outer, early_exit, resid, iters);
  ck(cudaMemcpy2DAsync(X, sizeof(double) * ld, dX.p, sizeof(double) * n, sizeof(double) * n, nrhs,
                       cudaMemcpyDeviceToHost, st), "D2H");
  ck(cudaStreamSynchronize(st), "sync");
  return rc;
  H2_API_END
}

int h2dev_gen_block(h2dev_handle_t h, int kernel, double singularity, double alpha, const double* bi, int64_t m,
                    const double* bj, int64_t n, double* out) {
  H2_API_BEGIN
  require(h && bi && bj && out && m >= 0 && n >= 0, "bad arguments");
  require(m * n < ((int64_t)1 << 31), "block too large");
  KernelParams kp = make_kp(kernel, singularity, alpha);
  if (m == 0 || n == 0) return H2DEV_OK;
  CurHandle ch(h);
  DVec<double> di, dj, dout;
  di.upload(std::vector<double>(bi, bi + 3 * m));
  dj.upload(std::vector<double>(bj, bj + 3 * n));
  if (kernel == H2DEV_KERNEL_HELMHOLTZ) {
    // Rows: both components of each bi body; columns: the real part of each
    // bj body.  The 2m x n real block is the m x n complex block with its
    // real and imaginary parts interleaved.
    require(2 * m * n < ((int64_t)1 << 31), "block too large");
    DVec<double> ei, ej;
    ei.alloc((size_t)6 * m);
    ej.alloc((size_t)3 * n);
    ck(launch_helm_expand(di.p, m, 2, ei.p, h->stream), "expand");
    ck(launch_helm_expand(dj.p, n, 1, ej.p, h->stream), "expand");
    std::swap(di, ei);
    std::swap(dj, ej);
    m *= 2;
  }
  dout.alloc((size_t)m * n);
  std::vector<GenTask> gt(1);
  gt[0].bi = di.p;
  gt[0].bj = dj.p;
  gt[0].m = (int)m;
  gt[0].n = (int)n;
  gt[0].out_off = 0;
  gt[0].ld = m;
  DVec<GenTask> dg;
  dg.upload(gt);
  ck(launch_gen_blocks<double>(kp, dg.p, 1, m, dout.p, h->stream, 0, gen_err()), "gen");
  ck(cudaStreamSynchronize(h->stream), "sync");
  ck(cudaMemcpy(out, dout.p, sizeof(double) * m * n, cudaMemcpyDeviceToHost), "D2H");
  return H2DEV_OK;
  H2_API_END
}

int h2dev_dense_matvec_device(h2dev_handle_t h, int kernel, double singularity, double alpha, const double* dbodies,
                              int64_t n, int64_t nrhs, const double* dX, double* dY, int64_t ld) {
  H2_API_BEGIN
  KernelParams kp = make_kp(kernel, singularity, alpha);
  const bool helm = kernel == H2DEV_KERNEL_HELMHOLTZ;
  require(h && dbodies && dX && dY && n > 0 && nrhs > 0 && ld >= (helm ? 2 * n : n), "bad arguments");
  CurHandle ch(h);
  if (helm) {
    // K X = S conj(X) over the tagged real-form bodies (2n unknowns).
    DVec<double> eb, cx;
    eb.alloc((size_t)6 * n);
    cx.alloc((size_t)2 * n * nrhs);
    ck(launch_helm_expand(dbodies, n, 2, eb.p, h->stream), "expand");
    ck(cudaMemcpy2DAsync(cx.p, sizeof(double) * 2 * n, dX, sizeof(double) * ld, sizeof(double) * 2 * n, nrhs,
                         cudaMemcpyDeviceToDevice, h->stream),
       "copy");
    ck(launch_conj_interleaved(cx.p, 2 * n, 2 * n, (int)nrhs, h->stream), "conj");
    Prof pf("dense_matvec", 8. * (double)n * n * nrhs, 32. * n * nrhs);
    ck(launch_dense_matvec(kp, eb.p, 2 * n, cx.p, 2 * n, dY, ld, (int)nrhs, h->stream), "dense_matvec");
    return H2DEV_OK;
  }
  Prof pf("dense_matvec", 2. * (double)n * n * nrhs, 16. * n * nrhs);
  ck(launch_dense_matvec(kp, dbodies, n, dX, ld, dY, ld, (int)nrhs, h->stream), "dense_matvec");
  return H2DEV_OK;
  H2_API_END
}

int h2dev_dense_matvec(h2dev_handle_t h, int kernel, double singularity, double alpha, const double* bodies,
                       int64_t n, int64_t nrhs, const double* X, double* Y, int64_t ld) {
  H2_API_BEGIN
  KernelParams kp = make_kp(kernel, singularity, alpha);
  const bool helm = kernel == H2DEV_KERNEL_HELMHOLTZ;
  const int64_t len = helm ? 2 * n : n;  // doubles per column
  require(h && bodies && X && Y && n > 0 && nrhs > 0 && ld >= len, "bad arguments");
  CurHandle ch(h);
  DVec<double> db, dx, dy;
  db.upload(std::vector<double>(bodies, bodies + 3 * n));
  dx.alloc((size_t)len * nrhs);
  dy.alloc((size_t)len * nrhs);
  // On the handle's (non-blocking) stream: a plain cudaMemcpy from pageable
  // memory may return before its DMA lands, so the kernels below would not be
  // ordered after it.
  ck(cudaMemcpy2DAsync(dx.p, sizeof(double) * len, X, sizeof(double) * ld, sizeof(double) * len, nrhs,
                       cudaMemcpyHostToDevice, h->stream), "H2D");
  if (helm) {
    // K X = S conj(X) over the tagged real-form bodies (2n unknowns).
    DVec<double> eb;
    eb.alloc((size_t)6 * n);
    ck(launch_helm_expand(db.p, n, 2, eb.p, h->stream), "expand");
    ck(launch_conj_interleaved(dx.p, len, len, (int)nrhs, h->stream), "conj");
    ck(launch_dense_matvec(kp, eb.p, len, dx.p, len, dy.p, len, (int)nrhs, h->stream), "dense_matvec");
  } else {
    ck(launch_dense_matvec(kp, db.p, n, dx.p, n, dy.p, n, (int)nrhs, h->stream), "dense_matvec");
  }
  ck(cudaStreamSynchronize(h->stream), "sync");
  ck(cudaMemcpy2D(Y, sizeof(double) * ld, dy.p, sizeof(double) * len, sizeof(double) * len, nrhs,
                  cudaMemcpyDeviceToHost), "D2H");
  return H2DEV_OK;
  H2_API_END
}

int h2dev_profile_enable(h2dev_handle_t h, int on) {
  H2_API_BEGIN
  require(h != nullptr, "null handle");
  ck(cudaStreamSynchronize(h->stream), "sync");
  h->clear();
  h->prof = on != 0;
  return H2DEV_OK;
  H2_API_END
}

int h2dev_profile_report(h2dev_handle_t h, int64_t cap, char* names, int64_t* launches, double* ms, double* flops,
                         double* bytes, int64_t* count) {
  H2_API_BEGIN
  require(h && count, "null argument");
  ck(cudaStreamSynchronize(h->stream), "sync");
  std::vector<std::string> keys;
  std::vector<int64_t> nl;
  std::vector<double> t, f, b;
  for (const auto& r : h->recs) {
    float e = 0.f;
    ck(cudaEventElapsedTime(&e, r.a, r.b), "cudaEventElapsedTime");
    size_t k = 0;
    while (k < keys.size() && keys[k] != r.name) k++;
    if (k == keys.size()) {
      keys.push_back(r.name);
      nl.push_back(0);
      t.push_back(0.);
      f.push_back(0.);
      b.push_back(0.);
    }
    nl[k]++;
    t[k] += e;
    f[k] += r.flops;
    b[k] += r.bytes;
  }
  *count = (int64_t)keys.size();
  for (size_t k = 0; k < keys.size() && (int64_t)k < cap; k++) {
    if (names) {
      std::strncpy(names + 48 * k, keys[k].c_str(), 47);
      names[48 * k + 47] = 0;
    }
    if (launches) launches[k] = nl[k];
    if (ms) ms[k] = t[k];
    if (flops) flops[k] = f[k];
    if (bytes) bytes[k] = b[k];
  }
  return H2DEV_OK;
  H2_API_END
}

int h2dev_batched_gemm_device(h2dev_handle_t h, int precision, int64_t batch, int64_t nterms, int64_t m, int64_t n,
                              int64_t k, int opA, int opB, double alpha, const void* A, int64_t lda, int64_t strideA,
                              const void* B, int64_t ldb, int64_t strideB, double beta, void* C, int64_t ldc,
                              int64_t strideC) {
  H2_API_BEGIN
  require(h && A && B && C, "null argument");
  require(precision == H2DEV_FP64 || precision == H2DEV_FP32, "precision");
  require(batch >= 0 && nterms >= 0 && m >= 0 && n >= 0 && k >= 0, "negative size");
  require(m < (1 << 30) && n < (1 << 30) && k < (1 << 30), "size too large");
  require((opA == 0 || opA == 1) && (opB == 0 || opB == 1), "op must be 0 or 1");
  require(lda >= std::max<int64_t>(1, opA ? k : m) && ldb >= std::max<int64_t>(1, opB ? n : k) &&
              ldc >= std::max<int64_t>(1, m),
          "leading dimension too small");
  ck(cudaSetDevice(h->device), "cudaSetDevice");
  CurHandle ch(h);
  if (precision == H2DEV_FP64)
    batched_gemm<double>(batch, nterms, m, n, k, opA, opB, alpha, (const double*)A, lda, strideA, (const double*)B,
                         ldb, strideB, beta, (double*)C, ldc, strideC, h->stream);
  else
    batched_gemm<float>(batch, nterms, m, n, k, opA, opB, alpha, (const float*)A, lda, strideA, (const float*)B, ldb,
                        strideB, beta, (float*)C, ldc, strideC, h->stream);
  return H2DEV_OK;
  H2_API_END
}

int h2dev_profile_timeline(h2dev_handle_t h, int64_t cap, char* names, double* start_ms, double* dur_ms,
                           int64_t* count) {
  H2_API_BEGIN
  require(h && count, "null argument");
  ck(cudaStreamSynchronize(h->stream), "sync");
  *count = (int64_t)h->recs.size();
  for (size_t k = 0; k < h->recs.size() && (int64_t)k < cap; k++) {
    const ProfRec& r = h->recs[k];
    float a = 0.f, d = 0.f;
    ck(cudaEventElapsedTime(&a, h->recs[0].a, r.a), "cudaEventElapsedTime");
    ck(cudaEventElapsedTime(&d, r.a, r.b), "cudaEventElapsedTime");
    if (names) {
      std::strncpy(names + 48 * k, r.name, 47);
      names[48 * k + 47] = 0;
    }
    if (start_ms) start_ms[k] = a;
    if (dur_ms) dur_ms[k] = d;
  }
  return H2DEV_OK;
  H2_API_END
}

int h2dev_autotune_report(h2dev_handle_t h, int64_t cap, char* keys, int* choice, double* ms, int64_t* count) {
  H2_API_BEGIN
  require(h && count, "null argument");
  *count = (int64_t)h->tune_order.size();
  for (int64_t i = 0; i < cap && i < *count; i++) {
    const auto& key = h->tune_order[(size_t)i];
    const auto& rec = h->tune.at(key);
    if (keys) {
      std::memset(keys + 64 * i, 0, 64);
      std::strncpy(keys + 64 * i, key.c_str(), 63);
    }
    if (choice) choice[i] = rec.choice;
    if (ms)
      for (int v = 0; v < 3; v++) ms[3 * i + v] = v < (int)rec.ms.size() ? rec.ms[(size_t)v] : -1.;
  }
  return H2DEV_OK;
  H2_API_END
}

int h2dev_launch_count(int64_t* count) {
  H2_API_BEGIN
  require(count != nullptr, "null argument");
  *count = (int64_t)launch_count();
  return H2DEV_OK;
  H2_API_END
}

int h2dev_probe_fma_peak(h2dev_handle_t h, int precision, double* tflops) {
  H2_API_BEGIN
  require(h && tflops && (precision == H2DEV_FP64 || precision == H2DEV_FP32), "bad arguments");
  int sms = 0;
  ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device), "attr");
  const int blocks = sms * 8, iters = precision == H2DEV_FP64 ? 4096 : 16384;
  DVec<double> out;
  out.alloc((size_t)blocks * 256);
  cudaEvent_t a, b;
  ck(cudaEventCreate(&a), "event");
  ck(cudaEventCreate(&b), "event");
  double best = 0.;
  for (int rep = 0; rep < 4; rep++) {
    ck(cudaEventRecord(a, h->stream), "record");
    ck(launch_fma_probe(precision, blocks, iters, out.p, h->stream), "fma probe");
    ck(cudaEventRecord(b, h->stream), "record");
    ck(cudaEventSynchronize(b), "sync");
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, a, b), "elapsed");
    double fl = 2. * 8. * iters * (double)blocks * 256;
    if (rep > 0) best = std::max(best, fl / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *tflops = best;
  return H2DEV_OK;
  H2_API_END
}

int h2dev_set_option(h2dev_handle_t h, int option, int64_t value) {
  H2_API_BEGIN
  require(h != nullptr, "null handle");
  if (option == H2DEV_OPT_SKINNY_TILED) {
    require(value == 0 || value == 1, "skinny option must be 0 or 1");
    g_force_tiled = value != 0;
    return H2DEV_OK;
  }
  if (option == H2DEV_OPT_TENSOR_CORES) {
    require(value >= 0 && value <= 2, "tensor-core option must be 0, 1 or 2");
    g_tensor_cores = (int)value;
    return H2DEV_OK;
  }
  if (option == H2DEV_OPT_SAMPLING) {
    require(value >= 0 && value <= 2, "sampling option must be 0, 1 or 2");
    h->sampling_mode = (int)value;
    return H2DEV_OK;
  }
  if (option == H2DEV_OPT_AUTOTUNE) {
    require(value == 0 || value == 1, "autotune option must be 0 or 1");
    h->autotune = value != 0;
    return H2DEV_OK;
  }
  if (option == H2DEV_OPT_GRAPH_SOLVE) {
    require(value == 0 || value == 1, "graph option must be 0 or 1");
    h->graph_solve = value != 0;
    return H2DEV_OK;
  }
  if (option == H2DEV_OPT_PRECOND_BF16) {
    require(value == 0 || value == 1, "BF16 substitution option must be 0 or 1");
    h->precond_bf16 = value != 0;
    return H2DEV_OK;
  }
  if (option == H2DEV_OPT_MATRIX_FREE) {
    require(value == 0 || value == 1, "matrix-free option must be 0 or 1");
    h->matrix_free = value != 0;
    return H2DEV_OK;
  }
  if (option == H2DEV_OPT_BASIS) {
    require(value == 0 || value == 1, "basis option must be 0 or 1");
    h->basis_mode = (int)value;
    return H2DEV_OK;
  }
  require(false, "unknown option");
  return H2DEV_ERR_ARG;
  H2_API_END
}

int h2dev_timer_start(h2dev_handle_t h) {
  H2_API_BEGIN
  require(h != nullptr, "null handle");
  if (!h->t0) ck(cudaEventCreate(&h->t0), "event");
  if (!h->t1) ck(cudaEventCreate(&h->t1), "event");
  ck(cudaEventRecord(h->t0, h->stream), "record");
  return H2DEV_OK;
  H2_API_END
}

int h2dev_timer_stop(h2dev_handle_t h, double* ms) {
  H2_API_BEGIN
  require(h && ms && h->t0 && h->t1, "timer not started");
  ck(cudaEventRecord(h->t1, h->stream), "record");
  ck(cudaEventSynchronize(h->t1), "sync");
  float e = 0.f;
  ck(cudaEventElapsedTime(&e, h->t0, h->t1), "elapsed");
  *ms = e;
  return H2DEV_OK;
  H2_API_END
}

int h2dev_solve_rel_err_device(h2dev_handle_t h, int64_t n, int64_t nrhs, const double* dX, const double* dRef,
                                int64_t ld, double* err) {
  H2_API_BEGIN
  require(h && dX && dRef && err && n > 0 && nrhs > 0 && ld >= n, "bad arguments");
  CurHandle ch(h);
  DVec<double> partial, out;
  partial.alloc((size_t)(2 * relerr_chunks(n) * nrhs));
  out.alloc(nrhs);
  {
    Prof pf("rel_err", 3. * n * nrhs, 16. * n * nrhs);
    ck(launch_relerr(dX, dRef, n, ld, (int)nrhs, partial.p, out.p, h->stream), "rel_err");
  }
  ck(cudaStreamSynchronize(h->stream), "sync");
  ck(cudaMemcpy(err, out.p, sizeof(double) * nrhs, cudaMemcpyDeviceToHost), "D2H");
  return H2DEV_OK;
  H2_API_END
}

int h2dev_solver_export_size(h2dev_solver_t s, int64_t level, int what, int64_t* count) {
  H2_API_BEGIN
  require(s && s->impl && count, "null argument");
  *count = s->impl->export_size(level, what);
  return H2DEV_OK;
  H2_API_END
}

int h2dev_solver_export(h2dev_solver_t s, int64_t level, int what, double* out) {
  H2_API_BEGIN
  require(s && s->impl && out, "null argument");
  s->impl->export_to(level, what, out);
  return H2DEV_OK;
  H2_API_END
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free solveRelErr.  Same two reduction kernels as
// h2dev_solve_rel_err_device; only the partial-sum scratch and the output
// differ: the scratch is a file-scope device array, the output is the
// caller's device array.

#include <cstdio>
#include <mutex>

namespace h2b {

// Partial-sum scratch of h2dev_solve_rel_err_device_noalloc: 16384 doubles
// (128 KiB).  Every GPU that loads this library keeps it until the process
// exits.
constexpr i64 NOALLOC_SCRATCH_DOUBLES = 16384;
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

constexpr int NOALLOC_MAX_DEVICES = 64;
static double* g_noalloc_ptr[NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mu;

// Device address of the scratch on ``dev``.  In host code the array's name
// only stands in for the symbol; the address is looked up once per device,
// with that device current, and cached for the life of the process (a
// cudaDeviceReset unloads the module and leaves the cached address stale, so
// the entry point must not be used after one).
static cudaError_t noalloc_scratch(int dev, double** out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return e;
    if (prev != dev && (e = cudaSetDevice(dev)) != cudaSuccess) return e;
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (prev != dev) cudaSetDevice(prev);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

}  // namespace h2b

extern "C" int h2dev_solve_rel_err_device_noalloc(h2dev_handle_t h, int64_t n, int64_t nrhs, const double* dX,
                                                  const double* dRef, int64_t ld, double* dErr) {
  H2_API_BEGIN
  require(h && dX && dRef && dErr && n > 0 && nrhs > 0 && ld >= n, "bad arguments");
  CurHandle ch(h);  // the handle's device current for the launch; allocates nothing
  // In 64-bit arithmetic, and bounded first, so no product can wrap.
  const int64_t chunks = relerr_chunks(n);
  const int64_t need = (chunks > NOALLOC_SCRATCH_DOUBLES || nrhs > NOALLOC_SCRATCH_DOUBLES)
                           ? NOALLOC_SCRATCH_DOUBLES + 1
                           : 2 * chunks * nrhs;
  if (need > NOALLOC_SCRATCH_DOUBLES) {
    char msg[200];
    snprintf(msg, sizeof(msg),
             "h2dev_solve_rel_err_device_noalloc: n=%lld, nrhs=%lld needs %lld scratch doubles; the fixed limit is "
             "%lld (2 * ceil(n / 16384) * nrhs)",
             (long long)n, (long long)nrhs, (long long)need, (long long)NOALLOC_SCRATCH_DOUBLES);
    throw H2Error{H2DEV_ERR_ARG, msg};
  }
  double* scratch = nullptr;
  ck(noalloc_scratch(h->device, &scratch), "cudaGetSymbolAddress(scratch)");
  // Every scratch slot the second pass reads is written by the first pass of
  // this same call, so nothing has to be cleared between calls.
  ck(launch_relerr(dX, dRef, n, ld, (int)nrhs, scratch, dErr, h->stream), "rel_err (no-alloc)");
  return H2DEV_OK;
  H2_API_END
}
