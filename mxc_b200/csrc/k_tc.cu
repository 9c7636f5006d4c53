// Segmented FP32 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// C_task = beta C_task + sum_e alpha_e op(A_e) op(B_e), the same task /
// entry lists as the SIMT segmented GEMM, for the FP32 contractions of the
// ULV factorization.  FP32 accuracy on TF32 tensor cores by the 3-term split
// x = hi + lo: A B ~= A_hi B_hi + A_hi B_lo + A_lo B_hi, every product
// accumulated in FP32 in tensor memory (the dropped A_lo B_lo term and the
// TF32 truncation of lo are below 2^-20 relative).
//
// 128 x 128 output tiles, 16-wide k slabs; one persistent warp-specialised
// CTA per SM (see k_tc_gemm_ws below for the roles and the stage ring).
#include "common.cuh"
#include "kernels.h"

#include <cstdint>

namespace h2b {

namespace {

constexpr int TC_BM = 128, TC_BN = 128, TC_KT = 16;
// Row-contiguous B conversion: 256 threads, 2 chunks of 16 bytes per thread.
constexpr int TC_NT = 256;
constexpr int TC_CPT = TC_BM * TC_KT / 4 / TC_NT;
constexpr int TC_KC = TC_KT / 4;            // 16-byte k-chunks per row
constexpr int TC_TILE = TC_BM * TC_KT * 4;  // bytes of one 128 x 16 FP32 operand tile
constexpr long long TC_WAIT_CYCLES = 4000000000LL;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Canonical no-swizzle K-major layout (byte offsets inside a 128 x 16
// tile): core matrix = 8 rows x 16 bytes (4 k); k-chunks 128 B apart
// (leading byte offset), 8-row groups 512 B apart (stride byte offset).
constexpr int TC_SBO = TC_KC * 128;
__device__ __forceinline__ int off_kmajor(int r, int kc) { return (r >> 3) * TC_SBO + kc * 128 + (r & 7) * 16; }
// Raw layouts.  k contiguous: row r is 64 bytes (4 chunks of 4 k), chunk
// kc stored at slot kc ^ ((r >> 1) & 3).  Rows contiguous: k-row k is 512
// bytes (32 chunks of 4 rows), chunk q stored at slot q ^ (2 ((k >> 2) & 3)).
__device__ __forceinline__ int raw_kc(int r, int kc) { return r * 64 + ((kc ^ ((r >> 1) & 3)) << 4); }
__device__ __forceinline__ int raw_rc(int q, int k) { return k * 512 + ((q ^ (((k >> 2) & 3) << 1)) << 4); }

__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, swizzle none
}

// Instruction descriptor: D FP32, A and B TF32 (both K-major), M = 128, N = n.
__device__ __forceinline__ uint32_t make_idesc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// mbarrier.try_wait suspends the thread in hardware until the phase
// completes or a system-dependent time limit passes.
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the given phase parity of an mbarrier.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (clock64() - t0 > TC_WAIT_CYCLES) return false;
  }
  return true;
}

__device__ __forceinline__ void cp16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp4(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// x rounded to the nearest TF32 value (10 explicit mantissa bits; ties away
// from zero): add half a TF32 ulp to the magnitude bits, clear the 13 low
// bits.  Integer ALU work only; inputs are finite and far below FLT_MAX.
__device__ __forceinline__ float tf32_hi(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

__device__ __forceinline__ float pick(const float4& v, int j) {
  return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}

__device__ __forceinline__ void store_split(unsigned char* hi, unsigned char* lo, int off, float4 x, float scale) {
  x.x *= scale; x.y *= scale; x.z *= scale; x.w *= scale;
  float4 h, l;
  h.x = tf32_hi(x.x); l.x = x.x - h.x;
  h.y = tf32_hi(x.y); l.y = x.y - h.y;
  h.z = tf32_hi(x.z); l.z = x.z - h.z;
  h.w = tf32_hi(x.w); l.w = x.w - h.w;
  *reinterpret_cast<float4*>(hi + off) = h;
  *reinterpret_cast<float4*>(lo + off) = l;
}

// Converts a raw operand tile into hi / lo K-major tiles.  Each 8-lane
// phase of the 16-byte shared loads and stores touches 8 distinct bank
// groups.  k contiguous: chunk c = tid + 256 i is row 8 (c >> 5) + (c & 7),
// k-chunk (c >> 3) & 3.  Rows contiguous: lane = 8p + 2a + b of warp w
// reads rows 4q..4q+3 (q = 8 (w & 3) + 2p + b) at the four k of k-chunk a
// and stores two rows of the transposed 4 x 4 block (steps t = 2 (w >> 2)
// and t + 1, row (t + a) & 3 in step t; warps w and w + 4 share a block).
__device__ __forceinline__ void convert_operand(const unsigned char* raw, int kcontig, float scale,
                                                unsigned char* hi, unsigned char* lo, int tid) {
  if (kcontig) {
#pragma unroll
    for (int i = 0; i < TC_CPT; i++) {
      const int c = tid + TC_NT * i;
      const int r = ((c >> 5) << 3) | (c & 7), kc = (c >> 3) & 3;
      const float4 x = *reinterpret_cast<const float4*>(raw + raw_kc(r, kc));
      store_split(hi, lo, off_kmajor(r, kc), x, scale);
    }
  } else {
    const int lane = tid & 31, warp = tid >> 5;
    const int p = lane >> 3, a = (lane >> 1) & 3, b = lane & 1;
    {
      const int q = (warp & 3) * 8 + 2 * p + b;
      const int kc = a;
      float4 v[4];
#pragma unroll
      for (int t = 0; t < 4; t++) v[t] = *reinterpret_cast<const float4*>(raw + raw_rc(q, 4 * kc + t));
      const int t0 = 2 * (warp >> 2);
#pragma unroll
      for (int tt = 0; tt < 2; tt++) {
        const int t = t0 + tt;
        const int j = (t + a) & 3;
        store_split(hi, lo, off_kmajor(4 * q + j, kc), make_float4(pick(v[0], j), pick(v[1], j), pick(v[2], j),
                                                                  pick(v[3], j)), scale);
      }
    }
  }
}

}  // namespace

// Set when an mbarrier wait expired (read and cleared by the host).

// Warp-specialised variant, one CTA per SM (25 warps, 512 TMEM columns),
// A operand in tensor memory, double-buffered accumulator.
//
// The tensor core reads a TF32 operand from a 32-bit container by ignoring
// its 13 low mantissa bits, so the split needs no rounding pass: hi = x as
// stored (truncated by the hardware), lo = x - trunc(x) (exact in FP32).
// Per slab the work is therefore: copy A raw and B (k-contiguous B straight
// into its K-major hi tile), then the converters write A_hi / A_lo from
// registers into TMEM (tcgen05.st; lane = tile row, column = k) and compute
// B_lo from B_hi in place.  Row-contiguous B is copied raw and converted
// (transposed, rounded split) as in the kernel above.  The MMAs read A from
// TMEM and only B from shared memory.
//
// Stage ring (WS_ST stages of 32 KB: A raw, B raw, B hi, B lo; TMEM A
// buffer of 32 columns per stage at 256 + 32 s):
//  warps 0-7   producers: wait stage_free (the MMAs of the stage's previous
//              slab done), cp.async the slab, cp.async.mbarrier.arrive on
//              full.
//  warps 8-15  converters: wait full; warp w writes A rows 32 (w & 3) ..
//              +31, k 8 h .. +7 (h = (w - 8) >> 2) to TMEM and its share of
//              B lo; signal conv_full.
//  warps 16-23 epilogue: wait acc_full, read TMEM lane quarter w & 3,
//              columns 64 ((w - 16) >> 2) .. +63, release the accumulator
//              (acc_empty), write C.
//  warp 24     one thread: wait conv_full (and, before a tile's first slab,
//              acc_empty of its accumulator), issue the slab's MMAs, commit
//              to stage_free and, after a tile's last slab, to acc_full.
// Every wait is bounded; an expired wait sets a CTA-wide abort flag that
// ends every role's loop.  Waits are taken by one lane and broadcast, so
// warp-collective instructions stay convergent; no named barrier is used
// inside the loops.
namespace {
constexpr int WS_NT = 800;
constexpr int WS_NP = 256;             // producer threads (warps 0-7)
constexpr int WS_PCH = 512 / WS_NP;    // 16-byte chunks per operand tile per producer thread
constexpr int WS_ST = 6;
constexpr int WS_STAGE = 4 * TC_TILE;  // A raw, B raw, B hi, B lo
constexpr int WS_SMEM = WS_ST * WS_STAGE;
constexpr int WS_TMEM_COLS = 512;
constexpr int WS_ACOL = 2 * TC_BN;  // first A buffer column
constexpr uint32_t TF32_MASK = 0xFFFFE000u;

// try_wait with a suspend-time hint (ns): a waiting thread sleeps in
// hardware until the phase completes instead of spinning on issue slots.
__device__ __forceinline__ bool mbar_try_sleep(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(1000000u)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool ws_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_sleep(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_sleep(bar, parity)) {
    if (*abort_flag) return false;
    if (clock64() - t0 > TC_WAIT_CYCLES) {
      *abort_flag = 1;
      return false;
    }
  }
  return true;
}

// Lane 0 waits, the warp learns the outcome (warp-uniform).
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int lane) {
  int ok = 1;
  if (lane == 0) ok = ws_wait(bar, parity, abort_flag) ? 1 : 0;
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mma_tf32_ta(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&v)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr), "r"(v[0]),
               "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}

struct WsTile {
  int m0, n0, mrows, ncols, e0, e1;
  GemmTask<float> task;
};

__device__ __forceinline__ WsTile ws_tile(const GemmTask<float>* tasks, const GemmEntry<float>* ents,
                                          const TileRef* tiles, int tile) {
  WsTile w;
  const TileRef tl = tiles[tile];
  w.task = tasks[tl.task];
  w.m0 = tl.tm * TC_BM;
  w.n0 = tl.tn * TC_BN;
  w.mrows = min(TC_BM, w.task.m - w.m0);
  w.ncols = min(TC_BN, w.task.n - w.n0);
  w.e0 = w.task.e0;
  w.e1 = w.task.e1;
  while (w.e0 < w.e1 && ents[w.e0].k <= 0) w.e0++;
  return w;
}

// A producer thread's 16-byte chunks of one operand tile (the chunks
// c = ptid + WS_NP j of the tile's 512), resolved once per entry: per slab
// only the k offset changes.  k contiguous: chunk c is row c >> 2, k-chunk
// c & 3, stored in the raw layout or, with kmajor, directly in the
// canonical K-major layout; rows contiguous: chunk c is row quad c & 31 of
// k-row c >> 5 (raw layout).
struct ProdChunks {
  const float* X;
  const float* src[WS_PCH];  // element (row, k = k0 + kofs) at src + k0 * kstep
  uint32_t dst[WS_PCH];
  i64 kstep;
  int kofs[WS_PCH];
  int nrow[WS_PCH];  // k contiguous: 4 if the row is in the tile else 0; rows contiguous: valid rows of the quad
  int kcontig, vec, K;
};

__device__ __forceinline__ void prod_prepare(ProdChunks& pc, const float* X, i64 ld, int rows, int r0, int K,
                                             int kcontig, int kmajor, uint32_t base, int ptid) {
  pc.X = X;
  pc.K = K;
  pc.kcontig = kcontig;
  pc.vec = ((reinterpret_cast<uintptr_t>(X) & 15) == 0) && (ld % 4 == 0);
#pragma unroll
  for (int j = 0; j < WS_PCH; j++) {
    const int c = ptid + WS_NP * j;
    if (kcontig) {
      const int r = c >> 2, kc = c & 3;
      pc.kofs[j] = 4 * kc;
      pc.nrow[j] = r < rows ? 4 : 0;
      pc.src[j] = X + (i64)(r0 + r) * ld + 4 * kc;
      pc.dst[j] = base + (kmajor ? off_kmajor(r, kc) : raw_kc(r, kc));
    } else {
      const int q = c & 31, k = c >> 5;
      int nr = rows - 4 * q;
      pc.kofs[j] = k;
      pc.nrow[j] = nr < 0 ? 0 : (nr > 4 ? 4 : nr);
      pc.src[j] = X + (i64)(r0 + 4 * q) + (i64)k * ld;
      pc.dst[j] = base + raw_rc(q, k);
    }
  }
  pc.kstep = kcontig ? 1 : ld;
}

// Issues the thread's chunks of the slab at k0 into stage offset `stage_off`.
__device__ __forceinline__ void prod_issue(const ProdChunks& pc, int k0, uint32_t stage_off) {
#pragma unroll
  for (int j = 0; j < WS_PCH; j++) {
    const int k = k0 + pc.kofs[j];
    int n;
    if (pc.kcontig) {
      n = pc.K - k;
      n = n < 0 ? 0 : (n > 4 ? 4 : n);
      if (!pc.nrow[j]) n = 0;
    } else {
      n = k < pc.K ? pc.nrow[j] : 0;
    }
    const float* p = pc.src[j] + (i64)k0 * pc.kstep;
    const uint32_t d = pc.dst[j] + stage_off;
    if (pc.vec) {
      cp16(d, n ? (const void*)p : (const void*)pc.X, n * 4);
    } else {  // the four elements of a chunk are adjacent in memory in both layouts
#pragma unroll
      for (int t = 0; t < 4; t++) cp4(d + 4 * t, t < n ? (const void*)(p + t) : (const void*)pc.X, t < n ? 4 : 0);
    }
  }
}
}  // namespace

__global__ void __launch_bounds__(WS_NT, 1)
    k_tc_gemm_ws(const GemmTask<float>* __restrict__ tasks, const GemmEntry<float>* __restrict__ ents,
                 const TileRef* __restrict__ tiles, int ntiles, int split, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[WS_ST], conv_full[WS_ST], stage_free[WS_ST], acc_full[2], acc_empty[2], drain;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int s = 0; s < WS_ST; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&full[s])), "r"(WS_NP) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 8;" ::"r"(smem_addr(&conv_full[s])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&stage_free[s])) : "memory");
    }
    for (int s = 0; s < 2; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&acc_full[s])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 8;" ::"r"(smem_addr(&acc_empty[s])) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&drain)) : "memory");
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(WS_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  if (warp < 8) {
    // ---------------------------------------------------------- producers
    int g = 0;
    bool ok = true;
    const uint32_t st0 = smem_addr(smem);
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
      const WsTile w = ws_tile(tasks, ents, tiles, tile);
      for (int e = w.e0; e < w.e1 && ok; e++) {
        const GemmEntry<float> en = ents[e];
        if (en.k <= 0) continue;
        const int b_kc = en.opB ? 0 : 1;
        ProdChunks pa, pb;
        prod_prepare(pa, en.A, en.lda, w.mrows, w.m0, en.k, en.opA, 0, st0, tid);
        prod_prepare(pb, en.B, en.ldb, w.ncols, w.n0, en.k, b_kc, b_kc, st0 + (b_kc ? 2 : 1) * TC_TILE, tid);
        for (int k0 = 0; k0 < en.k; k0 += TC_KT) {
          const int s = g % WS_ST;
          if (g >= WS_ST && !ws_wait(smem_addr(&stage_free[s]), (uint32_t)(((g / WS_ST) - 1) & 1), &abort_flag)) {
            ok = false;
            break;
          }
          prod_issue(pa, k0, (uint32_t)(s * WS_STAGE));
          prod_issue(pb, k0, (uint32_t)(s * WS_STAGE));
          asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(&full[s])) : "memory");
          g++;
        }
      }
    }
    cp_wait<0>();
  } else if (warp < 16) {
    // --------------------------------------------------------- converters
    const int ctid = tid - WS_NP;
    const int q = warp & 3, kh = (warp - 8) >> 2;
    const int r = q * 32 + lane;  // A row (TMEM lane) of this thread
    const uint32_t tmem_row = tmem + ((uint32_t)(q * 32) << 16);
    int g = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
      const WsTile w = ws_tile(tasks, ents, tiles, tile);
      for (int e = w.e0; e < w.e1 && ok; e++) {
        const GemmEntry<float> en = ents[e];
        if (en.k <= 0) continue;
        const int b_kc = en.opB ? 0 : 1;
        const bool unit = en.alpha == 1.f;
        for (int k0 = 0; k0 < en.k; k0 += TC_KT) {
          const int s = g % WS_ST;
          if (!warp_wait(smem_addr(&full[s]), (uint32_t)((g / WS_ST) & 1), &abort_flag, lane)) {
            ok = false;
            break;
          }
          unsigned char* st = smem + s * WS_STAGE;
          // A row r, k 8 kh .. 8 kh + 7 -> TMEM (hi = x, lo = x - trunc(x)).
          float v[8];
          if (en.opA) {
#pragma unroll
            for (int c = 0; c < 2; c++) {
              const float4 x = *reinterpret_cast<const float4*>(st + raw_kc(r, 2 * kh + c));
              v[4 * c] = x.x; v[4 * c + 1] = x.y; v[4 * c + 2] = x.z; v[4 * c + 3] = x.w;
            }
          } else {
#pragma unroll
            for (int k = 0; k < 8; k++) v[k] = *reinterpret_cast<const float*>(st + raw_rc(r >> 2, 8 * kh + k) + (r & 3) * 4);
          }
          uint32_t hi[8], lo[8];
#pragma unroll
          for (int k = 0; k < 8; k++) {
            const float x = unit ? v[k] : v[k] * en.alpha;
            hi[k] = __float_as_uint(x);
            lo[k] = __float_as_uint(x - __uint_as_float(hi[k] & TF32_MASK));
          }
          const uint32_t acol = (uint32_t)(WS_ACOL + s * 32 + 8 * kh);
          tmem_st8(tmem_row + acol, hi);
          tmem_st8(tmem_row + acol + 16, lo);
          // B lo (k-contiguous B: from the hi tile the copies filled).
          unsigned char* bhi = st + 2 * TC_TILE;
          unsigned char* blo = st + 3 * TC_TILE;
          if (b_kc) {
#pragma unroll
            for (int i = 0; i < 2; i++) {
              const int off = (ctid + 256 * i) * 16;
              const float4 x = *reinterpret_cast<const float4*>(bhi + off);
              float4 l;
              l.x = x.x - __uint_as_float(__float_as_uint(x.x) & TF32_MASK);
              l.y = x.y - __uint_as_float(__float_as_uint(x.y) & TF32_MASK);
              l.z = x.z - __uint_as_float(__float_as_uint(x.z) & TF32_MASK);
              l.w = x.w - __uint_as_float(__float_as_uint(x.w) & TF32_MASK);
              *reinterpret_cast<float4*>(blo + off) = l;
            }
          } else {
            convert_operand(st + TC_TILE, 0, 1.f, bhi, blo, ctid);
          }
          asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_addr(&conv_full[s]));
          g++;
        }
      }
    }
  } else if (warp < 24) {
    // ---------------------------------------------------------- epilogue
    const int q = warp & 3, ch = (warp - 16) >> 2;
    const int row = q * 32 + lane;
    int t = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      const WsTile w = ws_tile(tasks, ents, tiles, tile);
      const bool any = w.e0 < w.e1;
      const int ab = t & 1;
      const int cbeg = ch * 64;
      if (any && !warp_wait(smem_addr(&acc_full[ab]), (uint32_t)((t >> 1) & 1), &abort_flag, lane)) break;
      if (cbeg >= w.ncols) {
        // No columns for this warp; still hand the accumulator back.
        if (any) {
          if (lane == 0) mbar_arrive(smem_addr(&acc_empty[ab]));
          t++;
        }
        continue;
      }
      if (any) asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int cend = min(w.ncols, cbeg + 64);
      const float beta = w.task.beta;
      const bool rowok = row < w.mrows;
      for (int c0 = cbeg; c0 < cend; c0 += 32) {
        float acc[32];
        if (any) {
          uint32_t rr[32];
          const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * TC_BN + c0);
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
              "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
              : "=r"(rr[0]), "=r"(rr[1]), "=r"(rr[2]), "=r"(rr[3]), "=r"(rr[4]), "=r"(rr[5]), "=r"(rr[6]),
                "=r"(rr[7]), "=r"(rr[8]), "=r"(rr[9]), "=r"(rr[10]), "=r"(rr[11]), "=r"(rr[12]), "=r"(rr[13]),
                "=r"(rr[14]), "=r"(rr[15]), "=r"(rr[16]), "=r"(rr[17]), "=r"(rr[18]), "=r"(rr[19]), "=r"(rr[20]),
                "=r"(rr[21]), "=r"(rr[22]), "=r"(rr[23]), "=r"(rr[24]), "=r"(rr[25]), "=r"(rr[26]), "=r"(rr[27]),
                "=r"(rr[28]), "=r"(rr[29]), "=r"(rr[30]), "=r"(rr[31])
              : "r"(taddr));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int j = 0; j < 32; j++) acc[j] = __uint_as_float(rr[j]);
          if (c0 + 32 >= cend) {
            // Last read of this warp: hand the accumulator back.
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_addr(&acc_empty[ab]));
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; j++) acc[j] = 0.f;
        }
        if (rowok) {
          float* cp = w.task.C + (i64)(w.m0 + row) + (i64)(w.n0 + c0) * w.task.ldc;
          const i64 ldc = w.task.ldc;
          if (c0 + 32 <= w.ncols && beta == 0.f) {
#pragma unroll
            for (int j = 0; j < 32; j++) cp[(i64)j * ldc] = acc[j];
          } else {
#pragma unroll
            for (int j = 0; j < 32; j++) {
              if (c0 + j < w.ncols) {
                float* p = cp + (i64)j * ldc;
                *p = (beta == 0.f) ? acc[j] : beta * (*p) + acc[j];
              }
            }
          }
        }
      }
      if (any) t++;
    }
  } else if (lane == 0) {
    // ------------------------------------------------------- MMA issuer
    int g = 0, t = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
      const WsTile w = ws_tile(tasks, ents, tiles, tile);
      if (w.e0 >= w.e1) continue;
      const int ab = t & 1;
      const uint32_t idesc = make_idesc(((w.ncols + 15) / 16) * 16);
      const uint32_t dacc = tmem + (uint32_t)(ab * TC_BN);
      if (t >= 2 && !ws_wait(smem_addr(&acc_empty[ab]), (uint32_t)(((t >> 1) - 1) & 1), &abort_flag)) break;
      bool first = true;
      for (int e = w.e0; e < w.e1 && ok; e++) {
        const int K = ents[e].k;
        if (K <= 0) continue;
        int enext = e + 1;
        while (enext < w.e1 && ents[enext].k <= 0) enext++;
        for (int k0 = 0; k0 < K; k0 += TC_KT) {
          const int s = g % WS_ST;
          if (!ws_wait(smem_addr(&conv_full[s]), (uint32_t)((g / WS_ST) & 1), &abort_flag)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t base = smem_addr(smem + s * WS_STAGE + 2 * TC_TILE);
          const uint32_t acol = (uint32_t)(WS_ACOL + s * 32);
#pragma unroll
          for (int ks = 0; ks < TC_KT / 8; ks++) {
            const uint64_t bh = make_desc(base + ks * 256, 128, TC_SBO);
            const uint64_t bl = make_desc(base + TC_TILE + ks * 256, 128, TC_SBO);
            const uint32_t ah = tmem + acol + ks * 8, al = tmem + acol + 16 + ks * 8;
            const uint32_t accf = (first && ks == 0) ? 0u : 1u;
            if (split) {
              mma_tf32_ta(dacc, al, bh, idesc, accf);
              mma_tf32_ta(dacc, ah, bl, idesc, 1u);
              mma_tf32_ta(dacc, ah, bh, idesc, 1u);
            } else {
              mma_tf32_ta(dacc, ah, bh, idesc, accf);
            }
          }
          mma_commit(smem_addr(&stage_free[s]));
          if (enext >= w.e1 && k0 + TC_KT >= K) mma_commit(smem_addr(&acc_full[ab]));
          first = false;
          g++;
        }
      }
      t++;
    }
    // Every MMA this thread issued has completed before TMEM is freed.
    mma_commit(smem_addr(&drain));
    mbar_wait(smem_addr(&drain), 0);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid == 0 && abort_flag && err) atomicExch(err, 1);
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(WS_TMEM_COLS) : "memory");
}

int tc_gemm_tile() { return TC_BM; }

cudaError_t launch_tc_gemm(const GemmTask<float>* d_tasks, const GemmEntry<float>* d_ents, const TileRef* d_tiles,
                           int ntiles, int split, int* err, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k_tc_gemm_ws, cudaFuncAttributeMaxDynamicSharedMemorySize, WS_SMEM);
  if (e != cudaSuccess) return e;
  // Persistent: one CTA per SM walks the tile list with a stride of the grid.
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  const int grid = ntiles < sms ? ntiles : sms;
  note_launch();
  k_tc_gemm_ws<<<grid, WS_NT, WS_SMEM, st>>>(d_tasks, d_ents, d_tiles, ntiles, split, err);
  return cudaGetLastError();
}

}  // namespace h2b
