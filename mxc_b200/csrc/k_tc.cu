// Segmented FP32 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// C_task = beta C_task + sum_e alpha_e op(A_e) op(B_e), the same task /
// entry lists as the SIMT segmented GEMM, for the FP32 contractions of the
// ULV factorization.  FP32 accuracy on TF32 tensor cores by the 3-term split
// x = hi + lo (hi = x rounded to TF32, lo = x - hi exactly in FP32):
// A B ~= A_hi B_hi + A_hi B_lo + A_lo B_hi, every product accumulated in FP32
// in tensor memory (the dropped A_lo B_lo term and the TF32 truncation of lo
// are below 2^-21 relative).
//
// One CTA (256 threads, two per SM) owns a 128 x 128 output tile; its
// accumulator is 128 TMEM lanes x 128 columns.  The task's (entry, 16-wide
// k slab) sequence flows through three stages:
//  1. raw ring (3 slots): every thread issues cp.async copies of the slab's
//     A and B tiles in their global orientation (16-byte chunks, XOR-swizzled
//     so the reads of stage 2 are bank-conflict-free; rows past m / n and k
//     past K are zero-filled), two slabs ahead of the one being converted;
//  2. conversion: the slab is read back, scaled by alpha (A), split into hi
//     and lo and stored in the canonical no-swizzle K-major UMMA layout (row-
//     contiguous operands are transposed 4 x 4 in registers), into one of two
//     operand buffers;
//  3. one thread issues the slab's 6 MMAs (2 k-steps x 3 products) and
//     commits them to the buffer's mbarrier; the buffer is converted into
//     again once that barrier completes.
// Every mbarrier wait is bounded (about two seconds of clock cycles); on
// expiry the kernel records an error flag for the host and leaves.
#include "common.cuh"
#include "kernels.h"

#include <cstdint>

namespace h2b {

namespace {

constexpr int TC_BM = 128, TC_BN = 128, TC_KT = 16, TC_NT = 256;
constexpr int TC_CPT = TC_BM * TC_KT / 4 / TC_NT;  // 16-byte chunks per thread per operand
constexpr int TC_KC = TC_KT / 4;            // 16-byte k-chunks per row
constexpr int TC_TILE = TC_BM * TC_KT * 4;  // bytes of one 128 x 16 FP32 operand tile
constexpr int TC_RAW = 2 * TC_TILE;         // raw slot: A, B
constexpr int TC_HL = 4 * TC_TILE;          // operand buffer: A hi, A lo, B hi, B lo
constexpr int TC_RS = 3, TC_HS = 2;
constexpr int TC_SMEM = TC_RS * TC_RAW + TC_HS * TC_HL;
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

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
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
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t u;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(x));
  return __uint_as_float(u & 0xFFFFE000u);
}

// One operand of a slab: 128 rows (of op(X), rows of the output tile) by
// 16 k.  kcontig: element (r, k) at X[k + r * ld]; otherwise at X[r + k * ld].
struct OperandRef {
  const float* X;
  i64 ld;
  int rows;  // valid rows in the tile (from the tile origin)
  int r0;    // tile origin in rows
  int k0, K;
  int kcontig;
  int vec;  // 16-byte copies are aligned
};

// Issues this thread's copies (2 chunks of 16 bytes) of a raw operand tile.
// k contiguous: chunk c = tid + 256 i is row c >> 2, k-chunk c & 3 (a warp
// reads 8 rows x 64 contiguous bytes).  Rows contiguous: chunk c is row
// quad c & 31 of k-row c >> 5 (a warp reads 512 contiguous bytes).
__device__ __forceinline__ void issue_operand(const OperandRef& o, uint32_t raw, int tid) {
#pragma unroll
  for (int i = 0; i < TC_CPT; i++) {
    const int c = tid + TC_NT * i;
    if (o.kcontig) {
      const int r = c >> 2, kc = c & 3;
      const int gk = o.k0 + kc * 4;
      const uint32_t dst = raw + raw_kc(r, kc);
      const bool rowok = r < o.rows;
      int nk = o.K - gk;
      nk = nk < 0 ? 0 : (nk > 4 ? 4 : nk);
      if (!rowok) nk = 0;
      const float* p = o.X + (i64)gk + (i64)(o.r0 + r) * o.ld;
      if (o.vec) {
        cp16(dst, nk ? (const void*)p : (const void*)o.X, nk * 4);
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++) cp4(dst + 4 * j, j < nk ? (const void*)(p + j) : (const void*)o.X, j < nk ? 4 : 0);
      }
    } else {
      const int q = c & 31, k = c >> 5;
      const int gk = o.k0 + k, r = 4 * q;
      const uint32_t dst = raw + raw_rc(q, k);
      int nr = o.rows - r;
      nr = nr < 0 ? 0 : (nr > 4 ? 4 : nr);
      if (gk >= o.K) nr = 0;
      const float* p = o.X + (i64)(o.r0 + r) + (i64)gk * o.ld;
      if (o.vec) {
        cp16(dst, nr ? (const void*)p : (const void*)o.X, nr * 4);
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++) cp4(dst + 4 * j, j < nr ? (const void*)(p + j) : (const void*)o.X, j < nr ? 4 : 0);
      }
    }
  }
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

struct SlabCursor {
  int e, k0;
};

__device__ __forceinline__ void skip_empty(const GemmEntry<float>* ents, int e1, SlabCursor& c) {
  while (c.e < e1 && ents[c.e].k <= 0) c.e++;
}

__device__ __forceinline__ void advance(const GemmEntry<float>* ents, int e1, SlabCursor& c) {
  c.k0 += TC_KT;
  if (c.k0 >= ents[c.e].k) {
    c.k0 = 0;
    c.e++;
    skip_empty(ents, e1, c);
  }
}

}  // namespace

// Set when an mbarrier wait expired (read and cleared by the host).
__device__ int g_tc_err = 0;

// Position in a CTA's stream of (tile, entry, k slab): the CTA owns tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...
struct TileCursor {
  int tile, e, e1, k0;
};

__device__ __forceinline__ void tile_begin(const GemmTask<float>* tasks, const GemmEntry<float>* ents,
                                           const TileRef* tiles, int ntiles, TileCursor& c) {
  while (c.tile < ntiles) {
    const GemmTask<float>& t = tasks[tiles[c.tile].task];
    c.e = t.e0;
    c.e1 = t.e1;
    c.k0 = 0;
    while (c.e < c.e1 && ents[c.e].k <= 0) c.e++;
    return;
  }
}

// Next slab; moves on to the CTA's next tile after the last one of a tile.
__device__ __forceinline__ bool slab_next(const GemmTask<float>* tasks, const GemmEntry<float>* ents,
                                          const TileRef* tiles, int ntiles, TileCursor& c) {
  c.k0 += TC_KT;
  if (c.k0 >= ents[c.e].k) {
    c.k0 = 0;
    c.e++;
    while (c.e < c.e1 && ents[c.e].k <= 0) c.e++;
  }
  return c.e < c.e1;
}

__global__ void __launch_bounds__(TC_NT, 2)
    k_tc_gemm(const GemmTask<float>* __restrict__ tasks, const GemmEntry<float>* __restrict__ ents,
              const TileRef* __restrict__ tiles, int ntiles, int split) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bars[TC_HS];
  __shared__ uint32_t tmem_slot;
  __shared__ int wait_ok;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char* raw_base = smem;
  unsigned char* hl_base = smem + TC_RS * TC_RAW;

  if (tid == 0) {
    for (int s = 0; s < TC_HS; s++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[s])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(TC_BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  // Producer: copies of the slab at its cursor into raw slot `slot`, one
  // commit group per call (empty once the CTA's tiles are exhausted).  It
  // runs two slabs ahead of the consumer, across tile boundaries.
  TileCursor prod{(int)blockIdx.x, 0, 0, 0};
  tile_begin(tasks, ents, tiles, ntiles, prod);
  auto produce = [&](int slot) {
    while (prod.tile < ntiles && prod.e >= prod.e1) {  // tiles without slabs
      prod.tile += gridDim.x;
      tile_begin(tasks, ents, tiles, ntiles, prod);
    }
    if (prod.tile < ntiles) {
      const TileRef tl = tiles[prod.tile];
      const GemmTask<float> task = tasks[tl.task];
      const int m0 = tl.tm * TC_BM, n0 = tl.tn * TC_BN;
      const GemmEntry<float> en = ents[prod.e];
      const uint32_t raw = smem_addr(raw_base + slot * TC_RAW);
      OperandRef a, b;
      a.X = en.A; a.ld = en.lda; a.rows = min(TC_BM, task.m - m0); a.r0 = m0; a.k0 = prod.k0; a.K = en.k;
      a.kcontig = en.opA;  // op(A)(m, k) = A[k + m lda] when transposed
      a.vec = ((reinterpret_cast<uintptr_t>(en.A) & 15) == 0) && (en.lda % 4 == 0);
      b.X = en.B; b.ld = en.ldb; b.rows = min(TC_BN, task.n - n0); b.r0 = n0; b.k0 = prod.k0; b.K = en.k;
      b.kcontig = en.opB ? 0 : 1;  // op(B)(k, n) = B[k + n ldb] when not transposed
      b.vec = ((reinterpret_cast<uintptr_t>(en.B) & 15) == 0) && (en.ldb % 4 == 0);
      issue_operand(a, raw, tid);
      issue_operand(b, raw + TC_TILE, tid);
      if (!slab_next(tasks, ents, tiles, ntiles, prod)) {
        prod.tile += gridDim.x;
        tile_begin(tasks, ents, tiles, ntiles, prod);
      }
    }
    cp_commit();
  };
#pragma unroll
  for (int j = 0; j < TC_RS - 1; j++) produce(j);

  bool ok = true;
  int s = 0;  // slabs consumed by this CTA (all tiles)
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const TileRef tl = tiles[tile];
    const GemmTask<float> task = tasks[tl.task];
    const int m0 = tl.tm * TC_BM, n0 = tl.tn * TC_BN;
    const int mrows = min(TC_BM, task.m - m0), ncols = min(TC_BN, task.n - n0);
    const int nmma = ((ncols + 15) / 16) * 16;  // MMA N: multiple of 16, >= 16
    TileCursor cons{tile, 0, 0, 0};
    tile_begin(tasks, ents, tiles, ntiles, cons);
    const bool any = cons.e < cons.e1;
    if (any) {
      bool more = true;
      bool first_slab = true;
      while (more) {
        const int hb = s & 1;
        cp_wait<TC_RS - 2>();  // this thread's copies of slab s have landed
        // Slab s - 2 used the operand buffer hb; its MMAs must have finished
        // (phase (s - 2) / 2 of that buffer's barrier).
        if (s >= TC_HS && tid == 0)
          wait_ok = mbar_wait(smem_addr(&bars[hb]), (uint32_t)(((s - TC_HS) >> 1) & 1)) ? 1 : 0;
        __syncthreads();  // slab s visible to all; slot (s - 1) % RS free
        if (s >= TC_HS && !wait_ok) {
          ok = false;
          break;
        }
        produce((s + TC_RS - 1) % TC_RS);
        const GemmEntry<float> en = ents[cons.e];
        const unsigned char* raw = raw_base + (s % TC_RS) * TC_RAW;
        unsigned char* hl = hl_base + hb * TC_HL;
        const int a_kc = en.opA, b_kc = en.opB ? 0 : 1;
        convert_operand(raw, a_kc, en.alpha, hl, hl + TC_TILE, tid);
        convert_operand(raw + TC_TILE, b_kc, 1.f, hl + 2 * TC_TILE, hl + 3 * TC_TILE, tid);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t idesc = make_idesc(nmma);
          const uint32_t base = smem_addr(hl);
#pragma unroll
          for (int ks = 0; ks < TC_KT / 8; ks++) {
            uint64_t ad[2], bd[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
              ad[h] = make_desc(base + h * TC_TILE + ks * 256, 128, TC_SBO);
              bd[h] = make_desc(base + (2 + h) * TC_TILE + ks * 256, 128, TC_SBO);
            }
            const uint32_t first = (first_slab && ks == 0) ? 0u : 1u;
            if (split) {
              mma_tf32(tmem, ad[1], bd[0], idesc, first);  // lo x hi
              mma_tf32(tmem, ad[0], bd[1], idesc, 1u);     // hi x lo
              mma_tf32(tmem, ad[0], bd[0], idesc, 1u);     // hi x hi
            } else {
              mma_tf32(tmem, ad[0], bd[0], idesc, first);  // one TF32 product
            }
          }
          mma_commit(smem_addr(&bars[hb]));
        }
        first_slab = false;
        more = slab_next(tasks, ents, tiles, ntiles, cons);
        s++;
      }
      if (ok) {
        // The tile's last slab (s - 1): its MMAs and all earlier ones done.
        if (tid == 0) wait_ok = mbar_wait(smem_addr(&bars[(s - 1) & 1]), (uint32_t)(((s - 1) >> 1) & 1)) ? 1 : 0;
        __syncthreads();
        ok = wait_ok != 0;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (!ok) break;

    // Epilogue: warp w reads TMEM lanes 32 (w & 3) .. +31 (tile rows; a warp
    // may only read its lane quarter), warps 0-3 columns 0-63 and warps 4-7
    // columns 64-127, 32 per load; C = beta C + acc, coalesced along the rows
    // of a column.
    const int row = (warp & 3) * 32 + lane;
    for (int c0 = (warp >> 2) * (TC_BN / 2); c0 < (warp >> 2 ? TC_BN : TC_BN / 2); c0 += 32) {
      if (c0 >= ncols) break;
      float acc[32];
      if (any) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)c0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
              "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
              "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 32; j++) acc[j] = __uint_as_float(r[j]);
      } else {
#pragma unroll
        for (int j = 0; j < 32; j++) acc[j] = 0.f;
      }
      if (row < mrows) {
#pragma unroll
        for (int j = 0; j < 32; j++) {
          if (c0 + j < ncols) {
            float* p = task.C + (i64)(m0 + row) + (i64)(n0 + c0 + j) * task.ldc;
            *p = (task.beta == 0.f) ? acc[j] : task.beta * (*p) + acc[j];
          }
        }
      }
    }
    // The next tile's first MMA overwrites the accumulator: every warp's
    // tcgen05.ld must be complete first.
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  cp_wait<0>();
  if (!ok && tid == 0) atomicExch(&g_tc_err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_BN) : "memory");
}

int tc_gemm_tile() { return TC_BM; }

cudaError_t launch_tc_gemm(const GemmTask<float>* d_tasks, const GemmEntry<float>* d_ents, const TileRef* d_tiles,
                           int ntiles, int split, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
  if (e != cudaSuccess) return e;
  // Persistent: two CTAs per SM walk the tile list with a stride of the grid.
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  const int grid = ntiles < 2 * sms ? ntiles : 2 * sms;
  note_launch();
  k_tc_gemm<<<grid, TC_NT, TC_SMEM, st>>>(d_tasks, d_ents, d_tiles, ntiles, split);
  return cudaGetLastError();
}

// Reads and clears the expired-wait flag (synchronises the stream).
cudaError_t tc_gemm_take_error(int* flag, cudaStream_t st) {
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyFromSymbol(flag, g_tc_err, sizeof(int));
  if (e != cudaSuccess) return e;
  const int zero = 0;
  return cudaMemcpyToSymbol(g_tc_err, &zero, sizeof(int));
}

}  // namespace h2b
