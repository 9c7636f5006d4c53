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
// One CTA (128 threads) owns a 128 x 128 output tile; its accumulator is 128
// TMEM lanes x 128 columns.  The task's (entry, 32-wide k slab) sequence is
// double buffered in shared memory: all threads load slab s+1 from global
// memory into registers while the tensor cores multiply slab s, then split
// it into hi / lo and store it in the canonical no-swizzle K-major UMMA
// layout (operands stored with rows contiguous are transposed 4 x 4 in
// registers on the way; every global load is a 16-byte vector of
// consecutive elements and every shared store is conflict-free).  One
// thread issues the 12 MMAs of a slab (4 k-steps x 3 products) and commits
// them to the slab's mbarrier; the buffer is refilled after that barrier
// completes.  Every mbarrier wait is bounded (about a second of clock
// cycles); on expiry the kernel records an error code and leaves.
#include "common.cuh"
#include "kernels.h"

#include <cstdint>

namespace h2b {

namespace {

constexpr int TC_BM = 128, TC_BN = 128, TC_KT = 32, TC_NT = 128;
constexpr int TC_TILE = TC_BM * TC_KT * 4;  // bytes of one 128 x 32 FP32 operand tile
constexpr int TC_STAGE = 4 * TC_TILE;       // A hi, A lo, B hi, B lo
constexpr int TC_STAGES = 2;
constexpr int TC_SMEM = TC_STAGES * TC_STAGE + 128;
constexpr long long TC_WAIT_CYCLES = 4000000000LL;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Canonical no-swizzle K-major layout (byte offsets inside a 128 x 32
// tile): core matrix = 8 rows x 16 bytes (4 k); k-chunks 128 B apart
// (leading byte offset), 8-row groups 1024 B apart (stride byte offset).
__device__ __forceinline__ int off_kmajor(int r, int kc) { return (r >> 3) * 1024 + kc * 128 + (r & 7) * 16; }

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

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the given phase parity of an mbarrier.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_test(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_test(bar, parity)) {
    if (clock64() - t0 > TC_WAIT_CYCLES) return false;
    __nanosleep(64);
  }
  return true;
}

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t u;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(x));
  return __uint_as_float(u & 0xFFFFE000u);
}

// One operand of a slab: 128 rows (of op(X), rows of the output tile) by
// 32 k.  kcontig: element (r, k) at X[k + r * ld]; otherwise at X[r + k * ld].
struct OperandRef {
  const float* X;
  i64 ld;
  int rows;  // valid rows in the tile (from the tile origin)
  int r0;    // tile origin in rows
  int k0, K;
  int kcontig;
  int vec;   // 16-byte vector loads are aligned
  float scale;
};

// Thread-to-chunk maps of a 128 x 32 operand tile (1024 chunks of 16 bytes,
// 8 per thread).  Both store into the K-major layout; each 8-lane phase of a
// 16-byte shared store covers 8 distinct rows mod 8, so stores are
// conflict-free.
//  - k contiguous in global memory: chunk c = tid + 128 i holds row
//    ((c >> 6) << 3) | (c & 7), k-chunk (c >> 3) & 7, one 16-byte load.
//  - rows contiguous: lane = 8p + 2a + b loads, for warp task wt = warp + 4i
//    (i < 2), rows 4q..4q+3 with q = 8 (wt & 3) + 2p + b at the four k of
//    k-chunk kc = 4 (wt >> 2) + a (four 16-byte loads along the rows), and
//    stores the transposed 4 x 4 block row by row, starting at row
//    (t + a) & 3 in step t so the eight lanes of a phase hit eight rows.
__device__ __forceinline__ float pick(const float4& v, int j) {
  return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}

__device__ __forceinline__ void load_operand(const OperandRef& o, float4 (&v)[8], int tid) {
  if (o.kcontig) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int c = tid + TC_NT * i;
      const int r = ((c >> 6) << 3) | (c & 7), k = ((c >> 3) & 7) * 4;
      const int gk = o.k0 + k;
      float e[4] = {0.f, 0.f, 0.f, 0.f};
      if (r < o.rows) {
        const float* p = o.X + (i64)gk + (i64)(o.r0 + r) * o.ld;
        if (o.vec && gk + 3 < o.K) {
          const float4 t = __ldg(reinterpret_cast<const float4*>(p));
          e[0] = t.x; e[1] = t.y; e[2] = t.z; e[3] = t.w;
        } else {
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (gk + j < o.K) e[j] = __ldg(p + j);
        }
      }
      v[i] = make_float4(e[0] * o.scale, e[1] * o.scale, e[2] * o.scale, e[3] * o.scale);
    }
  } else {
    const int lane = tid & 31, warp = tid >> 5;
    const int p = lane >> 3, a = (lane >> 1) & 3, b = lane & 1;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const int wt = warp + 4 * i;
      const int r = 4 * ((wt & 3) * 8 + 2 * p + b);
      const int kc = (wt >> 2) * 4 + a;
#pragma unroll
      for (int t = 0; t < 4; t++) {
        const int gk = o.k0 + 4 * kc + t;
        float e[4] = {0.f, 0.f, 0.f, 0.f};
        if (gk < o.K) {
          const float* q = o.X + (i64)(o.r0 + r) + (i64)gk * o.ld;
          if (o.vec && r + 3 < o.rows) {
            const float4 x = __ldg(reinterpret_cast<const float4*>(q));
            e[0] = x.x; e[1] = x.y; e[2] = x.z; e[3] = x.w;
          } else {
#pragma unroll
            for (int j = 0; j < 4; j++)
              if (r + j < o.rows) e[j] = __ldg(q + j);
          }
        }
        v[4 * i + t] = make_float4(e[0] * o.scale, e[1] * o.scale, e[2] * o.scale, e[3] * o.scale);
      }
    }
  }
}

__device__ __forceinline__ void store_split(unsigned char* hi, unsigned char* lo, int off, const float4& x) {
  float4 h, l;
  h.x = tf32_hi(x.x); l.x = x.x - h.x;
  h.y = tf32_hi(x.y); l.y = x.y - h.y;
  h.z = tf32_hi(x.z); l.z = x.z - h.z;
  h.w = tf32_hi(x.w); l.w = x.w - h.w;
  *reinterpret_cast<float4*>(hi + off) = h;
  *reinterpret_cast<float4*>(lo + off) = l;
}

// Splits the chunks into hi / lo and stores them K-major.
__device__ __forceinline__ void store_operand(const float4 (&v)[8], int kcontig, unsigned char* hi,
                                              unsigned char* lo, int tid) {
  if (kcontig) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int c = tid + TC_NT * i;
      store_split(hi, lo, off_kmajor(((c >> 6) << 3) | (c & 7), (c >> 3) & 7), v[i]);
    }
  } else {
    const int lane = tid & 31, warp = tid >> 5;
    const int p = lane >> 3, a = (lane >> 1) & 3, b = lane & 1;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const int wt = warp + 4 * i;
      const int r = 4 * ((wt & 3) * 8 + 2 * p + b);
      const int kc = (wt >> 2) * 4 + a;
#pragma unroll
      for (int t = 0; t < 4; t++) {
        const int j = (t + a) & 3;
        const float4 x = make_float4(pick(v[4 * i], j), pick(v[4 * i + 1], j), pick(v[4 * i + 2], j),
                                     pick(v[4 * i + 3], j));
        store_split(hi, lo, off_kmajor(r + j, kc), x);
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

}  // namespace

// Set when an mbarrier wait expired (read and cleared by the host).
__device__ int g_tc_err = 0;

__global__ void __launch_bounds__(TC_NT, 1)
    k_tc_gemm(const GemmTask<float>* __restrict__ tasks, const GemmEntry<float>* __restrict__ ents,
              const TileRef* __restrict__ tiles) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bars[TC_STAGES];
  __shared__ uint32_t tmem_slot;
  __shared__ int wait_ok;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const TileRef tl = tiles[blockIdx.x];
  const GemmTask<float> task = tasks[tl.task];
  const int m0 = tl.tm * TC_BM, n0 = tl.tn * TC_BN;
  const int mrows = min(TC_BM, task.m - m0), ncols = min(TC_BN, task.n - n0);
  const int nmma = ((ncols + 15) / 16) * 16;  // MMA N: multiple of 16, >= 16

  if (tid == 0) {
    for (int s = 0; s < TC_STAGES; s++)
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

  SlabCursor cur{task.e0, 0};
  skip_empty(ents, task.e1, cur);
  const bool any = cur.e < task.e1;
  bool ok = true;
  int s = 0;
  if (any) {
    float4 va[8], vb[8];
    int a_kc = 0, b_kc = 0;
    auto fetch = [&](const SlabCursor& c) {
      const GemmEntry<float> en = ents[c.e];
      OperandRef a, b;
      a.X = en.A; a.ld = en.lda; a.rows = mrows; a.r0 = m0; a.k0 = c.k0; a.K = en.k;
      a.kcontig = en.opA;  // op(A)(m, k) = A[k + m lda] when transposed
      a.vec = ((reinterpret_cast<uintptr_t>(en.A) & 15) == 0) && (en.lda % 4 == 0);
      a.scale = en.alpha;
      b.X = en.B; b.ld = en.ldb; b.rows = ncols; b.r0 = n0; b.k0 = c.k0; b.K = en.k;
      b.kcontig = en.opB ? 0 : 1;  // op(B)(k, n) = B[k + n ldb] when not transposed
      b.vec = ((reinterpret_cast<uintptr_t>(en.B) & 15) == 0) && (en.ldb % 4 == 0);
      b.scale = 1.f;
      load_operand(a, va, tid);
      load_operand(b, vb, tid);
      a_kc = a.kcontig;
      b_kc = b.kcontig;
    };
    fetch(cur);
    uint32_t phase[TC_STAGES] = {0u, 0u};
    for (;;) {
      const int buf = s & 1;
      unsigned char* st = smem + buf * TC_STAGE;
      if (s >= TC_STAGES) {
        // The MMAs that read this buffer two slabs ago must have finished
        // (one thread waits; the verdict is shared so all leave together).
        if (tid == 0) wait_ok = mbar_wait(smem_addr(&bars[buf]), phase[buf]) ? 1 : 0;
        __syncthreads();
        if (!wait_ok) {
          ok = false;
          break;
        }
        phase[buf] ^= 1u;
      }
      store_operand(va, a_kc, st, st + TC_TILE, tid);
      store_operand(vb, b_kc, st + 2 * TC_TILE, st + 3 * TC_TILE, tid);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t idesc = make_idesc(nmma);
        const uint32_t base = smem_addr(st);
#pragma unroll
        for (int ks = 0; ks < TC_KT / 8; ks++) {
          uint64_t ad[2], bd[2];
#pragma unroll
          for (int h = 0; h < 2; h++) {
            ad[h] = make_desc(base + h * TC_TILE + ks * 256, 128, 1024);
            bd[h] = make_desc(base + (2 + h) * TC_TILE + ks * 256, 128, 1024);
          }
          const uint32_t first = (s == 0 && ks == 0) ? 0u : 1u;
          mma_tf32(tmem, ad[1], bd[0], idesc, first);  // lo x hi
          mma_tf32(tmem, ad[0], bd[1], idesc, 1u);     // hi x lo
          mma_tf32(tmem, ad[0], bd[0], idesc, 1u);     // hi x hi
        }
        mma_commit(smem_addr(&bars[buf]));
      }
      // Next slab.
      cur.k0 += TC_KT;
      if (cur.k0 >= ents[cur.e].k) {
        cur.k0 = 0;
        cur.e++;
        skip_empty(ents, task.e1, cur);
      }
      s++;
      if (cur.e >= task.e1) break;
      fetch(cur);
    }
    if (ok) {
      // Wait for the last slab's MMAs (all earlier ones complete before it).
      const int buf = (s - 1) & 1;
      if (tid == 0) wait_ok = mbar_wait(smem_addr(&bars[buf]), phase[buf]) ? 1 : 0;
      __syncthreads();
      ok = wait_ok != 0;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (!ok && tid == 0) atomicExch(&g_tc_err, 1);

  // Epilogue: warp w reads TMEM lanes 32w..32w+31 (tile rows), 32 columns
  // per load; C = beta C + acc, coalesced along the rows of a column.
  const int row = warp * 32 + lane;
  for (int c0 = 0; c0 < TC_BN; c0 += 32) {
    if (c0 >= ncols) break;
    float acc[32];
    if (any && ok) {
      uint32_t r[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
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
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_BN) : "memory");
}

int tc_gemm_tile() { return TC_BM; }

cudaError_t launch_tc_gemm(const GemmTask<float>* d_tasks, const GemmEntry<float>* d_ents, const TileRef* d_tiles,
                           int ntiles, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
  if (e != cudaSuccess) return e;
  note_launch();
  k_tc_gemm<<<ntiles, TC_NT, TC_SMEM, st>>>(d_tasks, d_ents, d_tiles);
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
