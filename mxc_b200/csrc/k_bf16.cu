// BF16 storage for the ULV substitution (preconditioner apply) of an FP32
// preconditioner: every block the forward / backward substitution streams
// (V, the sr and rs parts of the near blocks, U; h2matrix.cpp:448-537) is
// kept as BF16 scaled per block by a power of two (so the stored values lie
// in [-1, 1] and the scaling itself is exact), and applied with FP32
// accumulation: C = beta C + sum_e (alpha_e s_e) A_e B_e.  For 5-16
// right-hand sides the products run on the BF16 tensor cores with B split
// into two BF16 terms; for 1-4 A is converted from BF16 on the fly on the
// FMA pipe.  The apply streams 2 bytes per matrix element instead of 4;
// BF16 keeps 8 significand bits, so the preconditioner is less accurate and
// GMRES may need more steps (the ablation in the benchmark records both).
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"

namespace h2b {

namespace {

__device__ __forceinline__ void bf_cp16(void* smem, const void* gmem, int bytes) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bf_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bf_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

}  // namespace

// One CTA per block: s = 2^ceil(log2(max |A|)) (1 for a zero block), dst =
// bf16(A / s) column-major with leading dimension ldd (a multiple of 8, so
// every column starts on a 16-byte boundary), *scale = s.
__global__ void __launch_bounds__(256) k_bf16_pack(const BfPackTask* __restrict__ tasks) {
  __shared__ float red[32];
  const BfPackTask t = tasks[blockIdx.x];
  float mx = 0.f;
  for_each_rc(t.m, t.k, [&](int r, int c, int) { mx = fmaxf(mx, fabsf(t.src[r + (i64)c * t.lds])); });
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = mx;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  mx = red[0];
  int e = 0;
  if (mx > 0.f && isfinite(mx)) frexpf(mx, &e);  // mx = f 2^e, f in [0.5, 1): 2^e >= mx
  const float s = ldexpf(1.f, e), inv = ldexpf(1.f, -e);
  for_each_rc(t.m, t.k, [&](int r, int c, int) { t.dst[r + (i64)c * t.ldd] = __float2bfloat16_rn(t.src[r + (i64)c * t.lds] * inv); });
  if (threadIdx.x == 0) *t.scale = s;
}

cudaError_t launch_bf16_pack(const BfPackTask* d_tasks, int ntasks, cudaStream_t st) {
  if (ntasks == 0) return cudaSuccess;
  note_launch();
  k_bf16_pack<<<ntasks, 256, 0, st>>>(d_tasks);
  return cudaGetLastError();
}

// Streaming apply, one CTA per {task, BM-row block}: each thread owns two
// consecutive rows and accumulates NR right-hand sides in FP32 registers;
// A slabs (BF16, KS columns x BM rows) and B slabs (FP32, KS x NR) go
// through a 3-slot cp.async ring.  A columns start on 16-byte boundaries
// (packed layout) and task rows start at multiples of 8, so every A copy is
// a 16-byte vector of 8 BF16 values.
constexpr int BF_KS = 16, BF_ST = 3;

template <int NR, int BM>
__global__ void __launch_bounds__(BM / 2) k_stream_bf16(const GemmTask<float>* __restrict__ tasks,
                                                        const BfEntry* __restrict__ ents,
                                                        const int2* __restrict__ tiles) {
  constexpr int NT = BM / 2;
  __shared__ __align__(16) __nv_bfloat16 As[BF_ST][BF_KS][BM];
  __shared__ __align__(16) float Bs[BF_ST][BF_KS][NR];
  const int2 tl = tiles[blockIdx.x];
  const GemmTask<float> task = tasks[tl.x];
  const int m0 = tl.y * BM;
  const int mrows = min(BM, task.m - m0);
  const int tid = threadIdx.x;

  int pe = task.e0, pk = 0;
  while (pe < task.e1 && ents[pe].k <= 0) pe++;
  auto issue = [&](int slot) {
    if (pe < task.e1) {
      const BfEntry en = ents[pe];
      for (int c = tid; c < BF_KS * (BM / 8); c += NT) {
        const int k = c / (BM / 8), r = (c % (BM / 8)) * 8;
        int valid = mrows - r;
        valid = valid < 0 ? 0 : (valid > 8 ? 8 : valid);
        if (pk + k >= en.k) valid = 0;
        const __nv_bfloat16* src = valid ? en.A + (i64)(m0 + r) + (i64)(pk + k) * en.lda : en.A;
        bf_cp16(&As[slot][k][r], src, valid * 2);
      }
      for (int c = tid; c < BF_KS * NR; c += NT) {
        const int k = c / NR, j = c % NR;
        const bool ok = j < task.n && pk + k < en.k;
        if (ok)
          Bs[slot][k][j] = en.B[(i64)(pk + k) + (i64)j * en.ldb];
        else
          Bs[slot][k][j] = 0.f;
      }
      pk += BF_KS;
      if (pk >= en.k) {
        pk = 0;
        pe++;
        while (pe < task.e1 && ents[pe].k <= 0) pe++;
      }
    }
    bf_commit();
  };

  float acc[2][NR];
#pragma unroll
  for (int t = 0; t < 2; t++)
#pragma unroll
    for (int j = 0; j < NR; j++) acc[t][j] = 0.f;

#pragma unroll
  for (int s = 0; s < BF_ST - 1; s++) issue(s);
  int ce = task.e0, ck = 0;
  while (ce < task.e1 && ents[ce].k <= 0) ce++;
  int slot = 0;
  while (ce < task.e1) {
    const float alpha = ents[ce].alpha * *ents[ce].scale;
    bf_wait<BF_ST - 2>();
    __syncthreads();
    issue((slot + BF_ST - 1) % BF_ST);
#pragma unroll
    for (int k = 0; k < BF_KS; k++) {
      const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&As[slot][k][2 * tid]));
      const float a0 = a.x * alpha, a1 = a.y * alpha;
#pragma unroll
      for (int j = 0; j < NR; j++) {
        const float bj = Bs[slot][k][j];
        acc[0][j] = fmaf(a0, bj, acc[0][j]);
        acc[1][j] = fmaf(a1, bj, acc[1][j]);
      }
    }
    ck += BF_KS;
    if (ck >= ents[ce].k) {
      ck = 0;
      ce++;
      while (ce < task.e1 && ents[ce].k <= 0) ce++;
    }
    slot = (slot + 1) % BF_ST;
  }
  bf_wait<0>();
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int r = 2 * tid + t;
    if (r >= mrows) continue;
#pragma unroll
    for (int j = 0; j < NR; j++) {
      if (j >= task.n) break;
      float* p = task.C + (m0 + r) + (i64)j * task.ldc;
      *p = (task.beta == 0.f) ? acc[t][j] : task.beta * (*p) + acc[t][j];
    }
  }
}

// Tensor-core variant for 5-16 right-hand sides: mma.sync m16n8k16 with
// BF16 A (the stored blocks) and the FP32 right-hand sides split into two
// BF16 terms (hi = bf16(b), lo = bf16(b - hi): 16 significand bits of b),
// FP32 accumulation, so the product carries A's BF16 rounding and little
// else.  256 threads per 256-row tile, each warp 32 rows x NR columns as two
// 16-row MMA blocks interleaved in groups of four rows (MMA row g / g + 8 of
// block rb is tile row 4g + 2rb / 4g + 2rb + 1), so one 8-byte load gives a
// lane its four rows of one column and byte permutes pair them along k.
// 32-column stages through a 3-slot cp.async ring; A columns are stored
// BM + 8 values apart and B rows 24 floats apart (bank-conflict-free
// fragment loads).
constexpr int BFM_KS = 32, BFM_ST = 3, BFM_BM = 256, BFM_AS = BFM_BM + 8, BFM_BS = 24;

constexpr size_t stream_bf16_mma_smem() {
  return (size_t)BFM_ST * BFM_KS * (BFM_AS * sizeof(__nv_bfloat16) + BFM_BS * sizeof(float));
}

__device__ __forceinline__ void bfm_cp4(void* smem, const void* gmem, int bytes) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}

__device__ __forceinline__ uint32_t bfm_pack(float x, float y) {
  __nv_bfloat162 v = __floats2bfloat162_rn(x, y);  // .x (low half) = x
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void bfm_mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int NR>
__global__ void __launch_bounds__(BFM_BM, 2) k_stream_bf16_mma(const GemmTask<float>* __restrict__ tasks,
                                                              const BfEntry* __restrict__ ents,
                                                              const int2* __restrict__ tiles) {
  constexpr int NT = BFM_BM, NF = NR / 8;
  extern __shared__ __align__(16) unsigned char bfm_smem[];
  __nv_bfloat16* As = reinterpret_cast<__nv_bfloat16*>(bfm_smem);               // [ST][KS][AS]
  float* Bs = reinterpret_cast<float*>(As + (size_t)BFM_ST * BFM_KS * BFM_AS);  // [ST][KS][BS]
  const int2 tl = tiles[blockIdx.x];
  const GemmTask<float> task = tasks[tl.x];
  const int m0 = tl.y * BFM_BM;
  const int mrows = min(BFM_BM, task.m - m0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  int pe = task.e0, pk = 0;
  while (pe < task.e1 && ents[pe].k <= 0) pe++;
  auto issue = [&](int slot) {
    if (pe < task.e1) {
      const BfEntry en = ents[pe];
      __nv_bfloat16* as = As + (size_t)slot * BFM_KS * BFM_AS;
      float* bs = Bs + (size_t)slot * BFM_KS * BFM_BS;
      for (int c = tid; c < BFM_KS * (BFM_BM / 8); c += NT) {
        const int k = c / (BFM_BM / 8), r = (c % (BFM_BM / 8)) * 8;
        int valid = mrows - r;
        valid = valid < 0 ? 0 : (valid > 8 ? 8 : valid);
        if (pk + k >= en.k) valid = 0;
        const __nv_bfloat16* src = valid ? en.A + (i64)(m0 + r) + (i64)(pk + k) * en.lda : en.A;
        bf_cp16(as + k * BFM_AS + r, src, valid * 2);
      }
      for (int c = tid; c < BFM_KS * NR; c += NT) {
        const int k = c % BFM_KS, j = c / BFM_KS;
        const bool ok = j < task.n && pk + k < en.k;
        bfm_cp4(bs + k * BFM_BS + j, ok ? en.B + (i64)(pk + k) + (i64)j * en.ldb : en.B, ok ? 4 : 0);
      }
      pk += BFM_KS;
      if (pk >= en.k) {
        pk = 0;
        pe++;
        while (pe < task.e1 && ents[pe].k <= 0) pe++;
      }
    }
    bf_commit();
  };

  float acc[2][NF][4];
#pragma unroll
  for (int rb = 0; rb < 2; rb++)
#pragma unroll
    for (int cb = 0; cb < NF; cb++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[rb][cb][q] = 0.f;

#pragma unroll
  for (int s = 0; s < BFM_ST - 1; s++) issue(s);
  int ce = task.e0, ck = 0;
  while (ce < task.e1 && ents[ce].k <= 0) ce++;
  int slot = 0;
  const int g8 = lane >> 2, t4 = lane & 3, wr = warp * 32;
  const bool live = wr < mrows;
  while (ce < task.e1) {
    const float alpha = ents[ce].alpha * *ents[ce].scale;
    bf_wait<BFM_ST - 2>();
    __syncthreads();
    issue((slot + BFM_ST - 1) % BFM_ST);
    if (live) {
      const __nv_bfloat16* as = As + (size_t)slot * BFM_KS * BFM_AS + wr + 4 * g8;
      const float* bs = Bs + (size_t)slot * BFM_KS * BFM_BS + g8;
#pragma unroll
      for (int ks = 0; ks < BFM_KS; ks += 16) {
        // A: rows 4g .. 4g + 3 of columns ks + 2t + {0, 1} (fragment regs 0, 1)
        // and ks + 2t + 8 + {0, 1} (regs 2, 3).
        uint32_t a[2][4];
#pragma unroll
        for (int p = 0; p < 2; p++) {
          const int c = ks + 2 * t4 + 8 * p;
          const uint2 v0 = *reinterpret_cast<const uint2*>(as + c * BFM_AS);
          const uint2 v1 = *reinterpret_cast<const uint2*>(as + (c + 1) * BFM_AS);
          a[0][2 * p] = __byte_perm(v0.x, v1.x, 0x5410);      // row 4g     (block 0, MMA row g)
          a[0][2 * p + 1] = __byte_perm(v0.x, v1.x, 0x7632);  // row 4g + 1 (block 0, MMA row g + 8)
          a[1][2 * p] = __byte_perm(v0.y, v1.y, 0x5410);      // row 4g + 2 (block 1, MMA row g)
          a[1][2 * p + 1] = __byte_perm(v0.y, v1.y, 0x7632);  // row 4g + 3 (block 1, MMA row g + 8)
        }
#pragma unroll
        for (int cb = 0; cb < NF; cb++) {
          // B: k = ks + 2t + {0, 1} (reg 0) and ks + 2t + 8 + {0, 1} (reg 1), column cb * 8 + g.
          const float* bp = bs + cb * 8 + (ks + 2 * t4) * BFM_BS;
          float x[4] = {alpha * bp[0], alpha * bp[BFM_BS], alpha * bp[8 * BFM_BS], alpha * bp[9 * BFM_BS]};
          float lo[4];
#pragma unroll
          for (int q = 0; q < 4; q++) lo[q] = x[q] - __bfloat162float(__float2bfloat16_rn(x[q]));
          const uint32_t h0 = bfm_pack(x[0], x[1]), h1 = bfm_pack(x[2], x[3]);
          const uint32_t l0 = bfm_pack(lo[0], lo[1]), l1 = bfm_pack(lo[2], lo[3]);
#pragma unroll
          for (int rb = 0; rb < 2; rb++) {
            bfm_mma(acc[rb][cb], a[rb], l0, l1);
            bfm_mma(acc[rb][cb], a[rb], h0, h1);
          }
        }
      }
    }
    ck += BFM_KS;
    if (ck >= ents[ce].k) {
      ck = 0;
      ce++;
      while (ce < task.e1 && ents[ce].k <= 0) ce++;
    }
    slot = (slot + 1) % BFM_ST;
  }
  bf_wait<0>();
  if (!live) return;
  // C fragment of block rb: c[2h + q] is MMA row g8 + 8h = tile row
  // 4 g8 + 2 rb + h, column 2 t4 + q of the column block.
#pragma unroll
  for (int rb = 0; rb < 2; rb++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = wr + 4 * g8 + 2 * rb + h;
      if (r >= mrows) continue;
#pragma unroll
      for (int cb = 0; cb < NF; cb++)
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int c = cb * 8 + 2 * t4 + q;
          if (c < task.n) {
            float* p = task.C + (m0 + r) + (i64)c * task.ldc;
            const float v = acc[rb][cb][2 * h + q];
            *p = (task.beta == 0.f) ? v : task.beta * (*p) + v;
          }
        }
    }
}

int bf16_rows_per_cta() { return 256; }

cudaError_t launch_stream_bf16(int nr, const GemmTask<float>* d_tasks, const BfEntry* d_ents, const int2* d_tiles,
                               int ntiles, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  if (nr < 1 || nr > 16) return cudaErrorInvalidValue;
  note_launch();
  if (nr <= 1)
    k_stream_bf16<1, 256><<<ntiles, 128, 0, st>>>(d_tasks, d_ents, d_tiles);
  else if (nr <= 2)
    k_stream_bf16<2, 256><<<ntiles, 128, 0, st>>>(d_tasks, d_ents, d_tiles);
  else if (nr <= 4)
    k_stream_bf16<4, 256><<<ntiles, 128, 0, st>>>(d_tasks, d_ents, d_tiles);
  else {
    auto kern = nr <= 8 ? k_stream_bf16_mma<8> : k_stream_bf16_mma<16>;
    const size_t smem = stream_bf16_mma_smem();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<ntiles, BFM_BM, smem, st>>>(d_tasks, d_ents, d_tiles);
  }
  return cudaGetLastError();
}

}  // namespace h2b
