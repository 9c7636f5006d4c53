// BF16 storage for the ULV substitution (preconditioner apply) of an FP32
// preconditioner: every block the forward / backward substitution streams
// (V, the sr and rs parts of the near blocks, U; h2matrix.cpp:448-537) is
// kept as BF16 scaled per block by a power of two (so the stored values lie
// in [-1, 1] and the scaling itself is exact), and applied with FP32
// arithmetic: C = beta C + sum_e (alpha_e s_e) A_e B_e with A_e converted
// from BF16 on the fly.  The apply is HBM-bound (2 bytes per matrix element
// instead of 4); BF16 keeps 8 significand bits, so the preconditioner is
// less accurate and GMRES may need more steps (the ablation in the
// benchmark records both).
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
  else if (nr <= 8)
    k_stream_bf16<8, 256><<<ntiles, 128, 0, st>>>(d_tasks, d_ents, d_tiles);
  else
    k_stream_bf16<16, 256><<<ntiles, 128, 0, st>>>(d_tasks, d_ents, d_tiles);
  return cudaGetLastError();
}

}  // namespace h2b
