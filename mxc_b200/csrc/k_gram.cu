// Batched FP64 Gram matrices G = X^T X (X: S x M column-major per box, the
// far-sample block of the fixed-rank basis construction) on the FP64 tensor
// cores (mma.sync m8n8k4 .f64).
//
// Only the upper-triangle 64 x 64 tiles of each G are computed; each
// off-diagonal tile is also written transposed.  One CTA (4 warps, each a
// 32 x 32 quadrant as 4 x 4 m8n8k4 fragments) owns one tile.  The k (sample)
// dimension is streamed in 32-row slabs through a 3-slot cp.async ring: the
// slab holds the tile's 64 (diagonal tile) or 128 columns of X, each column
// 32 consecutive samples padded to 36 doubles so the fragment loads of a
// half-warp (4 columns x 4 samples) hit 16 distinct bank pairs.
#include "common.cuh"
#include "kernels.h"

#include <cstdint>

namespace h2b {

namespace {

constexpr int GR_T = 64, GR_KS = 32, GR_CS = 36, GR_ST = 3, GR_NT = 128;
constexpr int GR_SLOT = 2 * GR_T * GR_CS;  // doubles per ring slot (128 columns)
constexpr int GR_SMEM = GR_ST * GR_SLOT * 8;

__device__ __forceinline__ uint32_t gsmem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void gcp16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void gcp8(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void gcommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void gwait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

}  // namespace

__global__ void __launch_bounds__(GR_NT, 2) k_gram(const GramTask* __restrict__ tasks, const int4* __restrict__ tiles) {
  extern __shared__ __align__(16) double gsm[];
  const int4 tl = tiles[blockIdx.x];  // {task, tile row, tile col}
  const GramTask t = tasks[tl.x];
  const int c0 = tl.y * GR_T, c1 = tl.z * GR_T;
  const bool diag = tl.y == tl.z;
  const int ncol = diag ? GR_T : 2 * GR_T;  // columns staged per slab
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const bool vec = ((reinterpret_cast<uintptr_t>(t.X) & 15) == 0) && (t.ld % 2 == 0);
  const int nslab = (t.S + GR_KS - 1) / GR_KS;

  // Copies slab `sl` (samples sl*32 .. +31) into ring slot `slot`: staged
  // column j < 64 is X column c0 + j, column 64 + j is X column c1 + j.
  auto produce = [&](int sl, int slot) {
    if (sl < nslab) {
      double* dst = gsm + (size_t)slot * GR_SLOT;
      const int k0 = sl * GR_KS;
      for (int c = tid; c < ncol * (GR_KS / 2); c += GR_NT) {
        const int j = c >> 4, kk = (c & 15) * 2;
        const int col = j < GR_T ? c0 + j : c1 + (j - GR_T);
        const int k = k0 + kk;
        int nk = t.S - k;
        nk = nk < 0 ? 0 : (nk > 2 ? 2 : nk);
        if (col >= t.M) nk = 0;
        const double* src = t.X + (i64)k + (i64)col * t.ld;
        const uint32_t d = gsmem(dst + j * GR_CS + kk);
        if (vec) {
          gcp16(d, nk ? (const void*)src : (const void*)t.X, nk * 8);
        } else {
          gcp8(d, nk > 0 ? (const void*)src : (const void*)t.X, nk > 0 ? 8 : 0);
          gcp8(d + 8, nk > 1 ? (const void*)(src + 1) : (const void*)t.X, nk > 1 ? 8 : 0);
        }
      }
    }
    gcommit();
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.;

#pragma unroll
  for (int s = 0; s < GR_ST - 1; s++) produce(s, s);
  const int fr = lane >> 2, fk = lane & 3;  // fragment row / column within m8n8k4
  for (int sl = 0; sl < nslab; sl++) {
    gwait<GR_ST - 2>();
    __syncthreads();
    produce(sl + GR_ST - 1, (sl + GR_ST - 1) % GR_ST);
    const double* base = gsm + (size_t)(sl % GR_ST) * GR_SLOT;
    const double* as = base + (wm * 32 + fr) * GR_CS + fk;
    const double* bs = base + ((diag ? 0 : GR_T) + wn * 32 + fr) * GR_CS + fk;
#pragma unroll
    for (int ks = 0; ks < GR_KS; ks += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = as[i * 8 * GR_CS + ks];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = bs[j * 8 * GR_CS + ks];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) dmma(acc[i][j], a[i], b[j]);
    }
  }
  gwait<0>();

  // D fragment of m8n8k4: lane holds row lane >> 2, columns 2 (lane & 3) + {0, 1}.
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = c0 + wm * 32 + i * 8 + fr;
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int c = c1 + wn * 32 + j * 8 + 2 * fk + h;
        if (r < t.M && c < t.M) {
          t.G[(i64)r + (i64)c * t.ldg] = acc[i][j][h];
          if (!diag) t.G[(i64)c + (i64)r * t.ldg] = acc[i][j][h];
        }
      }
    }
  }
}

int gram_tile() { return GR_T; }

cudaError_t launch_gram(const GramTask* d_tasks, const int4* d_tiles, int ntiles, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, GR_SMEM);
  if (e != cudaSuccess) return e;
  note_launch();
  k_gram<<<ntiles, GR_NT, GR_SMEM, st>>>(d_tasks, d_tiles);
  return cudaGetLastError();
}

}  // namespace h2b
