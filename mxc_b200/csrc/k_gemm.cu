// Segmented batched GEMM: every output task C_t (m x n, column-major)
// receives beta * C_t + sum over its entries of alpha * op(A) op(B).  One
// CTA computes one BM x BN tile of one task; the task/tile list is built on
// the host once per level and reused.  This single kernel carries the ULV
// basis transforms and Schur updates (h2matrix.cpp:373-422), the H^2
// matvec passes (h2matrix.cpp:251-344) and the ULV substitution
// (h2matrix.cpp:448-537), with variable box sizes and ranks.
#include "common.cuh"
#include "kernels.h"

namespace h2b {

template <typename T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) k_seg_gemm(const GemmTask<T>* __restrict__ tasks,
                                                                    const GemmEntry<T>* __restrict__ ents,
                                                                    const TileRef* __restrict__ tiles) {
  constexpr int NT = (BM / TM) * (BN / TN);
  constexpr int RG = BM / TM;  // row groups: thread row index fastest
  __shared__ T As[BK][BM + 1];
  __shared__ T Bs[BK][BN + 1];
  const TileRef tr = tiles[blockIdx.x];
  const GemmTask<T> task = tasks[tr.task];
  const int m0 = tr.tm * BM, n0 = tr.tn * BN;
  const int tid = threadIdx.x;
  const int tr_ = tid % RG, tc_ = tid / RG;
  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++) acc[i][j] = T(0);

  for (int e = task.e0; e < task.e1; e++) {
    const GemmEntry<T> en = ents[e];
    const int K = en.k;
    for (int k0 = 0; k0 < K; k0 += BK) {
      if (en.opA == 0) {
        for (int idx = tid; idx < BM * BK; idx += NT) {
          int mm = idx % BM, kk = idx / BM;
          int r = m0 + mm, k = k0 + kk;
          As[kk][mm] = (r < task.m && k < K) ? en.alpha * en.A[r + (i64)k * en.lda] : T(0);
        }
      } else {
        for (int idx = tid; idx < BM * BK; idx += NT) {
          int kk = idx % BK, mm = idx / BK;
          int r = m0 + mm, k = k0 + kk;
          As[kk][mm] = (r < task.m && k < K) ? en.alpha * en.A[k + (i64)r * en.lda] : T(0);
        }
      }
      if (en.opB == 0) {
        for (int idx = tid; idx < BN * BK; idx += NT) {
          int kk = idx % BK, nn = idx / BK;
          int c = n0 + nn, k = k0 + kk;
          Bs[kk][nn] = (c < task.n && k < K) ? en.B[k + (i64)c * en.ldb] : T(0);
        }
      } else {
        for (int idx = tid; idx < BN * BK; idx += NT) {
          int nn = idx % BN, kk = idx / BN;
          int c = n0 + nn, k = k0 + kk;
          Bs[kk][nn] = (c < task.n && k < K) ? en.B[c + (i64)k * en.ldb] : T(0);
        }
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < BK; kk++) {
        T a[TM], b[TN];
#pragma unroll
        for (int i = 0; i < TM; i++) a[i] = As[kk][tr_ + i * RG];
#pragma unroll
        for (int j = 0; j < TN; j++) b[j] = Bs[kk][tc_ + j * (BN / TN)];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
          for (int j = 0; j < TN; j++) acc[i][j] += a[i] * b[j];
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int j = 0; j < TN; j++) {
    int c = n0 + tc_ + j * (BN / TN);
    if (c >= task.n) continue;
#pragma unroll
    for (int i = 0; i < TM; i++) {
      int r = m0 + tr_ + i * RG;
      if (r >= task.m) continue;
      T* p = task.C + r + (i64)c * task.ldc;
      *p = (task.beta == T(0)) ? acc[i][j] : task.beta * (*p) + acc[i][j];
    }
  }
}

int gemm_tile_m(int shape) { return shape == GEMM_BIG ? 64 : 128; }
int gemm_tile_n(int shape) { return shape == GEMM_BIG ? 64 : 16; }

template <typename T>
cudaError_t launch_seg_gemm(int shape, const GemmTask<T>* d_tasks, const GemmEntry<T>* d_ents, const TileRef* d_tiles,
                            int ntiles, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  if (shape == GEMM_BIG)
    k_seg_gemm<T, 64, 64, 16, 4, 4><<<ntiles, 256, 0, st>>>(d_tasks, d_ents, d_tiles);
  else
    k_seg_gemm<T, 128, 16, 16, 4, 2><<<ntiles, 256, 0, st>>>(d_tasks, d_ents, d_tiles);
  return cudaGetLastError();
}
template cudaError_t launch_seg_gemm<double>(int, const GemmTask<double>*, const GemmEntry<double>*, const TileRef*,
                                             int, cudaStream_t);
template cudaError_t launch_seg_gemm<float>(int, const GemmTask<float>*, const GemmEntry<float>*, const TileRef*, int,
                                            cudaStream_t);

template <typename T>
__global__ void __launch_bounds__(256) k_batched_copy(const CopyEntry<T>* __restrict__ ents) {
  const CopyEntry<T> e = ents[blockIdx.x];
  i64 total = (i64)e.m * e.n;
  for (i64 x = threadIdx.x; x < total; x += blockDim.x) {
    int r = (int)(x % e.m), c = (int)(x / e.m);
    e.dst[r + (i64)c * e.ldd] = e.trans ? e.src[c + (i64)r * e.lds] : e.src[r + (i64)c * e.lds];
  }
}

template <typename T>
cudaError_t launch_batched_copy(const CopyEntry<T>* d_ents, int n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_batched_copy<T><<<n, 256, 0, st>>>(d_ents);
  return cudaGetLastError();
}
template cudaError_t launch_batched_copy<double>(const CopyEntry<double>*, int, cudaStream_t);
template cudaError_t launch_batched_copy<float>(const CopyEntry<float>*, int, cudaStream_t);

template <typename T>
__global__ void __launch_bounds__(256) k_set_identity(T* base, const i64* __restrict__ qoff, const i64* __restrict__ dims) {
  const int box = blockIdx.x;
  const i64 M = dims[box];
  T* q = base + qoff[box];
  for (i64 e = threadIdx.x; e < M * M; e += blockDim.x) q[e] = (e % M == e / M) ? T(1) : T(0);
}

template <typename T>
cudaError_t launch_set_identity(T* base, const i64* qoff, const i64* dims, int nboxes, cudaStream_t st) {
  if (nboxes == 0) return cudaSuccess;
  k_set_identity<T><<<nboxes, 256, 0, st>>>(base, qoff, dims);
  return cudaGetLastError();
}
template cudaError_t launch_set_identity<double>(double*, const i64*, const i64*, int, cudaStream_t);
template cudaError_t launch_set_identity<float>(float*, const i64*, const i64*, int, cudaStream_t);

}  // namespace h2b
