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

namespace h2b {

// Multi-right-hand-side block-sparse apply: C_task (m x n, n <= NR) =
// beta C + sum_e alpha_e A_e B_e with A_e and B_e as stored (column-major).
// This is the shape of every H^2 matvec pass and every ULV substitution
// step except the transposed ones.  A is read once, straight from HBM into
// registers (consecutive threads own consecutive rows, so each k column is
// one coalesced row of loads, eight columns in flight per thread); B chunks
// of KC rows are staged in shared memory and read as broadcasts; all NR
// columns accumulate in registers.  One CTA covers NT*TM rows of one task.
template <typename T, int NR, int TM, int NT, int U>
__global__ void __launch_bounds__(NT) k_skinny_nn(const GemmTask<T>* __restrict__ tasks,
                                                  const GemmEntry<T>* __restrict__ ents,
                                                  const int2* __restrict__ tiles) {
  constexpr int BM = NT * TM, KC = 128;
  __shared__ __align__(16) T Bs[KC][NR];
  const int2 tl = tiles[blockIdx.x];
  const GemmTask<T> task = tasks[tl.x];
  const int m0 = tl.y * BM;
  const int tid = threadIdx.x;
  T acc[TM][NR];
#pragma unroll
  for (int t = 0; t < TM; t++)
#pragma unroll
    for (int j = 0; j < NR; j++) acc[t][j] = T(0);
  bool rv[TM];
#pragma unroll
  for (int t = 0; t < TM; t++) rv[t] = (m0 + tid + t * NT) < task.m;

  for (int e = task.e0; e < task.e1; e++) {
    const GemmEntry<T> en = ents[e];
    const int K = en.k;
    const T* Ab = en.A + (m0 + tid);
    for (int k0 = 0; k0 < K; k0 += KC) {
      const int kc = (K - k0) < KC ? (K - k0) : KC;
      for (int idx = tid; idx < KC * NR; idx += NT) {
        int kk = idx % KC, j = idx / KC;
        Bs[kk][j] = (kk < kc && j < task.n) ? en.B[(i64)(k0 + kk) + (i64)j * en.ldb] : T(0);
      }
      __syncthreads();
      // Two register batches of U columns of A: the loads of the next batch
      // are in flight while the current one is multiplied.
      T a0[U][TM], a1[U][TM];
#pragma unroll
      for (int u = 0; u < U; u++)
#pragma unroll
        for (int t = 0; t < TM; t++)
          a0[u][t] = (u < kc && rv[t]) ? en.alpha * Ab[(i64)(k0 + u) * en.lda + t * NT] : T(0);
      for (int kb = 0; kb < kc; kb += 2 * U) {
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
          for (int t = 0; t < TM; t++)
            a1[u][t] = (kb + U + u < kc && rv[t]) ? en.alpha * Ab[(i64)(k0 + kb + U + u) * en.lda + t * NT] : T(0);
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
          for (int j = 0; j < NR; j++) {
            const T bj = Bs[kb + u][j];
#pragma unroll
            for (int t = 0; t < TM; t++) acc[t][j] += a0[u][t] * bj;
          }
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
          for (int t = 0; t < TM; t++)
            a0[u][t] = (kb + 2 * U + u < kc && rv[t]) ? en.alpha * Ab[(i64)(k0 + kb + 2 * U + u) * en.lda + t * NT]
                                                       : T(0);
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
          for (int j = 0; j < NR; j++) {
            const T bj = Bs[(kb + U + u) < KC ? kb + U + u : KC - 1][j];
#pragma unroll
            for (int t = 0; t < TM; t++) acc[t][j] += a1[u][t] * bj;
          }
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int t = 0; t < TM; t++) {
    if (!rv[t]) continue;
    const int r = m0 + tid + t * NT;
#pragma unroll
    for (int j = 0; j < NR; j++) {
      if (j >= task.n) break;
      T* p = task.C + r + (i64)j * task.ldc;
      *p = (task.beta == T(0)) ? acc[t][j] : task.beta * (*p) + acc[t][j];
    }
  }
}

// dst = beta * dst + sum_{p < parts} src_p, the parts of one split task
// summed in a fixed order (deterministic).
template <typename T>
__global__ void __launch_bounds__(256) k_sum_parts(const SumTask<T>* __restrict__ tasks) {
  const SumTask<T> t = tasks[blockIdx.x];
  const i64 mn = (i64)t.m * t.n;
  for (i64 e = threadIdx.x; e < mn; e += blockDim.x) {
    const int r = (int)(e % t.m), c = (int)(e / t.m);
    T s = T(0);
    for (int p = 0; p < t.parts; p++) s += t.src[(i64)p * mn + e];
    T* d = t.dst + r + (i64)c * t.ldd;
    *d = (t.beta == T(0)) ? s : t.beta * (*d) + s;
  }
}

template <typename T>
cudaError_t launch_sum_parts(const SumTask<T>* d_tasks, int ntasks, cudaStream_t st) {
  if (ntasks == 0) return cudaSuccess;
  k_sum_parts<T><<<ntasks, 256, 0, st>>>(d_tasks);
  return cudaGetLastError();
}
template cudaError_t launch_sum_parts<double>(const SumTask<double>*, int, cudaStream_t);
template cudaError_t launch_sum_parts<float>(const SumTask<float>*, int, cudaStream_t);

}  // namespace h2b

namespace h2b {

int skinny_rows_per_cta() { return 256; }

template <typename T>
cudaError_t launch_skinny_nn(int nr, const GemmTask<T>* d_tasks, const GemmEntry<T>* d_ents, const int2* d_tiles,
                             int ntiles, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  // Every variant covers 256 rows per CTA: 2 rows per thread, deep load
  // batches (HBM-latency bound).
  if (nr <= 1)
    k_skinny_nn<T, 1, 2, 128, 8><<<ntiles, 128, 0, st>>>(d_tasks, d_ents, d_tiles);
  else if (nr <= 2)
    k_skinny_nn<T, 2, 2, 128, 8><<<ntiles, 128, 0, st>>>(d_tasks, d_ents, d_tiles);
  else if (nr <= 4)
    k_skinny_nn<T, 4, 2, 128, 8><<<ntiles, 128, 0, st>>>(d_tasks, d_ents, d_tiles);
  else if (nr <= 8)
    k_skinny_nn<T, 8, 2, 128, 8><<<ntiles, 128, 0, st>>>(d_tasks, d_ents, d_tiles);
  else if (nr <= 16)
    k_skinny_nn<T, 16, 2, 128, 8><<<ntiles, 128, 0, st>>>(d_tasks, d_ents, d_tiles);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}
template cudaError_t launch_skinny_nn<double>(int, const GemmTask<double>*, const GemmEntry<double>*, const int2*, int,
                                              cudaStream_t);
template cudaError_t launch_skinny_nn<float>(int, const GemmTask<float>*, const GemmEntry<float>*, const int2*, int,
                                             cudaStream_t);

}  // namespace h2b
