// Batched LU with partial pivoting of the redundant diagonal block A_rr and
// its explicit inverse (h2matrix.cpp:375-379, 399-400: the ULV needs both
// A_rr^{-1} U_r^T and A_rr^{-1} itself).  One CTA per box; the block is
// small enough to stay in L2 while the CTA works on it.
#include "common.cuh"
#include "kernels.h"

#include <cfloat>

namespace h2b {

template <typename T>
__global__ void __launch_bounds__(256) k_lu_inverse(const LuTask<T>* __restrict__ tasks) {
  const LuTask<T> t = tasks[blockIdx.x];
  const int n = t.n;
  const int tid = threadIdx.x, nt = blockDim.x;
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  if (n <= 0) {
    if (tid == 0) *t.info = 0;
    return;
  }
  T* A = t.A;
  const i64 lda = t.lda;
  for (int k = 0; k < n; k++) {
    // Pivot: first row with the largest magnitude in column k.
    double bv = -1.;
    int bi = 0x7fffffff;
    for (int r = k + tid; r < n; r += nt) {
      double v = fabs((double)A[r + (i64)k * lda]);
      if (v > bv) { bv = v; bi = r; }
    }
    argmax_first(bv, bi, red_v, red_i);
    // A column of NaNs gives no maximum: keep row k rather than swap with a
    // row outside the block.
    if (bi < k || bi >= n) bi = k;
    if (tid == 0) t.ipiv[k] = bi;
    if (bi != k)
      for (int c = tid; c < n; c += nt) {
        T x = A[k + (i64)c * lda];
        A[k + (i64)c * lda] = A[bi + (i64)c * lda];
        A[bi + (i64)c * lda] = x;
      }
    __syncthreads();
    const T piv = A[k + (i64)k * lda];
    if (piv != T(0))
      for (int r = k + 1 + tid; r < n; r += nt) A[r + (i64)k * lda] /= piv;
    __syncthreads();
    const int rem = n - k - 1;
    const i64 tot = (i64)rem * rem;
    for (i64 e = tid; e < tot; e += nt) {
      int r = k + 1 + (int)(e % rem), c = k + 1 + (int)(e / rem);
      A[r + (i64)c * lda] -= A[r + (i64)k * lda] * A[k + (i64)c * lda];
    }
    __syncthreads();
  }
  if (tid == 0) {
    // Eigen's determinant: product of U's diagonal times the permutation sign.
    double det = 1.;
    int swaps = 0;
    for (int k = 0; k < n; k++) {
      det *= (double)A[k + (i64)k * lda];
      swaps += t.ipiv[k] != k;
    }
    if (swaps & 1) det = -det;
    *t.info = fabs(det) <= DBL_MIN ? 1 : 0;
  }
  // Row permutation p: row k of P A is row p[k] of A.
  extern __shared__ int perm[];
  if (tid == 0) {
    for (int k = 0; k < n; k++) perm[k] = k;
    for (int k = 0; k < n; k++) {
      int q = t.ipiv[k];
      int x = perm[k]; perm[k] = perm[q]; perm[q] = x;
    }
  }
  __syncthreads();
  // Solve L U X = P I column by column; X is stored row-major (X[r][c] at
  // invT[r * ldinv + c]), i.e. invT holds (A^{-1})^T column-major.
  T* X = t.invT;
  const i64 ldx = t.ldinv;
  for (int c = tid; c < n; c += nt) {
    for (int r = 0; r < n; r++) {
      T s = (perm[r] == c) ? T(1) : T(0);
      for (int k = 0; k < r; k++) s -= A[r + (i64)k * lda] * X[(i64)k * ldx + c];
      X[(i64)r * ldx + c] = s;
    }
    for (int r = n - 1; r >= 0; r--) {
      T s = X[(i64)r * ldx + c];
      for (int k = r + 1; k < n; k++) s -= A[r + (i64)k * lda] * X[(i64)k * ldx + c];
      X[(i64)r * ldx + c] = s / A[r + (i64)r * lda];
    }
  }
}

template <typename T>
cudaError_t launch_lu_inverse(const LuTask<T>* d_tasks, int ntasks, cudaStream_t st) {
  if (ntasks == 0) return cudaSuccess;
  // Largest n is bounded by the caller (box dims <= 4096).
  note_launch();
  k_lu_inverse<T><<<ntasks, 256, 4096 * sizeof(int), st>>>(d_tasks);
  return cudaGetLastError();
}
template cudaError_t launch_lu_inverse<double>(const LuTask<double>*, int, cudaStream_t);
template cudaError_t launch_lu_inverse<float>(const LuTask<float>*, int, cudaStream_t);

}  // namespace h2b
