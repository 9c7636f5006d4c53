// Batched inverse of the redundant diagonal block A_rr with partial
// pivoting (h2matrix.cpp:375-379, 399-400: the ULV needs A_rr^{-1} U_r^T and
// A_rr^{-1} itself, and Eigen's PartialPivLU determinant for info).  One CTA
// per box: Gauss-Jordan elimination in shared memory when the block fits,
// otherwise in place in the (L2-resident) output.
#include "common.cuh"
#include "kernels.h"

#include <cfloat>

namespace h2b {

// Gauss-Jordan elimination with the partial pivoting of an LU (first row of
// largest magnitude in column k among rows k..n-1), so the pivots, ipiv and
// the determinant rule for info are those of PartialPivLU; the inverse's
// columns are unscrambled in reverse pivot order at the end.  A_rr itself is
// read, not overwritten (the ULV uses only its inverse).  Each step is one
// barrier-separated rank-1 update of the whole block by the CTA.
template <typename T, bool SMEM>
__global__ void __launch_bounds__(256) k_gj_inverse(const LuTask<T>* __restrict__ tasks) {
  const LuTask<T> t = tasks[blockIdx.x];
  const int n = t.n;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ double s_det;
  __shared__ int s_swaps;
  if (n <= 0) {
    if (tid == 0) *t.info = 0;
    return;
  }
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // The working block: in shared memory (padded leading dimension, so
  // row-wise sweeps are conflict-free) or, when it does not fit, in place in
  // the invT output (L2-resident), transposed at the end.
  const i64 ld = SMEM ? n + 1 : t.ldinv;
  T* a = SMEM ? reinterpret_cast<T*>(smem_raw) : t.invT;
  T* col = SMEM ? a + (size_t)n * ld : reinterpret_cast<T*>(smem_raw);  // column k before the update
  int* piv = reinterpret_cast<int*>(col + n);
  for (int c = warp; c < n; c += nw)
    for (int r = lane; r < n; r += 32) a[r + (i64)c * ld] = t.A[r + (i64)c * t.lda];
  if (!SMEM) __threadfence_block();
  if (tid == 0) {
    s_det = 1.;
    s_swaps = 0;
  }
  __syncthreads();
  for (int k = 0; k < n; k++) {
    double bv = -1.;
    int bi = 0x7fffffff;
    for (int r = k + tid; r < n; r += nt) {
      double v = fabs((double)a[r + (i64)k * ld]);
      if (v > bv) { bv = v; bi = r; }
    }
    argmax_first(bv, bi, red_v, red_i);
    if (bi < k || bi >= n) bi = k;  // a column of NaNs: no swap
    if (bi != k)
      for (int c = tid; c < n; c += nt) {
        T x = a[k + (i64)c * ld];
        a[k + (i64)c * ld] = a[bi + (i64)c * ld];
        a[bi + (i64)c * ld] = x;
      }
    __syncthreads();
    const T p = a[k + (i64)k * ld];
    if (tid == 0) {
      piv[k] = bi;
      s_det *= (double)p;
      s_swaps += bi != k;
    }
    const T inv = p != T(0) ? T(1) / p : T(0);
    for (int r = tid; r < n; r += nt) col[r] = r == k ? T(0) : a[r + (i64)k * ld];
    __syncthreads();
    for (int c = tid; c < n; c += nt) a[k + (i64)c * ld] = (c == k ? T(1) : a[k + (i64)c * ld]) * inv;
    __syncthreads();
    // Rank-1 update, one warp per column (no index division).
    for (int c = warp; c < n; c += nw) {
      T* ac = a + (i64)c * ld;
      const T akc = ac[k];
      for (int r = lane; r < n; r += 32) {
        if (r == k) continue;
        ac[r] = (c == k ? T(0) : ac[r]) - col[r] * akc;
      }
    }
    __syncthreads();
  }
  // Unscramble: the row swaps of the elimination become column swaps of the
  // inverse, applied in reverse order.
  for (int k = n - 1; k >= 0; k--) {
    const int q = piv[k];
    if (q != k)
      for (int r = tid; r < n; r += nt) {
        T x = a[r + (i64)k * ld];
        a[r + (i64)k * ld] = a[r + (i64)q * ld];
        a[r + (i64)q * ld] = x;
      }
    __syncthreads();
  }
  // invT holds (A^{-1})^T column-major: invT[r * ldinv + c] = A^{-1}[r][c].
  if (SMEM) {
    for (int r = warp; r < n; r += nw)
      for (int c = lane; c < n; c += 32) t.invT[(i64)r * t.ldinv + c] = a[r + (size_t)c * ld];
  } else {
    for (int c = warp; c < n; c += nw)
      for (int r = lane; r < c; r += 32) {
        T x = a[r + (i64)c * ld];
        a[r + (i64)c * ld] = a[c + (i64)r * ld];
        a[c + (i64)r * ld] = x;
      }
  }
  for (int k = tid; k < n; k += nt) t.ipiv[k] = piv[k];
  if (tid == 0) {
    // Eigen's determinant: product of U's diagonal times the permutation sign.
    const double det = (s_swaps & 1) ? -s_det : s_det;
    *t.info = fabs(det) <= DBL_MIN ? 1 : 0;
  }
}

template <typename T>
size_t gj_smem(int n) {
  return sizeof(T) * ((size_t)n * (n + 1) + n) + sizeof(int) * (size_t)n + 16;
}

template <typename T>
cudaError_t launch_lu_inverse(const LuTask<T>* d_tasks, int ntasks, int maxn, cudaStream_t st) {
  if (ntasks == 0) return cudaSuccess;
  if (gj_smem<T>(maxn) <= 200 * 1024) {
    const size_t smem = gj_smem<T>(maxn);
    cudaError_t e = cudaFuncSetAttribute(k_gj_inverse<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    note_launch();
    k_gj_inverse<T, true><<<ntasks, 256, smem, st>>>(d_tasks);
    return cudaGetLastError();
  }
  // Larger blocks (box dims <= 4096): the same elimination in place in the
  // output, with the pivot column and pivots in shared memory.
  const size_t smem = (sizeof(T) + sizeof(int)) * (size_t)maxn + 16;
  cudaError_t e = cudaFuncSetAttribute(k_gj_inverse<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  note_launch();
  k_gj_inverse<T, false><<<ntasks, 256, smem, st>>>(d_tasks);
  return cudaGetLastError();
}
template cudaError_t launch_lu_inverse<double>(const LuTask<double>*, int, int, cudaStream_t);
template cudaError_t launch_lu_inverse<float>(const LuTask<float>*, int, int, cudaStream_t);

}  // namespace h2b
