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

// Register-resident Gauss-Jordan for n <= NP (NP = 128 with 256 threads,
// FP32 NP = 256 with 1024 threads; the block is padded with the identity):
// warp w owns columns w + W j (j < CPW = NP / W), lane l owns rows l + 32 i
// (i < RPL = NP / 32), so each thread holds 64 values and a step costs two
// barriers (pivot column to shared memory, pivot index back) instead of a
// block-wide sweep through memory.  Row swaps and the pivot row travel by
// warp shuffles; pivot order, ipiv, the determinant rule and the column
// unscrambling are those of k_gj_inverse.
template <typename T, int NP>
__global__ void __launch_bounds__(NP * NP / 64) k_gj_reg(const LuTask<T>* __restrict__ tasks) {
  constexpr int NT = NP * NP / 64, W = NT / 32, CPW = NP / W, RPL = NP / 32;
  const LuTask<T> t = tasks[blockIdx.x];
  const int n = t.n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ T colk[2][NP];
  __shared__ int s_piv[NP];
  __shared__ int s_pos[NP];
  __shared__ int s_p;
  __shared__ double s_det;
  __shared__ int s_swaps;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* stage = reinterpret_cast<T*>(smem_raw);  // 32 x (NP + 1) output staging
  if (n <= 0) {
    if (tid == 0) *t.info = 0;
    return;
  }
  T x[CPW][RPL];
#pragma unroll
  for (int j = 0; j < CPW; j++) {
    const int c = warp + W * j;
#pragma unroll
    for (int i = 0; i < RPL; i++) {
      const int r = lane + 32 * i;
      x[j][i] = (r < n && c < n) ? t.A[r + (i64)c * t.lda] : (r == c ? T(1) : T(0));
    }
  }
  if (tid == 0) {
    s_det = 1.;
    s_swaps = 0;
  }
  for (int k = 0; k < n; k++) {
    const int wk = k % W, jk = k / W, lk = k & 31, ik = k >> 5;
    T* ck = colk[k & 1];
    // 1. The owner warp publishes column k.
    if (warp == wk) {
#pragma unroll
      for (int j = 0; j < CPW; j++)
        if (j == jk)
#pragma unroll
          for (int i = 0; i < RPL; i++) ck[lane + 32 * i] = x[j][i];
    }
    __syncthreads();
    // 2. Warp 0 finds the pivot: first row of largest magnitude, rows k..n-1.
    if (warp == 0) {
      double bv = -1.;
      int bi = 0x7fffffff;
      for (int r = k + lane; r < n; r += 32) {
        const double v = fabs((double)ck[r]);
        if (v > bv) { bv = v; bi = r; }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if (bi < k || bi >= n) bi = k;  // a column of NaNs: no swap
      if (lane == 0) {
        s_p = bi;
        s_piv[k] = bi;
        s_det *= (double)ck[bi];
        s_swaps += bi != k;
      }
    }
    __syncthreads();
    const int p = s_p, lp = p & 31, ip = p >> 5;
    const T piv = ck[p];
    const T inv = piv != T(0) ? T(1) / piv : T(0);
    // 3. Swap rows k and p of every owned column, then scale row k and
    //    broadcast it within the warp.
    T rowk[CPW];
#pragma unroll
    for (int j = 0; j < CPW; j++) {
      T vk = x[j][0], vp = x[j][0];
#pragma unroll
      for (int i = 1; i < RPL; i++) {
        if (i == ik) vk = x[j][i];
        if (i == ip) vp = x[j][i];
      }
      const T a_k = __shfl_sync(0xffffffffu, vk, lk);  // old row k
      const T a_p = __shfl_sync(0xffffffffu, vp, lp);  // old row p (new row k)
      const int c = warp + W * j;
      if (p != k) {
#pragma unroll
        for (int i = 0; i < RPL; i++) {
          if (i == ip && lane == lp) x[j][i] = a_k;
        }
      }
      const T nk = (c == k ? T(1) : a_p) * inv;  // new row k, scaled
#pragma unroll
      for (int i = 0; i < RPL; i++)
        if (i == ik && lane == lk) x[j][i] = nk;
      rowk[j] = nk;
    }
    // 4. Eliminate column k from every other row (multipliers from the
    //    published column, with rows k and p exchanged).
#pragma unroll
    for (int i = 0; i < RPL; i++) {
      const int r = lane + 32 * i;
      if (r == k) continue;
      const T m = r == p ? ck[k] : ck[r];
#pragma unroll
      for (int j = 0; j < CPW; j++) {
        const int c = warp + W * j;
        x[j][i] = (c == k ? T(0) : x[j][i]) - m * rowk[j];
      }
    }
  }
  __syncthreads();
  // Unscramble: position q of the inverse holds elimination column idx[q]
  // after the swaps (k, piv[k]) for k = n-1..0; s_pos[c] = position of c.
  if (tid == 0) {
    int* idx = s_pos;  // reused below as the inverse map
    for (int c = 0; c < NP; c++) idx[c] = c;
    for (int k = n - 1; k >= 0; k--) {
      const int q = s_piv[k];
      const int tmp = idx[k]; idx[k] = idx[q]; idx[q] = tmp;
    }
    // Invert idx in place through colk (free now) as scratch.
    int* inv_map = reinterpret_cast<int*>(colk);
    for (int q = 0; q < NP; q++) inv_map[idx[q]] = q;
    for (int c = 0; c < NP; c++) s_pos[c] = inv_map[c];
    const double det = (s_swaps & 1) ? -s_det : s_det;
    *t.info = fabs(det) <= DBL_MIN ? 1 : 0;
  }
  __syncthreads();
  for (int k = tid; k < n; k += NT) t.ipiv[k] = s_piv[k];
  // invT[r * ldinv + q] = A^{-1}[r][q], 32 rows at a time through shared
  // memory so the global stores run along q.
#pragma unroll
  for (int i = 0; i < RPL; i++) {
    if (32 * i >= n) break;
#pragma unroll
    for (int j = 0; j < CPW; j++) {
      const int c = warp + W * j;
      if (c < n) stage[lane * (NP + 1) + s_pos[c]] = x[j][i];
    }
    __syncthreads();
    for (int e = tid; e < 32 * NP; e += NT) {
      const int rr = e / NP, q = e % NP, r = 32 * i + rr;
      if (r < n && q < n) t.invT[(i64)r * t.ldinv + q] = stage[rr * (NP + 1) + q];
    }
    __syncthreads();
  }
}

// LU with partial pivoting of A_rr and the solve A_rr V_r = U_r^T
// (h2matrix.cpp:377-379: PartialPivLU, then solve).  One CTA per box.
// Factorization: the right-looking partial-pivot LU (pivot = first row of
// largest magnitude in column k among rows k..n-1; the column below the
// pivot divided by it; rank-1 update of the trailing block), unblocked in
// shared memory when the block fits, otherwise in the task's global scratch
// (FP32: blocked by panels of LU_NB columns, the trailing update as a tiled
// product).
// Solve: the row interchanges applied to the right-hand sides, then the
// unit-lower forward and the upper backward substitution, one warp per 32
// right-hand-side columns (lane = column), 32 rows at a time in registers,
// left-looking across row blocks (each earlier row block read back once).
// Right-hand sides and solution have row r contiguous over the columns
// (B[c + r ldb]), as U_r^T and V_r are laid out in the ULV.  info follows
// Eigen's determinant rule (product of U's diagonal, sign of the
// permutation, |det| <= DBL_MIN).
constexpr int LU_NB = 32;  // panel width of the blocked LU in global scratch
// Byte offset of the trailing-update tiles in the global variant's dynamic
// shared memory (after the pivot arrays, 16-byte aligned).
__host__ __device__ constexpr size_t lu_tile_offset(int n) { return ((2 * sizeof(int) * (size_t)n + 15) / 16) * 16; }
template <typename T>
constexpr size_t lu_tile_bytes() {
  return sizeof(T) * (size_t)(64 * (LU_NB + 1) + LU_NB * 65);
}

template <typename T, bool SMEM>
__global__ void __launch_bounds__(256, 2) k_lu_solve(const LuSolveTask<T>* __restrict__ tasks) {
  const LuSolveTask<T> t = tasks[blockIdx.x];
  const int n = t.n, m = t.m;
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
  const i64 ld = SMEM ? n + 1 : n;
  T* a = SMEM ? reinterpret_cast<T*>(smem_raw) : t.work;
  int* piv = SMEM ? reinterpret_cast<int*>(a + (size_t)n * ld) : reinterpret_cast<int*>(smem_raw);
  int* prow = piv + n;  // row of the right-hand sides that lands in row i of P B
  for (int c = warp; c < n; c += nw)
    for (int r = lane; r < n; r += 32) a[r + (i64)c * ld] = t.A[r + (i64)c * t.lda];
  if (!SMEM) __threadfence_block();
  if (tid == 0) {
    s_det = 1.;
    s_swaps = 0;
  }
  __syncthreads();
  // One pivot step of the partial-pivot LU: pivot search in column k among
  // rows k..n-1, row interchange over all n columns, the column below the
  // pivot divided by it, and the rank-1 update of columns k+1 .. c_end-1.
  auto pivot_step = [&](int k, int c_end) {
    double bv = -1.;
    int bi = 0x7fffffff;
    for (int r = k + tid; r < n; r += nt) {
      const double v = fabs((double)a[r + (i64)k * ld]);
      if (v > bv) { bv = v; bi = r; }
    }
    argmax_first(bv, bi, red_v, red_i);
    if (bi < k || bi >= n) bi = k;  // a column of NaNs: no swap
    if (bi != k)
      for (int c = tid; c < n; c += nt) {
        const T x = a[k + (i64)c * ld];
        a[k + (i64)c * ld] = a[bi + (i64)c * ld];
        a[bi + (i64)c * ld] = x;
      }
    if (!SMEM) __threadfence_block();
    __syncthreads();
    const T p = a[k + (i64)k * ld];
    if (tid == 0) {
      piv[k] = bi;
      s_det *= (double)p;
      s_swaps += bi != k;
    }
    if (p != T(0))
      for (int r = k + 1 + tid; r < n; r += nt) a[r + (i64)k * ld] = a[r + (i64)k * ld] / p;
    if (!SMEM) __threadfence_block();
    __syncthreads();
    for (int c = k + 1 + warp; c < c_end; c += nw) {
      T* ac = a + (i64)c * ld;
      const T akc = ac[k];
      for (int r = k + 1 + lane; r < n; r += 32) ac[r] -= a[r + (i64)k * ld] * akc;
    }
    if (!SMEM) __threadfence_block();
    __syncthreads();
  };
  if constexpr (SMEM || sizeof(T) == 8) {
    // FP64 keeps the unblocked order in global scratch too: it is the path
    // held to the oracle on the ill-conditioned reference configuration,
    // whose substitution moves by tens of percent with the rounding order.
    for (int k = 0; k < n; k++) pivot_step(k, n);
  } else {
    // FP32 (the mixed preconditioner) in global scratch: blocked
    // right-looking LU (panels of LU_NB columns, the same pivots as the
    // unblocked form up to rounding), so the trailing matrix is read and
    // written once per panel instead of once per pivot.
    // The trailing update runs in 64 x 64 tiles with the panel's L rows and
    // U columns staged in shared memory after the pivot arrays.
    T* Ls = reinterpret_cast<T*>(smem_raw + lu_tile_offset(n));  // [64][LU_NB + 1]
    T* Us = Ls + 64 * (LU_NB + 1);                               // [LU_NB][65]
    const int tx = tid & 15, ty = tid >> 4;                      // 4 x 4 outputs per thread
    for (int k0 = 0; k0 < n; k0 += LU_NB) {
      const int kb = min(LU_NB, n - k0), j0 = k0 + kb;
      for (int k = k0; k < j0; k++) pivot_step(k, j0);
      if (j0 >= n) break;
      // U12 = L11^-1 A12 (L11 unit lower), one column per thread
      for (int c = j0 + tid; c < n; c += nt) {
        T* ac = a + (i64)c * ld;
        for (int i = 0; i < kb; i++) {
          const T x = ac[k0 + i];
          for (int r = i + 1; r < kb; r++) ac[k0 + r] -= a[(k0 + r) + (i64)(k0 + i) * ld] * x;
        }
      }
      __threadfence_block();
      __syncthreads();
      // A22 -= L21 U12
      for (int tr = j0; tr < n; tr += 64)
        for (int tc = j0; tc < n; tc += 64) {
          for (int e = tid; e < 64 * LU_NB; e += nt) {
            const int rr = e % 64, i = e / 64;
            Ls[rr * (LU_NB + 1) + i] = (tr + rr < n && i < kb) ? a[(tr + rr) + (i64)(k0 + i) * ld] : T(0);
          }
          for (int e = tid; e < 64 * LU_NB; e += nt) {
            const int i = e % LU_NB, cc = e / LU_NB;
            Us[i * 65 + cc] = (tc + cc < n && i < kb) ? a[(k0 + i) + (i64)(tc + cc) * ld] : T(0);
          }
          __syncthreads();
          T acc[4][4];
#pragma unroll
          for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) acc[u][v] = T(0);
          for (int i = 0; i < kb; i++) {
            T lv[4], uv[4];
#pragma unroll
            for (int u = 0; u < 4; u++) lv[u] = Ls[(ty * 4 + u) * (LU_NB + 1) + i];
#pragma unroll
            for (int v = 0; v < 4; v++) uv[v] = Us[i * 65 + tx * 4 + v];
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
              for (int v = 0; v < 4; v++) acc[u][v] += lv[u] * uv[v];
          }
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int r = tr + ty * 4 + u;
            if (r >= n) continue;
#pragma unroll
            for (int v = 0; v < 4; v++) {
              const int c = tc + tx * 4 + v;
              if (c < n) a[r + (i64)c * ld] -= acc[u][v];
            }
          }
          __syncthreads();  // the tiles are restaged by the next (tr, tc)
        }
      __threadfence_block();
      __syncthreads();
    }
  }
  if (tid == 0) {
    for (int i = 0; i < n; i++) prow[i] = i;
    for (int k = 0; k < n; k++) {
      const int q = piv[k];
      const int x = prow[k];
      prow[k] = prow[q];
      prow[q] = x;
    }
    const double det = (s_swaps & 1) ? -s_det : s_det;
    *t.info = fabs(det) <= DBL_MIN ? 1 : 0;
  }
  for (int k = tid; k < n; k += nt) t.ipiv[k] = piv[k];
  __syncthreads();

  for (int c0 = warp * 32; c0 < m; c0 += nw * 32) {
    const int c = c0 + lane;
    const bool cv = c < m;
    // Forward: L y = P b, L unit lower.
    for (int b0 = 0; b0 < n; b0 += 32) {
      T r[32];
#pragma unroll
      for (int i = 0; i < 32; i++) r[i] = (cv && b0 + i < n) ? t.B[c + (i64)prow[b0 + i] * t.ldb] : T(0);
      for (int j = 0; j < b0; j++) {
        const T xj = cv ? t.X[c + (i64)j * t.ldx] : T(0);
#pragma unroll
        for (int i = 0; i < 32; i++)
          if (b0 + i < n) r[i] -= a[(b0 + i) + (i64)j * ld] * xj;
      }
#pragma unroll
      for (int jj = 0; jj < 32; jj++) {
        if (b0 + jj < n) {
#pragma unroll
          for (int i = jj + 1; i < 32; i++)
            if (b0 + i < n) r[i] -= a[(b0 + i) + (i64)(b0 + jj) * ld] * r[jj];
        }
      }
#pragma unroll
      for (int i = 0; i < 32; i++)
        if (cv && b0 + i < n) t.X[c + (i64)(b0 + i) * t.ldx] = r[i];
    }
    // Backward: U x = y.
    for (int b0 = ((n - 1) / 32) * 32; b0 >= 0; b0 -= 32) {
      T r[32];
#pragma unroll
      for (int i = 0; i < 32; i++) r[i] = (cv && b0 + i < n) ? t.X[c + (i64)(b0 + i) * t.ldx] : T(0);
      for (int j = b0 + 32; j < n; j++) {
        const T xj = cv ? t.X[c + (i64)j * t.ldx] : T(0);
#pragma unroll
        for (int i = 0; i < 32; i++) r[i] -= a[(b0 + i) + (i64)j * ld] * xj;
      }
#pragma unroll
      for (int jj = 31; jj >= 0; jj--) {
        if (b0 + jj < n) {
          r[jj] = r[jj] / a[(b0 + jj) + (i64)(b0 + jj) * ld];
#pragma unroll
          for (int i = 0; i < jj; i++) r[i] -= a[(b0 + i) + (i64)(b0 + jj) * ld] * r[jj];
        }
      }
#pragma unroll
      for (int i = 0; i < 32; i++)
        if (cv && b0 + i < n) t.X[c + (i64)(b0 + i) * t.ldx] = r[i];
    }
  }
}

template <typename T>
size_t lu_solve_smem(int n) {
  return sizeof(T) * (size_t)n * (n + 1) + 2 * sizeof(int) * (size_t)n + 16;
}

template <typename T>
cudaError_t launch_lu_solve(const LuSolveTask<T>* d_tasks, int ntasks, int maxn, cudaStream_t st) {
  if (ntasks == 0) return cudaSuccess;
  if (lu_solve_smem<T>(maxn) <= 200 * 1024) {
    const size_t smem = lu_solve_smem<T>(maxn);
    cudaError_t e = cudaFuncSetAttribute(k_lu_solve<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    note_launch();
    k_lu_solve<T, true><<<ntasks, 256, smem, st>>>(d_tasks);
    return cudaGetLastError();
  }
  const size_t smem = lu_tile_offset(maxn) + lu_tile_bytes<T>() + 16;
  cudaError_t e = cudaFuncSetAttribute(k_lu_solve<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  note_launch();
  k_lu_solve<T, false><<<ntasks, 256, smem, st>>>(d_tasks);
  return cudaGetLastError();
}
template cudaError_t launch_lu_solve<double>(const LuSolveTask<double>*, int, int, cudaStream_t);
template cudaError_t launch_lu_solve<float>(const LuSolveTask<float>*, int, int, cudaStream_t);

template <typename T>
size_t gj_smem(int n) {
  return sizeof(T) * ((size_t)n * (n + 1) + n) + sizeof(int) * (size_t)n + 16;
}

template <typename T>
cudaError_t launch_lu_inverse(const LuTask<T>* d_tasks, int ntasks, int maxn, cudaStream_t st) {
  if (ntasks == 0) return cudaSuccess;
  if (maxn <= (sizeof(T) == 4 ? 256 : 128)) {
    auto go = [&](auto kern, int np) {
      const size_t smem = sizeof(T) * 32 * (size_t)(np + 1);
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      note_launch();
      kern<<<ntasks, np * np / 64, smem, st>>>(d_tasks);
      return cudaGetLastError();
    };
    if (maxn <= 128) return go(k_gj_reg<T, 128>, 128);
    if constexpr (sizeof(T) == 4) return go(k_gj_reg<float, 256>, 256);
  }
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
