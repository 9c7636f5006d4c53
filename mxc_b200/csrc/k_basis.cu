// Shared-basis compression kernels (compute_basis, h2matrix.cpp:13-63).
//
// One CTA per box of a tree level.  Step 1 (k_sample_tsqr) forms the R
// factor of the far-field sample block XF = K(far samples, box bodies)
// without materialising XF: sample rows are generated 32 at a time into
// shared memory and folded into R with Householder reflectors on
// (row j of R, tile column j).  Step 2 (k_cpqr) runs the column-pivoted
// Householder QR of R with Eigen 3.4's ColPivHouseholderQR pivot, norm
// downdate and rank rules.  Step 3 (k_basis_finish) forms the interpolative
// decomposition [I, R11^-1 R12], permutes the box bodies skeleton-first and
// builds either the ID basis (operator mode) or the orthogonal basis with
// completion plus the triangular R (preconditioner mode).
#include "common.cuh"
#include "kernels.h"

#include <algorithm>
#include <cfloat>

namespace h2b {

template <typename T> struct Tiny;
template <> struct Tiny<double> { static __device__ double v() { return DBL_MIN; } };
template <> struct Tiny<float> { static __device__ float v() { return FLT_MIN; } };

constexpr int TS_THREADS = 256;
constexpr int TS_MAXCOL = 8;  // columns owned per thread: M <= 2048

// R (row-major M x M per box, zero on entry) of the sample block.  TR
// sample rows per tile (32, or 16 / 8 for wide boxes so the tile fits in
// shared memory); lane r of the reflector warp holds tile row r.
template <typename T, int TR>
__global__ void __launch_bounds__(TS_THREADS) k_sample_tsqr(
    KernelParams kp, const double* __restrict__ bodies, const double* __restrict__ pts,
    const i64* __restrict__ xoff, const i64* __restrict__ dims, const int* __restrict__ sidx,
    const i64* __restrict__ soff, T* __restrict__ Rws, const i64* __restrict__ qoff) {
  const int box = blockIdx.x;
  const int M = (int)dims[box];
  const i64 S = soff[box + 1] - soff[box];
  if (M == 0 || S == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);            // 32 x M, row-major
  T* vbuf = tile + TR * M;                             // 32
  double* sp = reinterpret_cast<double*>(vbuf + 32);   // 32 x 3
  __shared__ T s_tau;

  T* R = Rws + qoff[box];
  const int* my_sidx = sidx + soff[box];
  const double* bp = pts + 3 * xoff[box];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  double px[TS_MAXCOL], py[TS_MAXCOL], pz[TS_MAXCOL];
#pragma unroll
  for (int k = 0; k < TS_MAXCOL; k++) {
    int c = tid + k * TS_THREADS;
    px[k] = c < M ? bp[3 * c] : 0.;
    py[k] = c < M ? bp[3 * c + 1] : 0.;
    pz[k] = c < M ? bp[3 * c + 2] : 0.;
  }

  int rows = 0;  // rows of R that can be nonzero so far
  for (i64 t0 = 0; t0 < S; t0 += TR) {
    const int nrows = (int)((S - t0) < TR ? (S - t0) : TR);
    if (tid < nrows) {
      const double* q = bodies + 3 * (i64)my_sidx[t0 + tid];
      sp[3 * tid] = q[0];
      sp[3 * tid + 1] = q[1];
      sp[3 * tid + 2] = q[2];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < TS_MAXCOL; k++) {
      int c = tid + k * TS_THREADS;
      if (c < M)
        for (int r = 0; r < TR; r++)
          tile[r * M + c] = r < nrows ? (T)kernel_fast_pair(kp, sp[3 * r], sp[3 * r + 1], sp[3 * r + 2], px[k], py[k], pz[k]) : T(0);
    }
    __syncthreads();
    const int jend = (rows + nrows) < M ? (rows + nrows) : M;
    for (int j = 0; j < jend; j++) {
      const int owner = j % TS_THREADS;
      if (warp == (owner >> 5)) {
        // Reflector on (R[j][j], tile[:, j]), computed by the owner's warp:
        // lane r holds tile row r.
        T x = lane < nrows ? tile[lane * M + j] : T(0);
        T sig = x * x;
        for (int o = 16; o > 0; o >>= 1) sig += __shfl_xor_sync(0xffffffffu, sig, o);
        T alpha = R[(i64)j * M + j];
        T tau = 0, scale = 0, beta = alpha;
        if (sig > Tiny<T>::v()) {
          T nrm = sqrt(alpha * alpha + sig);
          beta = alpha >= T(0) ? -nrm : nrm;
          tau = (beta - alpha) / beta;
          scale = T(1) / (alpha - beta);
        }
        vbuf[lane] = x * scale;
        if (lane == 0) {
          s_tau = tau;
          R[(i64)j * M + j] = beta;
        }
      }
      __syncthreads();
      const T tau = s_tau;
      if (tau != T(0)) {
#pragma unroll
        for (int k = 0; k < TS_MAXCOL; k++) {
          int c = tid + k * TS_THREADS;
          if (c > j && c < M) {
            T w = R[(i64)j * M + c];
            for (int r = 0; r < nrows; r++) w += vbuf[r] * tile[r * M + c];
            w *= tau;
            R[(i64)j * M + c] -= w;
            for (int r = 0; r < nrows; r++) tile[r * M + c] -= w * vbuf[r];
          }
        }
      }
      __syncthreads();
    }
    rows = jend;
  }
}

// Column-pivoted Householder QR (Eigen 3.4 ColPivHouseholderQR::computeInPlace
// restated) of the K x M row-major matrix in Rws.  ``steps`` bounds the
// number of pivots taken (min(K, M) in threshold mode, the fixed rank in
// fixed-rank mode; the first ``steps`` rows of R do not depend on later
// steps).  Writes perm (position k holds the original column), maxpivot and
// the nonzero-pivot count.
template <typename T>
__global__ void __launch_bounds__(256) k_cpqr(const i64* __restrict__ dims, const i64* __restrict__ krows,
                                              T* __restrict__ Rws, const i64* __restrict__ qoff,
                                              int* __restrict__ perm_out, const i64* __restrict__ xoff,
                                              double* __restrict__ maxpiv_out, int* __restrict__ nonzero_out,
                                              i64 step_cap) {
  const int box = blockIdx.x;
  const int M = (int)dims[box];
  const int K = (int)krows[box];
  if (M == 0 || K == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* nu = reinterpret_cast<double*>(smem_raw);  // updated norms
  double* nd = nu + M;                               // direct norms
  T* ess = reinterpret_cast<T*>(nd + M);             // K
  int* perm = reinterpret_cast<int*>(ess + K);       // M
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ T red_t[32];
  __shared__ int s_nonzero;
  __shared__ double s_maxpiv;

  T* W = Rws + qoff[box];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int size = K < M ? K : M;
  int steps = size;
  if (step_cap >= 0 && step_cap < steps) steps = (int)step_cap;

  for (int c = tid; c < M; c += nt) {
    double s = 0.;
    for (int r = 0; r < K; r++) {
      double v = (double)W[(i64)r * M + c];
      s += v * v;
    }
    nu[c] = sqrt(s);
    nd[c] = nu[c];
    perm[c] = c;
  }
  __syncthreads();
  double mx = 0.;
  int mi = 0;
  for (int c = tid; c < M; c += nt)
    if (nu[c] > mx) { mx = nu[c]; mi = c; }
  argmax_first(mx, mi, red_v, red_i);
  const double eps = (sizeof(T) == 8) ? DBL_EPSILON : (double)FLT_EPSILON;
  const double thr_helper = (mx * eps) * (mx * eps) / (double)K;
  const double downdate_thr = sqrt(eps);
  if (tid == 0) {
    s_nonzero = size;
    s_maxpiv = 0.;
  }
  __syncthreads();

  for (int k = 0; k < steps; k++) {
    double bv = -1.;
    int bi = 0x7fffffff;
    for (int c = k + tid; c < M; c += nt)
      if (nu[c] > bv) { bv = nu[c]; bi = c; }
    argmax_first(bv, bi, red_v, red_i);
    // No candidate compares greater when every norm is NaN: keep column k
    // rather than index outside the matrix.
    if (bi < k || bi >= M) bi = k;
    if (tid == 0) {
      if (s_nonzero == size && bv * bv < thr_helper * (double)(K - k)) s_nonzero = k;
      if (bi != k) {
        double t = nu[k]; nu[k] = nu[bi]; nu[bi] = t;
        t = nd[k]; nd[k] = nd[bi]; nd[bi] = t;
        int ti = perm[k]; perm[k] = perm[bi]; perm[bi] = ti;
      }
    }
    if (bi != k)
      for (int r = tid; r < K; r += nt) {
        T t = W[(i64)r * M + k];
        W[(i64)r * M + k] = W[(i64)r * M + bi];
        W[(i64)r * M + bi] = t;
      }
    __syncthreads();
    // Householder on column k, rows k..K-1.
    T part = 0;
    for (int r = k + 1 + tid; r < K; r += nt) {
      T v = W[(i64)r * M + k];
      part += v * v;
    }
    T tsq = BlockReduce<T>::sum(part, red_t);
    T c0 = W[(i64)k * M + k];
    T tau = 0, beta = c0, scale = 0;
    if (tsq > Tiny<T>::v()) {
      beta = sqrt(c0 * c0 + tsq);
      if (c0 >= T(0)) beta = -beta;
      scale = T(1) / (c0 - beta);
      tau = (beta - c0) / beta;
    }
    for (int r = k + 1 + tid; r < K; r += nt) {
      T e = W[(i64)r * M + k] * scale;
      ess[r] = e;
      W[(i64)r * M + k] = e;
    }
    if (tid == 0) {
      W[(i64)k * M + k] = beta;
      double ab = fabs((double)beta);
      if (ab > s_maxpiv) s_maxpiv = ab;
    }
    __syncthreads();
    for (int j = k + 1 + tid; j < M; j += nt) {
      if (tau != T(0)) {
        T w = W[(i64)k * M + j];
        for (int r = k + 1; r < K; r++) w += ess[r] * W[(i64)r * M + j];
        w *= tau;
        W[(i64)k * M + j] -= w;
        for (int r = k + 1; r < K; r++) W[(i64)r * M + j] -= w * ess[r];
      }
      if (nu[j] != 0.) {
        double t = fabs((double)W[(i64)k * M + j]) / nu[j];
        t = (1. + t) * (1. - t);
        if (t < 0.) t = 0.;
        double t2 = t * (nu[j] / nd[j]) * (nu[j] / nd[j]);
        if (t2 <= downdate_thr) {
          double s = 0.;
          for (int r = k + 1; r < K; r++) {
            double v = (double)W[(i64)r * M + j];
            s += v * v;
          }
          nd[j] = sqrt(s);
          nu[j] = nd[j];
        } else {
          nu[j] *= sqrt(t);
        }
      }
    }
    __syncthreads();
  }
  for (int c = tid; c < M; c += nt) perm_out[xoff[box] + c] = perm[c];
  if (tid == 0) {
    maxpiv_out[box] = s_maxpiv;
    nonzero_out[box] = s_nonzero;
  }
}

// Interpolative decomposition and the box basis.  W holds the packed CPQR
// (row-major); Q (col-major, in/out) holds the incoming Q (identity at a
// leaf, the children's R blocks above); R (col-major, out, zero on entry).
template <typename T>
__global__ void __launch_bounds__(256) k_basis_finish(
    const i64* __restrict__ dims, const i64* __restrict__ krows, T* __restrict__ Rws, T* __restrict__ Q,
    T* __restrict__ Rm, const i64* __restrict__ qoff, const int* __restrict__ perm_in,
    const i64* __restrict__ xoff, const double* __restrict__ maxpiv, const int* __restrict__ nonzero,
    double* __restrict__ pts, i64* __restrict__ ranks_out, double epi, int orth, int qin_identity,
    T* __restrict__ wy_taus, int xcap) {
  const int box = blockIdx.x;
  const int M = (int)dims[box];
  const int K = (int)krows[box];
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  if (M == 0 || K == 0) {
    if (tid == 0) ranks_out[box] = 0;
    return;
  }
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int* perm = reinterpret_cast<int*>(smem_raw);                          // M
  double* sp = reinterpret_cast<double*>(smem_raw + ((4 * M + 15) / 16) * 16);  // 3M
  T* taus = reinterpret_cast<T*>(sp + 3 * M);                            // M
  __shared__ int s_rank;
  __shared__ T s_red[32];
  T* W = Rws + qoff[box];
  T* Qb = Q + qoff[box];
  T* Rb = Rm + qoff[box];
  for (int c = tid; c < M; c += nt) perm[c] = perm_in[xoff[box] + c];
  if (tid == 0) {
    int size = K < M ? K : M;
    int r = (int)floor(epi);
    r = size < r ? size : r;
    if (epi < 1.) {
      double thr = fabs(maxpiv[box]) * epi;
      r = 0;
      for (int i = 0; i < nonzero[box]; i++) r += fabs((double)W[(i64)i * M + i]) > thr;
    }
    s_rank = r;
  }
  __syncthreads();
  const int rank = s_rank;
  if (!(0 < rank && rank < M)) {
    // R = upper triangle of the incoming Q, Q = identity (h2matrix.cpp:57-60).
    for_each_rc(M, M, [&](int r, int c, int e) {
      Rb[e] = r <= c ? Qb[e] : T(0);
    });
    __syncthreads();
    for_each_rc(M, M, [&](int r, int c, int e) {
      Qb[e] = r == c ? T(1) : T(0);
    });
    if (tid == 0) ranks_out[box] = rank;
    return;
  }
  // T = R11^{-1} R12 in place (rows 0..rank-1, columns rank..M-1), by
  // column chunks staged in shared memory (as many columns as fit, so
  // usually one chunk): back substitution with the whole CTA updating the
  // rows above the current one (one barrier per row, one reciprocal of the
  // pivot per row).
  {
    T* X = taus + M;  // rank x nc, row-major
    const int nc = max(1, min(M - rank, xcap / rank));
    for (int c0 = rank; c0 < M; c0 += nc) {
      const int w = min(nc, M - c0);
      for (int e = tid; e < rank * w; e += nt) X[e] = W[(i64)(e / w) * M + c0 + e % w];
      __syncthreads();
      for (int i = rank - 1; i >= 0; i--) {
        const T inv = T(1) / W[(i64)i * M + i];
        for (int k = warp; k < i; k += nw) {  // warp: row k, lanes: columns
          const T wki = W[(i64)k * M + i] * inv;
          for (int c = lane; c < w; c += 32) X[k * w + c] -= wki * X[i * w + c];
        }
        __syncthreads();
      }
      for (int e = tid; e < rank * w; e += nt) {
        const int i = e / w;
        W[(i64)i * M + c0 + e % w] = X[e] / W[(i64)i * M + i];
      }
      __syncthreads();
    }
  }
  // Skeleton-first order of the box bodies.
  double* bp = pts + 3 * xoff[box];
  for (int e = tid; e < 3 * M; e += nt) sp[e] = bp[e];
  __syncthreads();
  for (int k = tid; k < M; k += nt) {
    int p = perm[k];
    bp[3 * k] = sp[3 * p];
    bp[3 * k + 1] = sp[3 * p + 1];
    bp[3 * k + 2] = sp[3 * p + 2];
  }
  if (!orth) {
    // Q = P [I; T^T] padded with zero columns, R = I (h2matrix.cpp:50-55).
    for (i64 e = tid; e < (i64)M * M; e += nt) Qb[e] = T(0);
    __syncthreads();
    for_each_rc(M, rank, [&](int k, int i, int e) {
      T v = k < rank ? (k == i ? T(1) : T(0)) : W[(i64)i * M + k];
      Qb[(i64)perm[k] + (i64)i * M] = v;
    });
    for (int i = tid; i < rank; i += nt) Rb[(i64)i * M + i] = T(1);
    if (tid == 0) ranks_out[box] = rank;
    return;
  }
  // Orthogonal mode (h2matrix.cpp:43-49).  U_ID = P [I; T^T] (M x rank)
  // goes to R's slot as scratch, RX2 = triu(Qin) U_ID to W (col-major now).
  for_each_rc(M, rank, [&](int k, int i, int e) {
    T v = k < rank ? (k == i ? T(1) : T(0)) : W[(i64)i * M + k];
    Rb[(i64)perm[k] + (i64)i * M] = v;
  });
  __syncthreads();
  if (wy_taus) {
    // Blocked completion on the host side: U_ID is in R's slot, Q still
    // holds Q_in; the caller forms triu(Q_in) U_ID, its QR and Q.
    if (tid == 0) ranks_out[box] = rank;
    return;
  }
  for_each_rc(M, rank, [&](int p, int i, int e) {
    T s;
    if (qin_identity) {
      s = Rb[e];
    } else {
      s = 0;
      for (int l = p; l < M; l++) s += Qb[p + (i64)l * M] * Rb[l + (i64)i * M];
    }
    W[e] = s;
  });
  __syncthreads();
  // Householder QR of RX2 (M x rank), column-major in W.  One warp per
  // column for the reflector application.
  for (int k = 0; k < rank; k++) {
    T* colk = W + (i64)k * M;
    T part = 0;
    for (int r = k + 1 + tid; r < M; r += nt) part += colk[r] * colk[r];
    T tsq = BlockReduce<T>::sum(part, s_red);
    T c0 = colk[k];
    T tau = 0, beta = c0, scale = 0;
    if (tsq > Tiny<T>::v()) {
      beta = sqrt(c0 * c0 + tsq);
      if (c0 >= T(0)) beta = -beta;
      scale = T(1) / (c0 - beta);
      tau = (beta - c0) / beta;
    }
    __syncthreads();
    for (int r = k + 1 + tid; r < M; r += nt) colk[r] *= scale;
    if (tid == 0) {
      colk[k] = beta;
      taus[k] = tau;
    }
    __syncthreads();
    if (tau != T(0))
      for (int j = k + 1 + warp; j < rank; j += nw) {
        T* colj = W + (i64)j * M;
        T w = 0;
        for (int r = k + 1 + lane; r < M; r += 32) w += colk[r] * colj[r];
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        w = (w + colj[k]) * tau;
        if (lane == 0) colj[k] -= w;
        for (int r = k + 1 + lane; r < M; r += 32) colj[r] -= w * colk[r];
      }
    __syncthreads();
  }
  // R = triu(RX2[:rank, :rank]) (R's slot was scratch: clear first).
  for_each_rc(M, M, [&](int r, int c, int e) {
    Rb[e] = (c < rank && r <= c) ? W[r + (i64)c * M] : T(0);
  });
  // Q = H_0 ... H_{rank-1} applied to the identity.
  for_each_rc(M, M, [&](int r, int c, int e) {
    Qb[e] = r == c ? T(1) : T(0);
  });
  __syncthreads();
  for (int k = rank - 1; k >= 0; k--) {
    const T tau = taus[k];
    const T* colk = W + (i64)k * M;
    if (tau != T(0))
      for (int j = k + warp; j < M; j += nw) {
        T* qj = Qb + (i64)j * M;
        T w = 0;
        for (int r = k + 1 + lane; r < M; r += 32) w += colk[r] * qj[r];
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        w = (w + qj[k]) * tau;
        if (lane == 0) qj[k] -= w;
        for (int r = k + 1 + lane; r < M; r += 32) qj[r] -= w * colk[r];
      }
    __syncthreads();
  }
  if (tid == 0) ranks_out[box] = rank;
}

// ---------------------------------------------------------------- launchers

template <typename T>
cudaError_t launch_sample_tsqr(const KernelParams& kp, const double* bodies, const double* pts, const i64* xoff,
                               const i64* dims, const int* sidx, const i64* soff, T* Rws, const i64* qoff,
                               int nboxes, int maxM, cudaStream_t st) {
  if (nboxes == 0) return cudaSuccess;
  if (maxM > TS_THREADS * TS_MAXCOL) return cudaErrorInvalidValue;
  int tr = 32;
  while (tr > 8 && sizeof(T) * (tr * (size_t)maxM + 32) + sizeof(double) * 96 > 200 * 1024) tr /= 2;
  size_t smem = sizeof(T) * (tr * (size_t)maxM + 32) + sizeof(double) * 96;
  if (smem > 220 * 1024) return cudaErrorInvalidValue;  // box too large for one tile in shared memory
  auto fn = tr == 32 ? k_sample_tsqr<T, 32> : tr == 16 ? k_sample_tsqr<T, 16> : k_sample_tsqr<T, 8>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  note_launch();
  fn<<<nboxes, TS_THREADS, smem, st>>>(kp, bodies, pts, xoff, dims, sidx, soff, Rws, qoff);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_cpqr(const i64* dims, const i64* krows, T* Rws, const i64* qoff, int* perm, const i64* xoff,
                        double* maxpiv, int* nonzero, i64 step_cap, int nboxes, int maxM, cudaStream_t st) {
  if (nboxes == 0) return cudaSuccess;
  size_t smem = 2 * sizeof(double) * maxM + sizeof(T) * maxM + sizeof(int) * maxM + 64;
  auto fn = k_cpqr<T>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  note_launch();
  fn<<<nboxes, 256, smem, st>>>(dims, krows, Rws, qoff, perm, xoff, maxpiv, nonzero, step_cap);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_basis_finish(const i64* dims, const i64* krows, T* Rws, T* Q, T* R, const i64* qoff,
                                const int* perm, const i64* xoff, const double* maxpiv, const int* nonzero,
                                double* pts, i64* ranks, double epi, int orth, int qin_identity, int nboxes,
                                int maxM, cudaStream_t st, T* wy_taus) {
  if (nboxes == 0) return cudaSuccess;
  // Back-substitution chunk: columns of rank rows, at most 96 KB (all
  // M - rank columns of a 256-box at rank >= 64 in FP64).
  const int xcap = (int)std::min<size_t>((size_t)maxM * maxM, 96 * 1024 / sizeof(T));
  size_t smem = ((4 * (size_t)maxM + 15) / 16) * 16 + sizeof(double) * 3 * maxM + sizeof(T) * (maxM + xcap) + 64;
  auto fn = k_basis_finish<T>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  note_launch();
  fn<<<nboxes, 256, smem, st>>>(dims, krows, Rws, Q, R, qoff, perm, xoff, maxpiv, nonzero, pts, ranks, epi, orth,
                                qin_identity, wy_taus, xcap);
  return cudaGetLastError();
}

#define INST(T)                                                                                                     \
  template cudaError_t launch_sample_tsqr<T>(const KernelParams&, const double*, const double*, const i64*,       \
                                             const i64*, const int*, const i64*, T*, const i64*, int, int,       \
                                             cudaStream_t);                                                       \
  template cudaError_t launch_cpqr<T>(const i64*, const i64*, T*, const i64*, int*, const i64*, double*, int*,    \
                                      i64, int, int, cudaStream_t);                                               \
  template cudaError_t launch_basis_finish<T>(const i64*, const i64*, T*, T*, T*, const i64*, const int*,         \
                                              const i64*, const double*, const int*, double*, i64*, double, int,  \
                                              int, int, int, cudaStream_t, T*);
INST(double)
INST(float)
#undef INST

}  // namespace h2b

namespace h2b {

// Gathers each box's far-sample bodies into one contiguous array.
__global__ void k_gather_points(const double* __restrict__ bodies, const int* __restrict__ idx, i64 n,
                                double* __restrict__ out) {
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const double* p = bodies + 3 * (i64)idx[i];
    out[3 * i] = p[0];
    out[3 * i + 1] = p[1];
    out[3 * i + 2] = p[2];
  }
}

cudaError_t launch_gather_points(const double* bodies, const int* idx, i64 n, double* out, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  int grid = (int)((n + 255) / 256);
  grid = grid > 4096 ? 4096 : grid;
  note_launch();
  k_gather_points<<<grid, 256, 0, st>>>(bodies, idx, n, out);
  return cudaGetLastError();
}

}  // namespace h2b

namespace h2b {

// One 32-pivot panel of the blocked pivoted Cholesky of the Gram matrix
// G = XF^T XF (M x M per box, symmetric), stopped after ``steps`` pivots in
// all.  The pivot is the largest remaining Schur-complement diagonal (the
// squared column norm a column-pivoted QR of XF would pick), so pivots and
// rows of R equal those of ColPivHouseholderQR in exact arithmetic
// (h2matrix.cpp:27); R goes to Rws row-major in pivoted column order, where
// k_cpqr leaves it, for k_basis_finish.  Once the Schur diagonal falls to
// rounding noise of the FP64 Gram matrix (16 eps max diag), the pivots
// still to be taken get the row [floor, 0, ..., 0] with floor =
// sqrt(eps max diag): their interpolation coefficients come out exactly zero.
// G already carries the trailing updates of earlier panels; this panel's
// pivots are taken left-looking: the Schur diagonal of the remaining
// columns lives in shared memory and loses R[k][j]^2 after every pivot, and
// row k of R is G[k][j] minus the panel's earlier rows.  The caller applies
// G_trail -= R_panel^T R_panel (one batched GEMM) afterwards.
__global__ void __launch_bounds__(256) k_pivchol_panel(const i64* __restrict__ dims, const i64* __restrict__ steps_box,
                                                       double* __restrict__ G, double* __restrict__ Rws,
                                                       const i64* __restrict__ qoff, int* __restrict__ perm_g,
                                                       const i64* __restrict__ xoff, double* __restrict__ state,
                                                       int k0, int nb) {
  const int box = blockIdx.x;
  const int M = (int)dims[box];
  const int steps = (int)steps_box[box];
  if (M == 0 || k0 >= steps) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* dsch = reinterpret_cast<double*>(smem_raw);  // M
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  double* g = G + qoff[box];
  double* R = Rws + qoff[box];
  int* perm = perm_g + xoff[box];
  double* st = state + 3 * (i64)box;  // [rfloor, noise threshold, noise flag]
  const int tid = threadIdx.x, nt = blockDim.x;
  if (k0 == 0) {
    for (int c = tid; c < M; c += nt) perm[c] = c;
    double dmax = 0.;
    int dmi = 0;
    for (int j = tid; j < M; j += nt) {
      double v = g[(i64)j * M + j];
      if (v > dmax) { dmax = v; dmi = j; }
    }
    argmax_first(dmax, dmi, red_v, red_i);
    if (tid == 0) {
      double rf = sqrt(DBL_EPSILON * dmax);
      st[0] = rf > 0. ? rf : DBL_MIN;
      st[1] = 16. * DBL_EPSILON * dmax;
      st[2] = 0.;
    }
    __syncthreads();
  }
  const double rfloor = st[0], noise = st[1];
  bool noise_mode = st[2] != 0.;
  for (int j = tid; j < M; j += nt) dsch[j] = j >= k0 ? g[(i64)j * M + j] : 0.;
  __syncthreads();
  const int kend = (k0 + nb < steps) ? k0 + nb : steps;
  for (int k = k0; k < kend; k++) {
    double bv = -1.;
    int bi = 0x7fffffff;
    for (int j = k + tid; j < M; j += nt)
      if (dsch[j] > bv) { bv = dsch[j]; bi = j; }
    argmax_first(bv, bi, red_v, red_i);
    if (bi < k || bi >= M) bi = k;
    if (bi != k) {
      // Rows/columns k0.. of G are the live trailing matrix; earlier rows of
      // R (all panels) follow the column exchange.
      for (int c = k0 + tid; c < M; c += nt) {
        double t = g[(i64)k * M + c];
        g[(i64)k * M + c] = g[(i64)bi * M + c];
        g[(i64)bi * M + c] = t;
      }
      __syncthreads();
      for (int r = k0 + tid; r < M; r += nt) {
        double t = g[(i64)r * M + k];
        g[(i64)r * M + k] = g[(i64)r * M + bi];
        g[(i64)r * M + bi] = t;
      }
      for (int r = tid; r < k; r += nt) {
        double t = R[(i64)r * M + k];
        R[(i64)r * M + k] = R[(i64)r * M + bi];
        R[(i64)r * M + bi] = t;
      }
      if (tid == 0) {
        double t = dsch[k]; dsch[k] = dsch[bi]; dsch[bi] = t;
        int ti = perm[k]; perm[k] = perm[bi]; perm[bi] = ti;
      }
    }
    __syncthreads();
    const double d = dsch[k];
    if (!(d > noise)) noise_mode = true;
    if (noise_mode) {
      for (int j = k + tid; j < M; j += nt) R[(i64)k * M + j] = (j == k) ? rfloor : 0.;
      __syncthreads();
      continue;
    }
    const double rkk = sqrt(d);
    const double inv = 1. / rkk;
    for (int j = k + tid; j < M; j += nt) {
      double v;
      if (j == k) {
        v = rkk;
      } else {
        v = g[(i64)k * M + j];
        for (int p = k0; p < k; p++) v -= R[(i64)p * M + k] * R[(i64)p * M + j];
        v *= inv;
        dsch[j] -= v * v;
      }
      R[(i64)k * M + j] = v;
    }
    __syncthreads();
  }
  if (tid == 0) st[2] = noise_mode ? 1. : 0.;
}

cudaError_t launch_pivchol_panel(const i64* dims, const i64* steps_box, double* G, double* Rws, const i64* qoff,
                                 int* perm, const i64* xoff, double* state, int k0, int nb, int nboxes, int maxM,
                                 cudaStream_t st) {
  if (nboxes == 0) return cudaSuccess;
  size_t smem = sizeof(double) * (size_t)maxM + 16;
  note_launch();
  k_pivchol_panel<<<nboxes, 256, smem, st>>>(dims, steps_box, G, Rws, qoff, perm, xoff, state, k0, nb);
  return cudaGetLastError();
}

}  // namespace h2b

namespace h2b {

// T of the compact-WY form Q = H_0 ... H_{r-1} = I - V T V^T (forward,
// column by column: T[i][i] = tau_i, T[0:i, i] = -tau_i T[0:i,0:i] S[0:i, i]
// with S = V^T V), one CTA per box, r x r column-major at Tb + toff[box].
// Blocked: the 32 x 32 diagonal blocks are independent and are formed one
// per warp with the recurrence (lane j keeps row j of its block in
// registers, the column -tau_i S[0:i, i] is shared by shuffles; no barrier);
// the blocks above the diagonal follow from the product rule of compact-WY
// factors, T[A, B] = -T[A, A] S[A, B] T[B, B], for the leading columns A of
// each column block B in turn (two barriers per block instead of two per
// column).
constexpr int WY_B = 32;

template <typename T>
__device__ __forceinline__ void wy_diag_block(const WyTask<T>& t, int off, int bs, int lane) {
  const int r = t.r;
  T row[WY_B];
#pragma unroll
  for (int l = 0; l < WY_B; l++) row[l] = T(0);
#pragma unroll
  for (int i = 0; i < WY_B; i++) {
    if (i < bs) {
      const T tau = t.taus[off + i];
      const T c = lane < i ? -tau * t.S[(off + lane) + (i64)(off + i) * r] : T(0);
      T v = T(0);
#pragma unroll
      for (int l = 0; l < WY_B; l++) {
        const T cl = __shfl_sync(0xffffffffu, c, l);
        if (l < i) v += row[l] * cl;
      }
      if (lane < i) row[i] = v;
      if (lane == i) row[i] = tau;
    }
  }
  if (lane < bs) {
#pragma unroll
    for (int l = 0; l < WY_B; l++)
      if (l < bs) t.Tm[(off + lane) + (i64)(off + l) * r] = row[l];
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_wy_t(const WyTask<T>* __restrict__ tasks) {
  const WyTask<T> t = tasks[blockIdx.x];
  const int r = t.r;
  if (r <= 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* X = reinterpret_cast<T*>(smem_raw);  // (r - 32) x 32, column-major, ld r
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int nb = (r + WY_B - 1) / WY_B;
  // Zero the strictly lower triangle (the blocks below write only the upper part).
  for (i64 e = threadIdx.x; e < (i64)r * r; e += blockDim.x) {
    const int row = (int)(e % r), colm = (int)(e / r);
    if (row > colm) t.Tm[e] = T(0);
  }
  for (int b = warp; b < nb; b += nw) wy_diag_block(t, b * WY_B, min(WY_B, r - b * WY_B), lane);
  __syncthreads();
  for (int b = 1; b < nb; b++) {
    const int off = b * WY_B, bs = min(WY_B, r - off), p = off;
    // X = S[0:p, B] T[B, B]  (T[B, B] upper triangular)
    for (int e = threadIdx.x; e < p * bs; e += blockDim.x) {
      const int j = e % p, c = e / p;
      T v = T(0);
      for (int k = 0; k <= c; k++) v += t.S[j + (i64)(off + k) * r] * t.Tm[(off + k) + (i64)(off + c) * r];
      X[j + c * p] = v;
    }
    __syncthreads();
    // T[0:p, B] = -T[0:p, 0:p] X  (T[0:p, 0:p] upper triangular)
    for (int e = threadIdx.x; e < p * bs; e += blockDim.x) {
      const int j = e % p, c = e / p;
      T v = T(0);
      for (int k = j; k < p; k++) v += t.Tm[j + (i64)k * r] * X[k + c * p];
      t.Tm[j + (i64)(off + c) * r] = -v;
    }
    __syncthreads();
  }
}

template <typename T>
cudaError_t launch_wy_t(const WyTask<T>* d_tasks, int ntasks, int maxr, cudaStream_t st) {
  if (ntasks == 0) return cudaSuccess;
  const size_t smem = sizeof(T) * (size_t)std::max(1, maxr - WY_B) * WY_B;
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k_wy_t<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  note_launch();
  k_wy_t<T><<<ntasks, 256, smem, st>>>(d_tasks);
  return cudaGetLastError();
}
template cudaError_t launch_wy_t<double>(const WyTask<double>*, int, int, cudaStream_t);
template cudaError_t launch_wy_t<float>(const WyTask<float>*, int, int, cudaStream_t);

}  // namespace h2b

namespace h2b {

// One Householder panel of the M x rank matrix W (column-major, ld M) of a
// box: columns k0..k0+nb-1, rows k0..M-1, factored in shared memory with the
// same reflector convention as k_basis_finish (beta = -sign(c0) * norm).
// Writes back R (upper) and the reflector tails (lower), the explicit unit
// lower-trapezoidal V of the panel to Vp ((M-k0) x nb), the panel's
// compact-WY T (nb x nb, I - V T V^T = H_k0 ... H_k0+nb-1) to Tp and its
// taus.  The caller applies the panel to the trailing columns with GEMMs.
template <typename T>
__global__ void __launch_bounds__(256) k_qr_panel(const QrPanelTask<T>* __restrict__ tasks) {
  const QrPanelTask<T> t = tasks[blockIdx.x];
  const int m = t.M - t.k0, nb = t.nb;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* P = reinterpret_cast<T*>(smem_raw);  // m x nb, ld m
  T* tau = P + (size_t)m * nb;            // nb
  T* Tl = tau + nb;                       // nb x nb
  T* sc = Tl + (size_t)nb * nb;           // nb
  __shared__ T red[32];
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  T* Wp = t.W + (i64)t.k0 + (i64)t.k0 * t.M;
  for_each_rc(m, nb, [&](int r, int j, int e) {
    P[e] = Wp[r + (i64)j * t.M];
  });
  __syncthreads();
  for (int j = 0; j < nb; j++) {
    T* cj = P + (size_t)j * m;
    T part = 0;
    for (int r = j + 1 + tid; r < m; r += nt) part += cj[r] * cj[r];
    T tsq = BlockReduce<T>::sum(part, red);
    T c0 = cj[j];
    T tj = 0, beta = c0, scale = 0;
    if (tsq > Tiny<T>::v()) {
      beta = sqrt(c0 * c0 + tsq);
      if (c0 >= T(0)) beta = -beta;
      scale = T(1) / (c0 - beta);
      tj = (beta - c0) / beta;
    }
    __syncthreads();
    for (int r = j + 1 + tid; r < m; r += nt) cj[r] *= scale;
    if (tid == 0) {
      cj[j] = beta;
      tau[j] = tj;
    }
    __syncthreads();
    if (tj != T(0))
      for (int jj = j + 1 + warp; jj < nb; jj += nw) {
        T* c2 = P + (size_t)jj * m;
        T w = 0;
        for (int r = j + 1 + lane; r < m; r += 32) w += cj[r] * c2[r];
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        w = (w + c2[j]) * tj;
        if (lane == 0) c2[j] -= w;
        for (int r = j + 1 + lane; r < m; r += 32) c2[r] -= w * cj[r];
      }
    __syncthreads();
  }
  // S[l][i] = V(:,l)^T V(:,i) for l < i (V unit lower: V[i][i] = 1, zero above).
  for (int pr = warp; pr < nb * nb; pr += nw) {
    int l = pr % nb, i = pr / nb;
    if (l >= i) continue;
    T s = 0;
    for (int r = i + 1 + lane; r < m; r += 32) s += P[r + (size_t)l * m] * P[r + (size_t)i * m];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) Tl[l + i * nb] = s + P[i + (size_t)l * m];  // row i of V(:,l) times V[i][i] = 1
  }
  __syncthreads();
  // T recurrence, one warp: column i of S is staged in sc, then
  // T[:i, i] = -tau_i T[:i,:i] S[:i, i] and T[i][i] = tau_i.
  if (warp == 0) {
    for (int i = 0; i < nb; i++) {
      for (int j = lane; j < i; j += 32) sc[j] = Tl[j + i * nb];
      __syncwarp();
      for (int j = lane; j < i; j += 32) {
        T v = 0;
        for (int l = j; l < i; l++) v += Tl[j + l * nb] * sc[l];
        Tl[j + i * nb] = -tau[i] * v;
      }
      if (lane == 0) Tl[i + i * nb] = tau[i];
      __syncwarp();
    }
  }
  __syncthreads();
  for_each_rc(m, nb, [&](int r, int j, int e) {
    Wp[r + (i64)j * t.M] = P[e];
    t.Vp[e] = r < j ? T(0) : (r == j ? T(1) : P[e]);
  });
  for (int e = tid; e < nb * nb; e += nt) {
    int r = e % nb, c = e / nb;
    t.Tp[e] = r <= c ? Tl[e] : T(0);
  }
  for (int j = tid; j < nb; j += nt) t.taus[t.k0 + j] = tau[j];
}

template <typename T>
cudaError_t launch_qr_panel(const QrPanelTask<T>* d_tasks, int ntasks, int maxm, int nb, cudaStream_t st) {
  if (ntasks == 0) return cudaSuccess;
  size_t smem = sizeof(T) * ((size_t)maxm * nb + 2 * nb + (size_t)nb * nb) + 16;
  auto fn = k_qr_panel<T>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  note_launch();
  fn<<<ntasks, 256, smem, st>>>(d_tasks);
  return cudaGetLastError();
}
template cudaError_t launch_qr_panel<double>(const QrPanelTask<double>*, int, int, int, cudaStream_t);
template cudaError_t launch_qr_panel<float>(const QrPanelTask<float>*, int, int, int, cudaStream_t);

}  // namespace h2b

namespace h2b {

// After the blocked QR of W (M x rank): R's slot gets triu(W[:rank, :rank]),
// W becomes the explicit unit lower-trapezoidal V, Q the identity (for the
// compact-WY formation that follows).
template <typename T>
__global__ void __launch_bounds__(256) k_qr_extract(const QrExtractTask<T>* __restrict__ tasks) {
  const QrExtractTask<T> t = tasks[blockIdx.x];
  const int M = t.M, r = t.rank;
  for_each_rc(M, M, [&](int i, int c, int e) {
    t.R[e] = (c < r && i <= c) ? t.W[i + (i64)c * M] : T(0);
    t.Q[e] = i == c ? T(1) : T(0);
  });
  __syncthreads();
  for_each_rc(M, r, [&](int i, int c, int e) {
    if (i <= c) t.W[e] = i == c ? T(1) : T(0);
  });
}

template <typename T>
cudaError_t launch_qr_extract(const QrExtractTask<T>* d_tasks, int ntasks, cudaStream_t st) {
  if (ntasks == 0) return cudaSuccess;
  note_launch();
  k_qr_extract<T><<<ntasks, 256, 0, st>>>(d_tasks);
  return cudaGetLastError();
}
template cudaError_t launch_qr_extract<double>(const QrExtractTask<double>*, int, cudaStream_t);
template cudaError_t launch_qr_extract<float>(const QrExtractTask<float>*, int, cudaStream_t);

}  // namespace h2b
