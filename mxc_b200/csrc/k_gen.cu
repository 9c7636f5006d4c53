// Kernel-block generation (gen_matrix, kernel.cpp:71-85) and the
// matrix-free FP64 dense matvec used to verify residuals (main.cpp:83-84,
// 398-402 take A_dense x on the host).
#include "common.cuh"
#include "kernels.h"

namespace h2b {

// Column-major blocks K(bi[r], bj[c]); grid.x = task, grid.y = chunk of
// the block's elements.  Consecutive threads write consecutive rows; a
// thread finds its first (row, column) by one 32-bit division and then
// steps by the block size without dividing (blocks hold < 2^31 elements;
// larger ones take the 64-bit path).
template <typename T, bool FAST>
__global__ void __launch_bounds__(256) k_gen_blocks(KernelParams kp, const GenTask* __restrict__ tasks, T* __restrict__ out) {
  const GenTask t = tasks[blockIdx.x];
  const i64 total = (i64)t.m * t.n;
  if (total == 0) return;
  const i64 per = (total + gridDim.y - 1) / gridDim.y;
  const i64 e0 = per * blockIdx.y, e1 = e0 + per < total ? e0 + per : total;
  T* o = out + t.out_off;
  auto value = [&](int r, int c) {
    const double* a = t.bi + 3 * r;
    const double* b = t.bj + 3 * c;
    return FAST ? (T)kernel_fast(kp, a[0] - b[0], a[1] - b[1], a[2] - b[2])
                : (T)kernel_exact(kp, a[0] - b[0], a[1] - b[1], a[2] - b[2]);
  };
  if (total < ((i64)1 << 31)) {
    const int m = t.m, stride = (int)blockDim.x;
    const int dq = stride / m, dr = stride - dq * m;
    int e = (int)e0 + (int)threadIdx.x;
    const int end = (int)e1;
    if (e >= end) return;
    int c = e / m, r = e - c * m;
    for (; e < end; e += stride) {
      o[r + (i64)c * t.ld] = value(r, c);
      r += dr;
      c += dq;
      if (r >= m) {
        r -= m;
        c++;
      }
    }
    return;
  }
  for (i64 e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const int r = (int)(e % t.m), c = (int)(e / t.m);
    o[r + (i64)c * t.ld] = value(r, c);
  }
}

template <typename T>
cudaError_t launch_gen_blocks(const KernelParams& kp, const GenTask* d_tasks, int ntasks, int chunks, T* out,
                              cudaStream_t st, int fast) {
  if (ntasks == 0) return cudaSuccess;
  dim3 grid(ntasks, chunks < 1 ? 1 : chunks);
  if (fast) {
    note_launch();
    k_gen_blocks<T, true><<<grid, 256, 0, st>>>(kp, d_tasks, out);
  } else {
    note_launch();
    k_gen_blocks<T, false><<<grid, 256, 0, st>>>(kp, d_tasks, out);
  }
  return cudaGetLastError();
}
template cudaError_t launch_gen_blocks<double>(const KernelParams&, const GenTask*, int, int, double*, cudaStream_t,
                                               int);
template cudaError_t launch_gen_blocks<float>(const KernelParams&, const GenTask*, int, int, float*, cudaStream_t,
                                              int);

// Y = A_dense X for up to NR right-hand sides per pass.  Each thread owns a
// row; columns stream through shared memory in tiles of 256 bodies.
constexpr int DM_THREADS = 256;
template <int NR>
__global__ void __launch_bounds__(DM_THREADS) k_dense_mv(KernelParams kp, const double* __restrict__ b, i64 n,
                                                         const double* __restrict__ X, i64 ldx,
                                                         double* __restrict__ Y, i64 ldy, int nr) {
  __shared__ double sp[DM_THREADS * 3];
  __shared__ double sx[DM_THREADS * NR];
  i64 i = (i64)blockIdx.x * DM_THREADS + threadIdx.x;
  double xi = 0., yi = 0., zi = 0.;
  if (i < n) {
    xi = b[3 * i];
    yi = b[3 * i + 1];
    zi = b[3 * i + 2];
  }
  double acc[NR];
#pragma unroll
  for (int c = 0; c < NR; c++) acc[c] = 0.;
  for (i64 j0 = 0; j0 < n; j0 += DM_THREADS) {
    i64 j = j0 + threadIdx.x;
    if (j < n) {
      sp[3 * threadIdx.x] = b[3 * j];
      sp[3 * threadIdx.x + 1] = b[3 * j + 1];
      sp[3 * threadIdx.x + 2] = b[3 * j + 2];
#pragma unroll
      for (int c = 0; c < NR; c++) sx[threadIdx.x * NR + c] = c < nr ? X[j + (i64)c * ldx] : 0.;
    }
    __syncthreads();
    int jn = (n - j0) < DM_THREADS ? (int)(n - j0) : DM_THREADS;
    for (int jj = 0; jj < jn; jj++) {
      double k = kernel_fast(kp, xi - sp[3 * jj], yi - sp[3 * jj + 1], zi - sp[3 * jj + 2]);
#pragma unroll
      for (int c = 0; c < NR; c++) acc[c] += k * sx[jj * NR + c];
    }
    __syncthreads();
  }
  if (i < n)
    for (int c = 0; c < nr; c++) Y[i + (i64)c * ldy] = acc[c];
}

cudaError_t launch_dense_matvec(const KernelParams& kp, const double* bodies, i64 n, const double* X, i64 ldx,
                                double* Y, i64 ldy, int nrhs, cudaStream_t st) {
  int grid = (int)((n + DM_THREADS - 1) / DM_THREADS);
  for (int c0 = 0; c0 < nrhs; c0 += 16) {
    int nr = nrhs - c0 < 16 ? nrhs - c0 : 16;
    const double* x = X + (i64)c0 * ldx;
    double* y = Y + (i64)c0 * ldy;
    if (nr == 1) {
      note_launch();
      k_dense_mv<1><<<grid, DM_THREADS, 0, st>>>(kp, bodies, n, x, ldx, y, ldy, nr);
    } else if (nr <= 4) {
      note_launch();
      k_dense_mv<4><<<grid, DM_THREADS, 0, st>>>(kp, bodies, n, x, ldx, y, ldy, nr);
    } else if (nr <= 8) {
      note_launch();
      k_dense_mv<8><<<grid, DM_THREADS, 0, st>>>(kp, bodies, n, x, ldx, y, ldy, nr);
    } else {
      note_launch();
      k_dense_mv<16><<<grid, DM_THREADS, 0, st>>>(kp, bodies, n, x, ldx, y, ldy, nr);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace h2b
