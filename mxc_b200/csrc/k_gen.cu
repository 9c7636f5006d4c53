// Kernel-block generation (gen_matrix, kernel.cpp:71-85) and the
// matrix-free FP64 dense matvec used to verify residuals (main.cpp:83-84,
// 398-402 take A_dense x on the host).
#include "common.cuh"
#include "kernels.h"

namespace h2b {

// Column-major blocks K(bi[r], bj[c]); grid.x = task, grid.y = tile of 256
// rows.  The task's column bodies are staged in shared memory 256 at a time
// -- by one cp.async.bulk copy completing on an mbarrier when the tile starts
// on a 16-byte boundary, by coalesced loads otherwise -- and every thread
// keeps its row's body in registers, so each element costs one kernel
// evaluation (kind fixed at compile time) and one store; consecutive threads
// write consecutive rows of a column.  The wait on the bulk copy is bounded:
// an expired wait sets *err and the CTA falls back to plain loads.
constexpr int GEN_ROWS = 256, GEN_COLS = 256;
constexpr long long GEN_WAIT_CYCLES = 2000000000LL;  // about one second

template <int KIND>
__device__ __forceinline__ double gen_exact(const KernelParams& kp, double dx, double dy, double dz) {
  const double d = hypot3_exact(dx, dy, dz);
  if (d == 0.) return kp.diag;
  if constexpr (KIND == KERNEL_LAPLACE) return __ddiv_rn(1., d);
  if constexpr (KIND == KERNEL_QUADRATIC) return __dadd_rn(__dmul_rn(d, d), kp.alpha);
  return __ddiv_rn(exp(__dmul_rn(-kp.alpha, d)), d);
}

template <int KIND>
__device__ __forceinline__ double gen_fast(const KernelParams& kp, double dx, double dy, double dz) {
  const double r2 = dx * dx + dy * dy + dz * dz;
  if (r2 == 0.) return kp.diag;
  if constexpr (KIND == KERNEL_QUADRATIC) return r2 + kp.alpha;
  const double inv = rsqrt(r2);
  if constexpr (KIND == KERNEL_LAPLACE) return inv;
  return exp(-kp.alpha * (r2 * inv)) * inv;
}

// One element from the two bodies' coordinates (Helmholtz reads the
// component tags; the real kernels take the differences as above).
template <bool FAST, int KIND>
__device__ __forceinline__ double gen_pair(const KernelParams& kp, double xi, double yi, double zi, double xj,
                                           double yj, double zj) {
  if constexpr (KIND == KERNEL_HELMHOLTZ) return helm_entry<!FAST>(kp, xi, yi, zi, xj, yj, zj);
  const double dx = xi - xj, dy = yi - yj, dz = zi - zj;
  return FAST ? gen_fast<KIND>(kp, dx, dy, dz) : gen_exact<KIND>(kp, dx, dy, dz);
}

template <typename T, bool FAST, int KIND>
__global__ void __launch_bounds__(GEN_ROWS) k_gen_blocks(KernelParams kp, const GenTask* __restrict__ tasks,
                                                         T* __restrict__ out, int* __restrict__ err) {
  __shared__ __align__(16) double cpts[GEN_COLS * 3];
  __shared__ __align__(8) uint64_t bar;
  const GenTask t = tasks[blockIdx.x];
  const int r0 = blockIdx.y * GEN_ROWS;
  if (r0 >= t.m || t.n <= 0) return;
  const int r = r0 + (int)threadIdx.x;
  const bool live = r < t.m;
  double px = 0., py = 0., pz = 0.;
  if (live) {
    px = t.bi[3 * (i64)r];
    py = t.bi[3 * (i64)r + 1];
    pz = t.bi[3 * (i64)r + 2];
  }
  const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_s) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  T* o = out + t.out_off;
  uint32_t phase = 0;
  bool bulk_ok = true;  // cleared for good after an expired wait
  for (int c0 = 0; c0 < t.n; c0 += GEN_COLS) {
    const int nc = min(GEN_COLS, t.n - c0);
    const double* src = t.bj + 3 * (i64)c0;
    const uint32_t bytes = (uint32_t)(24 * nc);
    const bool bulk = bulk_ok && ((reinterpret_cast<uintptr_t>(src) & 15) == 0) && (bytes % 16 == 0);
    __syncthreads();  // the previous chunk's readers are done with cpts
    bool staged = false;
    if (bulk) {
      if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar_s), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                (uint32_t)__cvta_generic_to_shared(cpts)),
            "l"(src), "r"(bytes), "r"(bar_s)
            : "memory");
      }
      uint32_t ok = 0;
      const long long tw = clock64();
      while (true) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar_s), "r"(phase)
            : "memory");
        if (ok || clock64() - tw > GEN_WAIT_CYCLES) break;
      }
      phase ^= 1;
      staged = __syncthreads_and((int)ok) != 0;
      if (!staged) {
        bulk_ok = false;
        if (threadIdx.x == 0 && err) atomicExch(err, 1);
      }
    }
    if (!staged) {
      __syncthreads();
      for (int i = threadIdx.x; i < 3 * nc; i += GEN_ROWS) cpts[i] = src[i];
      __syncthreads();
    }
    if (live) {
      T* oc = o + r + (i64)c0 * t.ld;
#pragma unroll 4
      for (int c = 0; c < nc; c++) {
        oc[(i64)c * t.ld] = (T)gen_pair<FAST, KIND>(kp, px, py, pz, cpts[3 * c], cpts[3 * c + 1], cpts[3 * c + 2]);
      }
    }
  }
}

template <typename T, bool FAST>
static void gen_launch(const KernelParams& kp, dim3 grid, const GenTask* d_tasks, T* out, int* err, cudaStream_t st) {
  if (kp.kind == KERNEL_LAPLACE)
    k_gen_blocks<T, FAST, KERNEL_LAPLACE><<<grid, GEN_ROWS, 0, st>>>(kp, d_tasks, out, err);
  else if (kp.kind == KERNEL_YUKAWA)
    k_gen_blocks<T, FAST, KERNEL_YUKAWA><<<grid, GEN_ROWS, 0, st>>>(kp, d_tasks, out, err);
  else if (kp.kind == KERNEL_HELMHOLTZ)
    k_gen_blocks<T, FAST, KERNEL_HELMHOLTZ><<<grid, GEN_ROWS, 0, st>>>(kp, d_tasks, out, err);
  else
    k_gen_blocks<T, FAST, KERNEL_QUADRATIC><<<grid, GEN_ROWS, 0, st>>>(kp, d_tasks, out, err);
}

template <typename T>
cudaError_t launch_gen_blocks(const KernelParams& kp, const GenTask* d_tasks, int ntasks, i64 max_m, T* out,
                              cudaStream_t st, int fast, int* err) {
  if (ntasks == 0 || max_m <= 0) return cudaSuccess;
  const i64 ty = (max_m + GEN_ROWS - 1) / GEN_ROWS;
  if (ty > 65535) return cudaErrorInvalidValue;
  dim3 grid(ntasks, (unsigned)ty);
  note_launch();
  if (fast)
    gen_launch<T, true>(kp, grid, d_tasks, out, err, st);
  else
    gen_launch<T, false>(kp, grid, d_tasks, out, err, st);
  return cudaGetLastError();
}
template cudaError_t launch_gen_blocks<double>(const KernelParams&, const GenTask*, int, i64, double*, cudaStream_t,
                                               int, int*);
template cudaError_t launch_gen_blocks<float>(const KernelParams&, const GenTask*, int, i64, float*, cudaStream_t,
                                              int, int*);

// Helmholtz real form: body i of b (n x 3) becomes rows 2i + t of out
// (2n x 3), with bit 0 of x set to the component t (t = 0 real part, 1
// imaginary part).  comps = 1 writes only the t = 0 rows (n x 3 out).
__global__ void k_helm_expand(const double* __restrict__ b, i64 n, int comps, double* __restrict__ out) {
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const long long xb = __double_as_longlong(b[3 * i]) & ~1LL;
    const double y = b[3 * i + 1], z = b[3 * i + 2];
    for (int t = 0; t < comps; t++) {
      double* o = out + 3 * (comps * i + t);
      o[0] = __longlong_as_double(xb | t);
      o[1] = y;
      o[2] = z;
    }
  }
}
cudaError_t launch_helm_expand(const double* bodies, i64 n, int comps, double* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const i64 g = (n + 255) / 256;
  note_launch();
  k_helm_expand<<<(int)(g > 148 * 8 ? 148 * 8 : g), 256, 0, st>>>(bodies, n, comps, out);
  return cudaGetLastError();
}

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
      double k = kernel_fast_pair(kp, xi, yi, zi, sp[3 * jj], sp[3 * jj + 1], sp[3 * jj + 2]);
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
