// Matrix-free block applies for the H^2 operator in interpolative (ID)
// mode: C_task = beta C_task + sum_e alpha_e K(P_task, P_e) B_e, the kernel
// block K(P_task, P_e) evaluated on the fly from the two point sets instead
// of read from stored blocks.  In ID mode every block the matvec reads is a
// kernel evaluation: the leaf near blocks are K on the box bodies
// (h2matrix.cpp:184-188) and the couplings are K on the skeleton bodies
// (h2matrix.cpp:239-240), so the operator's matvec (h2matrix.cpp:251-344)
// needs only the bases and the points; nothing of size near-pairs x M^2 or
// far-pairs x rank^2 is stored.
//
// One CTA of 128 threads per {task, 256-row block}; each thread owns two
// rows (their bodies in registers) and accumulates all right-hand sides in
// registers.  The task's entries are walked in 32-column slabs: the slab's
// column bodies and the 32 x NR right-hand-side values go to shared memory
// (row-contiguous, so each is read by a broadcast vector load), then every
// thread evaluates its two rows against the 32 columns and updates its
// accumulators.  FP64 throughout, one reciprocal square root per pair
// (rsqrt_newton: an FP32 seed refined by two FP64 Newton steps, about 1 ulp;
// the whole entry is a few ulp from the reference's std::hypot form); the
// summation order is fixed by the plan, so results are deterministic.  Bound: FP64 FMA throughput (2 NR
// multiply-adds plus one kernel evaluation per pair), not HBM.
#include "common.cuh"
#include "kernels.h"

namespace h2b {

namespace {

constexpr int MF_NT = 128, MF_RPT = 2, MF_BM = MF_NT * MF_RPT, MF_KS = 32;

template <int NR, int KIND>
__global__ void __launch_bounds__(MF_NT, 4)
    k_mf_apply(KernelParams kp, const MfTask* __restrict__ tasks, const MfEntry* __restrict__ ents,
               const int2* __restrict__ tiles, int nr) {
  constexpr int NRP = NR < 2 ? 2 : NR;  // padded row of the right-hand-side slab (16-byte loads)
  __shared__ __align__(16) double bs[MF_KS * NRP];
  __shared__ double cs[MF_KS * 3];
  const int2 tl = tiles[blockIdx.x];
  const MfTask t = tasks[tl.x];
  const int tid = threadIdx.x;
  const int r0 = tl.y * MF_BM + tid, r1 = r0 + MF_NT;
  const bool v0 = r0 < t.m, v1 = r1 < t.m;
  double p0x = 0., p0y = 0., p0z = 0., p1x = 0., p1y = 0., p1z = 0.;
  if (v0) {
    p0x = t.pts[3 * r0];
    p0y = t.pts[3 * r0 + 1];
    p0z = t.pts[3 * r0 + 2];
  }
  if (v1) {
    p1x = t.pts[3 * r1];
    p1y = t.pts[3 * r1 + 1];
    p1z = t.pts[3 * r1 + 2];
  }
  double a0[NR], a1[NR];
#pragma unroll
  for (int c = 0; c < NR; c++) a0[c] = a1[c] = 0.;

  for (int e = t.e0; e < t.e1; e++) {
    const MfEntry en = ents[e];
    for (int k0 = 0; k0 < en.k; k0 += MF_KS) {
      const int kn = min(MF_KS, en.k - k0);
      __syncthreads();
      for (int q = tid; q < MF_KS * NR; q += MF_NT) {
        const int b = q % MF_KS, c = q / MF_KS;
        bs[b * NRP + c] = (b < kn && c < nr) ? en.alpha * en.B[(i64)(k0 + b) + (i64)c * en.ldb] : 0.;
      }
      for (int q = tid; q < MF_KS * 3; q += MF_NT) cs[q] = q < 3 * kn ? en.pts[3 * (i64)k0 + q] : 0.;
      __syncthreads();
      for (int b = 0; b < kn; b++) {
        const double cx = cs[3 * b], cy = cs[3 * b + 1], cz = cs[3 * b + 2];
        const double k0v = kernel_eval<KIND>(kp, p0x - cx, p0y - cy, p0z - cz);
        const double k1v = kernel_eval<KIND>(kp, p1x - cx, p1y - cy, p1z - cz);
        const double* br = bs + b * NRP;
        if constexpr (NR == 1) {
          const double x = br[0];
          a0[0] = fma(k0v, x, a0[0]);
          a1[0] = fma(k1v, x, a1[0]);
        } else {
#pragma unroll
          for (int c = 0; c < NR; c += 2) {
            const double2 x = *reinterpret_cast<const double2*>(br + c);
            a0[c] = fma(k0v, x.x, a0[c]);
            a0[c + 1] = fma(k0v, x.y, a0[c + 1]);
            a1[c] = fma(k1v, x.x, a1[c]);
            a1[c + 1] = fma(k1v, x.y, a1[c + 1]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < NR; c++) {
    if (c >= nr) break;
    if (v0) {
      double* o = t.C + r0 + (i64)c * t.ldc;
      *o = t.beta == 0. ? a0[c] : t.beta * *o + a0[c];
    }
    if (v1) {
      double* o = t.C + r1 + (i64)c * t.ldc;
      *o = t.beta == 0. ? a1[c] : t.beta * *o + a1[c];
    }
  }
}

}  // namespace

int mf_rows_per_cta() { return MF_BM; }

template <int KIND>
static cudaError_t mf_go(const KernelParams& kp, int nr, const MfTask* d_tasks, const MfEntry* d_ents,
                         const int2* d_tiles, int ntiles, cudaStream_t st) {
  switch (nr) {
    case 1: k_mf_apply<1, KIND><<<ntiles, MF_NT, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr); break;
    case 2: k_mf_apply<2, KIND><<<ntiles, MF_NT, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr); break;
    case 3:
    case 4: k_mf_apply<4, KIND><<<ntiles, MF_NT, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr); break;
    case 5:
    case 6:
    case 7:
    case 8: k_mf_apply<8, KIND><<<ntiles, MF_NT, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr); break;
    default: k_mf_apply<16, KIND><<<ntiles, MF_NT, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr);
  }
  return cudaGetLastError();
}

cudaError_t launch_mf_apply(const KernelParams& kp, int nr, const MfTask* d_tasks, const MfEntry* d_ents,
                            const int2* d_tiles, int ntiles, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  if (nr < 1 || nr > 16) return cudaErrorInvalidValue;
  note_launch();
  if (kp.kind == KERNEL_LAPLACE) return mf_go<KERNEL_LAPLACE>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
  if (kp.kind == KERNEL_YUKAWA) return mf_go<KERNEL_YUKAWA>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
  return mf_go<KERNEL_QUADRATIC>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
}

}  // namespace h2b
