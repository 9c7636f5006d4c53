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
// One CTA of 128 threads per {task, 128 RPT-row block}; each thread owns
// RPT rows (their bodies in registers) and accumulates all right-hand sides
// in registers.  The task's entries are walked in 32-column slabs: the slab's
// column bodies and the 32 x NR right-hand-side values go to shared memory
// (row-contiguous, so each is read by a broadcast vector load), then every
// thread evaluates its rows against the 32 columns and updates its
// accumulators.  FP64 throughout, one reciprocal square root per pair
// (rsqrt_newton: an FP32 seed refined by two FP64 Newton steps, about 1 ulp;
// the whole entry is a few ulp from the reference's std::hypot form); the
// summation order is fixed by the plan, so results are deterministic.  Bound: FP64 FMA throughput (2 NR
// multiply-adds plus one kernel evaluation per pair), not HBM.
#include "common.cuh"
#include "kernels.h"

namespace h2b {

namespace {

constexpr int MF_NT = 128, MF_KS = 32;

// RPT rows per thread (BM = 128 RPT rows per CTA): RPT = 2 shares each
// right-hand-side load between two rows; RPT = 1 halves the registers, so
// twice as many warps fit on an SM to hide the FP64 latency.  Per row the
// pairs are accumulated in the same order either way (bit-identical
// results); the plan times both once and keeps the faster.
template <int NR, int KIND, int RPT>
__global__ void __launch_bounds__(MF_NT, RPT == 1 ? 8 : 4)
    k_mf_apply(KernelParams kp, const MfTask* __restrict__ tasks, const MfEntry* __restrict__ ents,
               const int2* __restrict__ tiles, int nr) {
  constexpr int NRP = NR < 2 ? 2 : NR;  // padded row of the right-hand-side slab (16-byte loads)
  __shared__ __align__(16) double bs[MF_KS * NRP];
  __shared__ double cs[MF_KS * 3];
  const int2 tl = tiles[blockIdx.x];
  const MfTask t = tasks[tl.x];
  const int tid = threadIdx.x;
  int row[RPT];
  bool val[RPT];
  double px[RPT], py[RPT], pz[RPT];
  double acc[RPT][NR];
#pragma unroll
  for (int q = 0; q < RPT; q++) {
    row[q] = tl.y * MF_NT * RPT + tid + q * MF_NT;
    val[q] = row[q] < t.m;
    px[q] = val[q] ? t.pts[3 * row[q]] : 0.;
    py[q] = val[q] ? t.pts[3 * row[q] + 1] : 0.;
    pz[q] = val[q] ? t.pts[3 * row[q] + 2] : 0.;
#pragma unroll
    for (int c = 0; c < NR; c++) acc[q][c] = 0.;
  }

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
        double kv[RPT];
#pragma unroll
        for (int q = 0; q < RPT; q++) kv[q] = kernel_eval<KIND>(kp, px[q] - cx, py[q] - cy, pz[q] - cz);
        const double* br = bs + b * NRP;
        if constexpr (NR == 1) {
          const double x = br[0];
#pragma unroll
          for (int q = 0; q < RPT; q++) acc[q][0] = fma(kv[q], x, acc[q][0]);
        } else {
#pragma unroll
          for (int c = 0; c < NR; c += 2) {
            const double2 x = *reinterpret_cast<const double2*>(br + c);
#pragma unroll
            for (int q = 0; q < RPT; q++) {
              acc[q][c] = fma(kv[q], x.x, acc[q][c]);
              acc[q][c + 1] = fma(kv[q], x.y, acc[q][c + 1]);
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < NR; c++) {
    if (c >= nr) break;
#pragma unroll
    for (int q = 0; q < RPT; q++) {
      if (!val[q]) continue;
      double* o = t.C + row[q] + (i64)c * t.ldc;
      *o = t.beta == 0. ? acc[q][c] : t.beta * *o + acc[q][c];
    }
  }
}

}  // namespace

int mf_rows_per_cta(int rpt) { return MF_NT * rpt; }

template <int KIND, int RPT>
static cudaError_t mf_go(const KernelParams& kp, int nr, const MfTask* d_tasks, const MfEntry* d_ents,
                         const int2* d_tiles, int ntiles, cudaStream_t st) {
  switch (nr) {
    case 1: k_mf_apply<1, KIND, RPT><<<ntiles, MF_NT, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr); break;
    case 2: k_mf_apply<2, KIND, RPT><<<ntiles, MF_NT, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr); break;
    case 3:
    case 4: k_mf_apply<4, KIND, RPT><<<ntiles, MF_NT, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr); break;
    case 5:
    case 6:
    case 7:
    case 8: k_mf_apply<8, KIND, RPT><<<ntiles, MF_NT, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr); break;
    default: k_mf_apply<16, KIND, RPT><<<ntiles, MF_NT, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr);
  }
  return cudaGetLastError();
}

template <int RPT>
static cudaError_t mf_kind(const KernelParams& kp, int nr, const MfTask* d_tasks, const MfEntry* d_ents,
                           const int2* d_tiles, int ntiles, cudaStream_t st) {
  if (kp.kind == KERNEL_LAPLACE) return mf_go<KERNEL_LAPLACE, RPT>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
  if (kp.kind == KERNEL_YUKAWA) return mf_go<KERNEL_YUKAWA, RPT>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
  return mf_go<KERNEL_QUADRATIC, RPT>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
}

cudaError_t launch_mf_apply(const KernelParams& kp, int nr, int rpt, const MfTask* d_tasks, const MfEntry* d_ents,
                            const int2* d_tiles, int ntiles, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  if (nr < 1 || nr > 16 || (rpt != 1 && rpt != 2)) return cudaErrorInvalidValue;
  note_launch();
  return rpt == 1 ? mf_kind<1>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st)
                  : mf_kind<2>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
}

}  // namespace h2b
