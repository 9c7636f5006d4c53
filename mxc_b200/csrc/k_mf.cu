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
// (about 1 ulp; the whole entry is a few ulp from the reference's std::hypot
// form); the summation order is fixed by the plan, so results are
// deterministic.  Bound: FP64 FMA throughput (2 NR multiply-adds plus one
// kernel evaluation per pair), not HBM.
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
        for (int q = 0; q < RPT; q++) kv[q] = kernel_eval_pair<KIND>(kp, px[q], py[q], pz[q], cx, cy, cz);
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

// Tensor-core variant for 5-16 right-hand sides: the kernel block is
// generated straight into mma.sync m16n8k16 FP64 fragments and multiplied
// by the right-hand sides on the FP64 tensor cores; no shared memory and
// no block barriers.  Four warps per CTA share the column bodies and
// right-hand sides through L1 (one-warp CTAs, which idle no warp beside
// short tasks, measured 5-10% slower).  Each warp owns 32 rows of a task
// (its lane holds rows
// g, g + 8, g + 16, g + 24 with their bodies in registers) and walks the
// task's entries in 16-column steps: a lane evaluates K for its 4 rows x 4
// columns (t, t + 4, t + 8, t + 12 of the step; bodies and right-hand sides
// read through L1, where the CTA's other warps find them again) and the warp
// issues 2 x NR / 8 MMAs.  Rows past m evaluate against a copy of row 0 and
// are not stored; columns past the entry's k contribute zero.  Per row the
// pairs are summed by the MMAs in k order, a fixed order for a given plan.
constexpr int MFD_WARPS = 4;

template <int NR, int KIND>
__global__ void __launch_bounds__(32 * MFD_WARPS) k_mf_dmma(KernelParams kp, const MfTask* __restrict__ tasks,
                                                             const MfEntry* __restrict__ ents,
                                                             const int2* __restrict__ tiles, int nr) {
  constexpr int NF = NR / 8;
  const int2 tl = tiles[blockIdx.x];
  const MfTask t = tasks[tl.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g8 = lane >> 2, t4 = lane & 3;
  const int r0 = tl.y * 32 * MFD_WARPS + warp * 32;
  if (r0 >= t.m) return;
  double px[4], py[4], pz[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int r = r0 + g8 + 8 * q;
    const int rr = r < t.m ? r : 0;
    px[q] = t.pts[3 * rr];
    py[q] = t.pts[3 * rr + 1];
    pz[q] = t.pts[3 * rr + 2];
  }
  double acc[2][NF][4];
#pragma unroll
  for (int rb = 0; rb < 2; rb++)
#pragma unroll
    for (int cb = 0; cb < NF; cb++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[rb][cb][q] = 0.;
  for (int e = t.e0; e < t.e1; e++) {
    const MfEntry en = ents[e];
    for (int k0 = 0; k0 < en.k; k0 += 16) {
      double a[2][8], b[NF][4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int c = k0 + t4 + 4 * j;
        const bool cv = c < en.k;
        const double* cp = en.pts + 3 * (i64)(cv ? c : 0);
        const double cx = __ldg(cp), cy = __ldg(cp + 1), cz = __ldg(cp + 2);
#pragma unroll
        for (int cb = 0; cb < NF; cb++)
          b[cb][j] = (cv && cb * 8 + g8 < nr) ? en.alpha * __ldg(en.B + c + (i64)(cb * 8 + g8) * en.ldb) : 0.;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          // row g8 + 8q: block q >> 1, fragment half q & 1
          const double v = kernel_eval_pair<KIND>(kp, px[q], py[q], pz[q], cx, cy, cz);
          a[q >> 1][2 * j + (q & 1)] = cv ? v : 0.;
        }
      }
#pragma unroll
      for (int rb = 0; rb < 2; rb++)
#pragma unroll
        for (int cb = 0; cb < NF; cb++)
          asm volatile(
              "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
              "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
              : "+d"(acc[rb][cb][0]), "+d"(acc[rb][cb][1]), "+d"(acc[rb][cb][2]), "+d"(acc[rb][cb][3])
              : "d"(a[rb][0]), "d"(a[rb][1]), "d"(a[rb][2]), "d"(a[rb][3]), "d"(a[rb][4]), "d"(a[rb][5]),
                "d"(a[rb][6]), "d"(a[rb][7]), "d"(b[cb][0]), "d"(b[cb][1]), "d"(b[cb][2]), "d"(b[cb][3]));
    }
  }
  // c[2h + q] of block rb: row 16 rb + g8 + 8h, column cb * 8 + 2 t4 + q.
#pragma unroll
  for (int rb = 0; rb < 2; rb++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = r0 + 16 * rb + g8 + 8 * h;
      if (r >= t.m) continue;
#pragma unroll
      for (int cb = 0; cb < NF; cb++)
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int c = cb * 8 + 2 * t4 + q;
          if (c >= nr) continue;
          double* o = t.C + r + (i64)c * t.ldc;
          *o = t.beta == 0. ? acc[rb][cb][2 * h + q] : t.beta * *o + acc[rb][cb][2 * h + q];
        }
    }
}

}  // namespace

int mf_rows_per_cta(int rpt) { return MF_NT * rpt; }
int mf_dmma_rows_per_cta() { return 32 * MFD_WARPS; }

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

template <int KIND>
static cudaError_t mf_dmma_go(const KernelParams& kp, int nr, const MfTask* d_tasks, const MfEntry* d_ents,
                              const int2* d_tiles, int ntiles, cudaStream_t st) {
  if (nr <= 8)
    k_mf_dmma<8, KIND><<<ntiles, 32 * MFD_WARPS, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr);
  else
    k_mf_dmma<16, KIND><<<ntiles, 32 * MFD_WARPS, 0, st>>>(kp, d_tasks, d_ents, d_tiles, nr);
  return cudaGetLastError();
}

template <int RPT>
static cudaError_t mf_kind(const KernelParams& kp, int nr, const MfTask* d_tasks, const MfEntry* d_ents,
                           const int2* d_tiles, int ntiles, cudaStream_t st) {
  if (RPT == 1 && nr > 4) {  // tiles of mf_dmma_rows_per_cta() rows
    if (kp.kind == KERNEL_LAPLACE) return mf_dmma_go<KERNEL_LAPLACE>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
    if (kp.kind == KERNEL_YUKAWA) return mf_dmma_go<KERNEL_YUKAWA>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
    if (kp.kind == KERNEL_HELMHOLTZ)
      return mf_dmma_go<KERNEL_HELMHOLTZ>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
    return mf_dmma_go<KERNEL_QUADRATIC>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
  }
  if (kp.kind == KERNEL_LAPLACE) return mf_go<KERNEL_LAPLACE, RPT>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
  if (kp.kind == KERNEL_YUKAWA) return mf_go<KERNEL_YUKAWA, RPT>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
  if (kp.kind == KERNEL_HELMHOLTZ) return mf_go<KERNEL_HELMHOLTZ, RPT>(kp, nr, d_tasks, d_ents, d_tiles, ntiles, st);
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
