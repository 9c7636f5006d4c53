// Batched FP64 Gram matrices G = X^T X (X: S x M column-major per box, the
// far-sample block of the fixed-rank basis construction) on the FP64 tensor
// cores (mma.sync m8n8k4 .f64).
//
// Only the upper-triangle 64 x 64 tiles of each G are computed; each
// off-diagonal tile is also written transposed.  One CTA (4 warps, each a
// 32 x 32 quadrant as 2 x 4 mma.sync m16n8k16 FP64 fragments) owns one tile.
// The k (sample) dimension is streamed in 16-row slabs through a 3-slot
// cp.async ring: the slab holds the tile's 64 (diagonal tile) or 128 columns
// of X, each column 16 consecutive samples padded to 18 doubles.  MMA k index
// t + 4j is slab sample 4t + j, so a lane's fragment values of one row (or
// column) are 4 consecutive samples: two 16-byte loads, which the 18-double
// column stride puts on distinct banks for each quarter warp.
#include "common.cuh"
#include "kernels.h"

#include <cstdint>

namespace h2b {

namespace {

constexpr int GR_T = 64, GR_KS = 16, GR_CS = GR_KS + 2, GR_ST = 3, GR_NT = 128;
constexpr int GR_KP = GR_KS / 2;  // 16-byte pairs per staged column
constexpr int GR_SLOT = 2 * GR_T * GR_CS;  // doubles per ring slot (128 columns)
constexpr int GR_SMEM = GR_ST * GR_SLOT * 8;

__device__ __forceinline__ uint32_t gsmem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void gcp16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void gcp8(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void gcommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void gwait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void dmma16(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

}  // namespace

__global__ void __launch_bounds__(GR_NT, 3) k_gram(const GramTask* __restrict__ tasks, const int4* __restrict__ tiles) {
  extern __shared__ __align__(16) double gsm[];
  const int4 tl = tiles[blockIdx.x];  // {task, tile row, tile col}
  const GramTask t = tasks[tl.x];
  const int c0 = tl.y * GR_T, c1 = tl.z * GR_T;
  const bool diag = tl.y == tl.z;
  const int ncol = diag ? GR_T : 2 * GR_T;  // columns staged per slab
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const bool vec = ((reinterpret_cast<uintptr_t>(t.X) & 15) == 0) && (t.ld % 2 == 0);
  const int nslab = (t.S + GR_KS - 1) / GR_KS;

  // Copies slab `sl` (samples sl*16 .. +15) into ring slot `slot`: staged
  // column j < 64 is X column c0 + j, column 64 + j is X column c1 + j.
  auto produce = [&](int sl, int slot) {
    if (sl < nslab) {
      double* dst = gsm + (size_t)slot * GR_SLOT;
      const int k0 = sl * GR_KS;
      for (int c = tid; c < ncol * GR_KP; c += GR_NT) {
        const int j = c / GR_KP, kk = (c % GR_KP) * 2;
        const int col = j < GR_T ? c0 + j : c1 + (j - GR_T);
        const int k = k0 + kk;
        int nk = t.S - k;
        nk = nk < 0 ? 0 : (nk > 2 ? 2 : nk);
        if (col >= t.M) nk = 0;
        const double* src = t.X + (i64)k + (i64)col * t.ld;
        const uint32_t d = gsmem(dst + j * GR_CS + kk);
        if (vec) {
          gcp16(d, nk ? (const void*)src : (const void*)t.X, nk * 8);
        } else {
          gcp8(d, nk > 0 ? (const void*)src : (const void*)t.X, nk > 0 ? 8 : 0);
          gcp8(d + 8, nk > 1 ? (const void*)(src + 1) : (const void*)t.X, nk > 1 ? 8 : 0);
        }
      }
    }
    gcommit();
  };

  double acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.;

#pragma unroll
  for (int s = 0; s < GR_ST - 1; s++) produce(s, s);
  const int g8 = lane >> 2, t4 = lane & 3;
  for (int sl = 0; sl < nslab; sl++) {
    gwait<GR_ST - 2>();
    __syncthreads();
    produce(sl + GR_ST - 1, (sl + GR_ST - 1) % GR_ST);
    const double* base = gsm + (size_t)(sl % GR_ST) * GR_SLOT;
    // A row (G row) c0 + wm 32 + 16 i + g8 + 8 h, samples 4 t4 .. 4 t4 + 3:
    // a[2 j + h] is sample 4 t4 + j (MMA row g8 + 8 h, MMA k t4 + 4 j).
    const double* as = base + (wm * 32 + g8) * GR_CS + 4 * t4;
    const double* bs = base + ((diag ? 0 : GR_T) + wn * 32 + g8) * GR_CS + 4 * t4;
    double a[2][8], b[4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const double* p = as + (16 * i + 8 * h) * GR_CS;
        const double2 x0 = *reinterpret_cast<const double2*>(p);
        const double2 x1 = *reinterpret_cast<const double2*>(p + 2);
        a[i][h] = x0.x;
        a[i][2 + h] = x0.y;
        a[i][4 + h] = x1.x;
        a[i][6 + h] = x1.y;
      }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const double* p = bs + 8 * j * GR_CS;
      const double2 x0 = *reinterpret_cast<const double2*>(p);
      const double2 x1 = *reinterpret_cast<const double2*>(p + 2);
      b[j][0] = x0.x;
      b[j][1] = x0.y;
      b[j][2] = x1.x;
      b[j][3] = x1.y;
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) dmma16(acc[i][j], a[i], b[j]);
  }
  gwait<0>();

  // D fragment of m16n8: c[2 h + q] is row g8 + 8 h, column 2 t4 + q.
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = c0 + wm * 32 + 16 * i + g8 + 8 * h;
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int c = c1 + wn * 32 + 8 * j + 2 * t4 + q;
          if (r < t.M && c < t.M) {
            t.G[(i64)r + (i64)c * t.ldg] = acc[i][j][2 * h + q];
            if (!diag) t.G[(i64)c + (i64)r * t.ldg] = acc[i][j][2 * h + q];
          }
        }
    }
}

int gram_tile() { return GR_T; }

cudaError_t launch_gram(const GramTask* d_tasks, const int4* d_tiles, int ntiles, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, GR_SMEM);
  if (e != cudaSuccess) return e;
  note_launch();
  k_gram<<<ntiles, GR_NT, GR_SMEM, st>>>(d_tasks, d_tiles);
  return cudaGetLastError();
}

}  // namespace h2b

namespace h2b {

// Segmented FP64 GEMM on the FP64 tensor cores: C_task = beta C_task + sum_e
// alpha_e op(A_e) op(B_e) over 64 x 64 output tiles (the FP64 plans of the
// factorization and basis completion).  Same ring and fragments as k_gram;
// each operand slab (16 k) is staged in the orientation it has in memory:
// k contiguous -> [row][20] (rows of 16 k, padded), rows contiguous ->
// [k][68] (k-rows of 64 rows, padded), so every cp.async is a 16-byte
// vector of consecutive elements and every fragment load of a half-warp hits
// 16 distinct bank pairs.
namespace {

constexpr int DG_T = 64, DG_KS = 16, DG_ST = 3, DG_NT = 128;
constexpr int DG_KP = DG_KS / 2;  // 16-byte pairs per k-contiguous row
constexpr int DG_RK = DG_KS + 4;  // [row][k] stride (doubles)
constexpr int DG_KR = 68;  // [k][row] stride (doubles)
constexpr int DG_OP = DG_T * DG_RK > DG_KS * DG_KR ? DG_T * DG_RK : DG_KS * DG_KR;  // doubles per operand
constexpr int DG_SMEM = DG_ST * 2 * DG_OP * 8;

struct DgOperand {
  const double* X;
  i64 ld;
  int rows, r0, k0, K;
  int kcontig;  // element (r, k) at X[k + r ld]; otherwise X[r + k ld]
  int vec;
};

__device__ __forceinline__ void dg_issue(const DgOperand& o, double* dst, int tid) {
  if (o.kcontig) {
    for (int c = tid; c < DG_T * DG_KP; c += DG_NT) {
      const int r = c / DG_KP, kk = (c % DG_KP) * 2;
      const int k = o.k0 + kk;
      int nk = o.K - k;
      nk = nk < 0 ? 0 : (nk > 2 ? 2 : nk);
      if (r >= o.rows) nk = 0;
      const double* src = o.X + (i64)k + (i64)(o.r0 + r) * o.ld;
      const uint32_t d = gsmem(dst + r * DG_RK + kk);
      if (o.vec) {
        gcp16(d, nk ? (const void*)src : (const void*)o.X, nk * 8);
      } else {
        gcp8(d, nk > 0 ? (const void*)src : (const void*)o.X, nk > 0 ? 8 : 0);
        gcp8(d + 8, nk > 1 ? (const void*)(src + 1) : (const void*)o.X, nk > 1 ? 8 : 0);
      }
    }
  } else {
    for (int c = tid; c < DG_KS * (DG_T / 2); c += DG_NT) {
      const int kk = c >> 5, r = (c & 31) * 2;
      const int k = o.k0 + kk;
      int nr = o.rows - r;
      nr = nr < 0 ? 0 : (nr > 2 ? 2 : nr);
      if (k >= o.K) nr = 0;
      const double* src = o.X + (i64)(o.r0 + r) + (i64)k * o.ld;
      const uint32_t d = gsmem(dst + kk * DG_KR + r);
      if (o.vec) {
        gcp16(d, nr ? (const void*)src : (const void*)o.X, nr * 8);
      } else {
        gcp8(d, nr > 0 ? (const void*)src : (const void*)o.X, nr > 0 ? 8 : 0);
        gcp8(d + 8, nr > 1 ? (const void*)(src + 1) : (const void*)o.X, nr > 1 ? 8 : 0);
      }
    }
  }
}

}  // namespace

__global__ void __launch_bounds__(DG_NT, 3) k_dgemm(const GemmTask<double>* __restrict__ tasks,
                                                   const GemmEntry<double>* __restrict__ ents,
                                                   const TileRef* __restrict__ tiles) {
  extern __shared__ __align__(16) double dsm[];
  const TileRef tl = tiles[blockIdx.x];
  const GemmTask<double> task = tasks[tl.task];
  const int m0 = tl.tm * DG_T, n0 = tl.tn * DG_T;
  const int mrows = min(DG_T, task.m - m0), ncols = min(DG_T, task.n - n0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int fr = lane >> 2, fk = lane & 3;

  int pe = task.e0, pk = 0;
  while (pe < task.e1 && ents[pe].k <= 0) pe++;
  auto produce = [&](int slot) {
    if (pe < task.e1) {
      const GemmEntry<double> en = ents[pe];
      double* base = dsm + (size_t)slot * 2 * DG_OP;
      DgOperand a, b;
      a.X = en.A; a.ld = en.lda; a.rows = mrows; a.r0 = m0; a.k0 = pk; a.K = en.k;
      a.kcontig = en.opA;  // op(A)(m, k) = A[k + m lda] when transposed
      a.vec = ((reinterpret_cast<uintptr_t>(en.A) & 15) == 0) && (en.lda % 2 == 0);
      b.X = en.B; b.ld = en.ldb; b.rows = ncols; b.r0 = n0; b.k0 = pk; b.K = en.k;
      b.kcontig = en.opB ? 0 : 1;  // op(B)(k, n) = B[k + n ldb] when not transposed
      b.vec = ((reinterpret_cast<uintptr_t>(en.B) & 15) == 0) && (en.ldb % 2 == 0);
      dg_issue(a, base, tid);
      dg_issue(b, base + DG_OP, tid);
      pk += DG_KS;
      if (pk >= en.k) {
        pk = 0;
        pe++;
        while (pe < task.e1 && ents[pe].k <= 0) pe++;
      }
    }
    gcommit();
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.;

#pragma unroll
  for (int s = 0; s < DG_ST - 1; s++) produce(s);
  int ce = task.e0, ck = 0, slot = 0;
  while (ce < task.e1 && ents[ce].k <= 0) ce++;
  while (ce < task.e1) {
    gwait<DG_ST - 2>();
    __syncthreads();
    produce((slot + DG_ST - 1) % DG_ST);
    const GemmEntry<double> en = ents[ce];
    const double* as = dsm + (size_t)slot * 2 * DG_OP;
    const double* bs = as + DG_OP;
    const int a_kc = en.opA, b_kc = en.opB ? 0 : 1;
    const double alpha = en.alpha;
#pragma unroll
    for (int ks = 0; ks < DG_KS; ks += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = wm * 32 + i * 8 + fr, k = ks + fk;
        a[i] = alpha * (a_kc ? as[r * DG_RK + k] : as[k * DG_KR + r]);
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int r = wn * 32 + j * 8 + fr, k = ks + fk;
        b[j] = b_kc ? bs[r * DG_RK + k] : bs[k * DG_KR + r];
      }
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) dmma(acc[i][j], a[i], b[j]);
    }
    ck += DG_KS;
    if (ck >= en.k) {
      ck = 0;
      ce++;
      while (ce < task.e1 && ents[ce].k <= 0) ce++;
    }
    slot = (slot + 1) % DG_ST;
  }
  gwait<0>();
  // D fragment of m8n8k4: lane holds row lane >> 2, columns 2 (lane & 3) + {0, 1}.
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = wm * 32 + i * 8 + fr;
    if (r >= mrows) continue;
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int c = wn * 32 + j * 8 + 2 * fk + h;
        if (c < ncols) {
          double* p = task.C + (i64)(m0 + r) + (i64)(n0 + c) * task.ldc;
          *p = (task.beta == 0.) ? acc[i][j][h] : task.beta * (*p) + acc[i][j][h];
        }
      }
  }
}

int dgemm_tile() { return DG_T; }

cudaError_t launch_dgemm(const GemmTask<double>* d_tasks, const GemmEntry<double>* d_ents, const TileRef* d_tiles,
                         int ntiles, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k_dgemm, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM);
  if (e != cudaSuccess) return e;
  note_launch();
  k_dgemm<<<ntiles, DG_NT, DG_SMEM, st>>>(d_tasks, d_ents, d_tiles);
  return cudaGetLastError();
}

}  // namespace h2b
