// Segmented batched GEMM: every output task C_t (m x n, column-major)
// receives beta * C_t + sum over its entries of alpha * op(A) op(B).  One
// CTA computes one BM x BN tile of one task; the task/tile list is built on
// the host once per level and reused.  This single kernel carries the ULV
// basis transforms and Schur updates (h2matrix.cpp:373-422), the H^2
// matvec passes (h2matrix.cpp:251-344) and the ULV substitution
// (h2matrix.cpp:448-537), with variable box sizes and ranks.
#include "common.cuh"
#include "kernels.h"

#include <cstdint>

namespace h2b {

template <typename T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) k_seg_gemm(const GemmTask<T>* __restrict__ tasks,
                                                                    const GemmEntry<T>* __restrict__ ents,
                                                                    const TileRef* __restrict__ tiles) {
  constexpr int NT = (BM / TM) * (BN / TN);
  constexpr int RG = BM / TM;  // row groups: thread row index fastest
  __shared__ T As[BK][BM + 1];
  __shared__ T Bs[BK][BN + 1];
  const TileRef tr = tiles[blockIdx.x];
  const GemmTask<T> task = tasks[tr.task];
  const int m0 = tr.tm * BM, n0 = tr.tn * BN;
  const int tid = threadIdx.x;
  const int tr_ = tid % RG, tc_ = tid / RG;
  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++) acc[i][j] = T(0);

  for (int e = task.e0; e < task.e1; e++) {
    const GemmEntry<T> en = ents[e];
    const int K = en.k;
    for (int k0 = 0; k0 < K; k0 += BK) {
      if (en.opA == 0) {
        for (int idx = tid; idx < BM * BK; idx += NT) {
          int mm = idx % BM, kk = idx / BM;
          int r = m0 + mm, k = k0 + kk;
          As[kk][mm] = (r < task.m && k < K) ? en.alpha * en.A[r + (i64)k * en.lda] : T(0);
        }
      } else {
        for (int idx = tid; idx < BM * BK; idx += NT) {
          int kk = idx % BK, mm = idx / BK;
          int r = m0 + mm, k = k0 + kk;
          As[kk][mm] = (r < task.m && k < K) ? en.alpha * en.A[k + (i64)r * en.lda] : T(0);
        }
      }
      if (en.opB == 0) {
        for (int idx = tid; idx < BN * BK; idx += NT) {
          int kk = idx % BK, nn = idx / BK;
          int c = n0 + nn, k = k0 + kk;
          Bs[kk][nn] = (c < task.n && k < K) ? en.B[k + (i64)c * en.ldb] : T(0);
        }
      } else {
        for (int idx = tid; idx < BN * BK; idx += NT) {
          int nn = idx % BN, kk = idx / BN;
          int c = n0 + nn, k = k0 + kk;
          Bs[kk][nn] = (c < task.n && k < K) ? en.B[c + (i64)k * en.ldb] : T(0);
        }
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < BK; kk++) {
        T a[TM], b[TN];
#pragma unroll
        for (int i = 0; i < TM; i++) a[i] = As[kk][tr_ + i * RG];
#pragma unroll
        for (int j = 0; j < TN; j++) b[j] = Bs[kk][tc_ + j * (BN / TN)];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
          for (int j = 0; j < TN; j++) acc[i][j] += a[i] * b[j];
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int j = 0; j < TN; j++) {
    int c = n0 + tc_ + j * (BN / TN);
    if (c >= task.n) continue;
#pragma unroll
    for (int i = 0; i < TM; i++) {
      int r = m0 + tr_ + i * RG;
      if (r >= task.m) continue;
      T* p = task.C + r + (i64)c * task.ldc;
      *p = (task.beta == T(0)) ? acc[i][j] : task.beta * (*p) + acc[i][j];
    }
  }
}

int gemm_tile_m(int shape) { return shape == GEMM_BIG ? 64 : 128; }
int gemm_tile_n(int shape) { return shape == GEMM_BIG ? 64 : 16; }

template <typename T>
cudaError_t launch_seg_gemm(int shape, const GemmTask<T>* d_tasks, const GemmEntry<T>* d_ents, const TileRef* d_tiles,
                            int ntiles, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  if (shape == GEMM_BIG) {
    note_launch();
    k_seg_gemm<T, 64, 64, 16, 4, 4><<<ntiles, 256, 0, st>>>(d_tasks, d_ents, d_tiles);
  } else {
    note_launch();
    k_seg_gemm<T, 128, 16, 16, 4, 2><<<ntiles, 256, 0, st>>>(d_tasks, d_ents, d_tiles);
  }
  return cudaGetLastError();
}
template cudaError_t launch_seg_gemm<double>(int, const GemmTask<double>*, const GemmEntry<double>*, const TileRef*,
                                             int, cudaStream_t);
template cudaError_t launch_seg_gemm<float>(int, const GemmTask<float>*, const GemmEntry<float>*, const TileRef*, int,
                                            cudaStream_t);

// One CTA per entry: dst (m x n, ld ldd) = src or src^T (ld lds).  Plain
// copies walk the elements column by column (consecutive threads on
// consecutive rows, one division per thread, none per element); transposed
// copies go through 32 x 32 shared-memory tiles so that both the reads of
// src and the writes of dst are coalesced.
template <typename T>
__global__ void __launch_bounds__(256) k_batched_copy(const CopyEntry<T>* __restrict__ ents) {
  const CopyEntry<T> e = ents[blockIdx.x];
  const int m = e.m, n = e.n;
  if (m <= 0 || n <= 0) return;
  if (!e.trans) {
    if ((i64)m * n < ((i64)1 << 31)) {
      const int stride = (int)blockDim.x, dq = stride / m, dr = stride - dq * m, total = m * n;
      int x = (int)threadIdx.x;
      int c = x / m, r = x - c * m;
      for (; x < total; x += stride) {
        e.dst[r + (i64)c * e.ldd] = e.src[r + (i64)c * e.lds];
        r += dr;
        c += dq;
        if (r >= m) {
          r -= m;
          c++;
        }
      }
    } else {
      for (i64 x = threadIdx.x; x < (i64)m * n; x += blockDim.x) {
        const int r = (int)(x % m), c = (int)(x / m);
        e.dst[r + (i64)c * e.ldd] = e.src[r + (i64)c * e.lds];
      }
    }
    return;
  }
  // dst(r, c) = src(c, r): the tile at dst rows r0.., columns c0.. is the
  // tile at src rows c0.., columns r0...
  __shared__ T tile[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 rows of 32 per pass
  for (int c0 = 0; c0 < n; c0 += 32)
    for (int r0 = 0; r0 < m; r0 += 32) {
      for (int i = ty; i < 32; i += 8) {
        const int sr = c0 + tx, sc = r0 + i;  // src(sr, sc) = dst(sc, sr)
        tile[i][tx] = (sr < n && sc < m) ? e.src[sr + (i64)sc * e.lds] : T(0);
      }
      __syncthreads();
      for (int i = ty; i < 32; i += 8) {
        const int dr = r0 + tx, dc = c0 + i;
        if (dr < m && dc < n) e.dst[dr + (i64)dc * e.ldd] = tile[tx][i];
      }
      __syncthreads();
    }
}

template <typename T>
cudaError_t launch_batched_copy(const CopyEntry<T>* d_ents, int n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  note_launch();
  k_batched_copy<T><<<n, 256, 0, st>>>(d_ents);
  return cudaGetLastError();
}
template cudaError_t launch_batched_copy<double>(const CopyEntry<double>*, int, cudaStream_t);
template cudaError_t launch_batched_copy<float>(const CopyEntry<float>*, int, cudaStream_t);

template <typename T>
__global__ void __launch_bounds__(256) k_set_identity(T* base, const i64* __restrict__ qoff, const i64* __restrict__ dims) {
  const int box = blockIdx.x;
  const i64 M = dims[box];
  T* q = base + qoff[box];
  for (i64 e = threadIdx.x; e < M * M; e += blockDim.x) q[e] = (e % M == e / M) ? T(1) : T(0);
}

template <typename T>
cudaError_t launch_set_identity(T* base, const i64* qoff, const i64* dims, int nboxes, cudaStream_t st) {
  if (nboxes == 0) return cudaSuccess;
  note_launch();
  k_set_identity<T><<<nboxes, 256, 0, st>>>(base, qoff, dims);
  return cudaGetLastError();
}
template cudaError_t launch_set_identity<double>(double*, const i64*, const i64*, int, cudaStream_t);
template cudaError_t launch_set_identity<float>(float*, const i64*, const i64*, int, cudaStream_t);

}  // namespace h2b

namespace h2b {

// Multi-right-hand-side block-sparse apply: C_task (m x n, n <= NR) =
// beta C + sum_e alpha_e A_e B_e with A_e and B_e as stored (column-major).
// This is the shape of every H^2 matvec pass and every ULV substitution
// step except the transposed ones, and it is bound by streaming A from HBM
// once.  One CTA (BM / 2 threads) covers BM = 128 or 256 rows of a task
// (tasks of at most 128 rows take the narrow variant).  The (entry, k-slab)
// sequence of the task is one stream of stages: each stage is a BM x KS
// slab of A and the KS x NR slab of B, copied by cp.async into a
// ST-deep shared-memory ring (16-byte copies where the column starts are
// 16-byte aligned, element copies otherwise; rows past m and k past K are
// zero-filled), so ST-1 slabs are in flight while one is multiplied.  Each
// thread owns two adjacent rows and all NR columns; B rows are read as
// shared-memory broadcasts.  alpha_e != 1 scales the B slab in place.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async_16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes));
}
template <int N>
__device__ __forceinline__ void cp_async_ca(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(smem_u32(dst)), "l"(src), "n"(N),
               "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename T>
struct StreamCfg;
template <>
struct StreamCfg<double> { static constexpr int KS = 8, ST = 3; };
template <>
struct StreamCfg<float> { static constexpr int KS = 16, ST = 3; };

template <typename T, int NR, int BM>
constexpr size_t stream_smem() {
  return sizeof(T) * (size_t)StreamCfg<T>::ST * StreamCfg<T>::KS * (BM + NR);
}

template <typename T, int NR, int BM>
__global__ void __launch_bounds__(BM / 2, 1024 / BM) k_stream_nn(const GemmTask<T>* __restrict__ tasks,
                                                      const GemmEntry<T>* __restrict__ ents,
                                                      const int2* __restrict__ tiles) {
  constexpr int KS = StreamCfg<T>::KS, ST = StreamCfg<T>::ST, NT = BM / 2;
  constexpr int V = 16 / sizeof(T);  // elements per 16-byte copy
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);  // [ST][KS][BM]
  T* Bs = As + (size_t)ST * KS * BM;       // [ST][KS][NR]
  const int2 tl = tiles[blockIdx.x];
  const GemmTask<T> task = tasks[tl.x];
  const int m0 = tl.y * BM;
  const int mrows = min(BM, task.m - m0);
  const int tid = threadIdx.x;

  // Producer cursor: next (entry, k0) to stage.
  int pe = task.e0, pk = 0;
  while (pe < task.e1 && ents[pe].k <= 0) pe++;
  auto issue = [&](int slot) {
    if (pe < task.e1) {
      const GemmEntry<T> en = ents[pe];
      T* as = As + (size_t)slot * KS * BM;
      T* bs = Bs + (size_t)slot * KS * NR;
      const bool vec = ((reinterpret_cast<uintptr_t>(en.A) & 15) == 0) && (en.lda % V == 0);
      if (vec) {
        for (int c = tid; c < KS * (BM / V); c += NT) {
          const int k = c / (BM / V), r = (c % (BM / V)) * V;
          int valid = mrows - r;
          valid = valid < 0 ? 0 : (valid > V ? V : valid);
          if (pk + k >= en.k) valid = 0;
          const T* src = valid ? en.A + (i64)(m0 + r) + (i64)(pk + k) * en.lda : en.A;
          cp_async_16(as + k * BM + r, src, valid * (int)sizeof(T));
        }
      } else {
        for (int c = tid; c < KS * BM; c += NT) {
          const int k = c / BM, r = c % BM;
          const bool ok = r < mrows && pk + k < en.k;
          const T* src = ok ? en.A + (i64)(m0 + r) + (i64)(pk + k) * en.lda : en.A;
          cp_async_ca<sizeof(T)>(as + k * BM + r, src, ok ? (int)sizeof(T) : 0);
        }
      }
      for (int c = tid; c < KS * NR; c += NT) {
        const int k = c / NR, j = c % NR;
        const bool ok = j < task.n && pk + k < en.k;
        const T* src = ok ? en.B + (i64)(pk + k) + (i64)j * en.ldb : en.B;
        cp_async_ca<sizeof(T)>(bs + c, src, ok ? (int)sizeof(T) : 0);
      }
      pk += KS;
      if (pk >= en.k) {
        pk = 0;
        pe++;
        while (pe < task.e1 && ents[pe].k <= 0) pe++;
      }
    }
    cp_async_commit();
  };

  T acc[2][NR];
#pragma unroll
  for (int t = 0; t < 2; t++)
#pragma unroll
    for (int j = 0; j < NR; j++) acc[t][j] = T(0);

#pragma unroll
  for (int s = 0; s < ST - 1; s++) issue(s);
  // Consumer cursor.
  int ce = task.e0, ck = 0;
  while (ce < task.e1 && ents[ce].k <= 0) ce++;
  int slot = 0;
  while (ce < task.e1) {
    const T alpha = ents[ce].alpha;
    cp_async_wait<ST - 2>();
    if (alpha != T(1)) {
      // Scale the B elements this thread copied into the slot.
      T* bs = Bs + (size_t)slot * KS * NR;
      for (int c = tid; c < KS * NR; c += NT) bs[c] *= alpha;
    }
    __syncthreads();
    issue((slot + ST - 1) % ST);
    const T* as = As + (size_t)slot * KS * BM + 2 * tid;
    const T* bs = Bs + (size_t)slot * KS * NR;
#pragma unroll
    for (int k = 0; k < KS; k++) {
      T a0, a1;
      if constexpr (sizeof(T) == 8) {
        const double2 v = *reinterpret_cast<const double2*>(as + k * BM);
        a0 = v.x;
        a1 = v.y;
      } else {
        const float2 v = *reinterpret_cast<const float2*>(as + k * BM);
        a0 = v.x;
        a1 = v.y;
      }
#pragma unroll
      for (int j = 0; j < NR; j++) {
        const T bj = bs[k * NR + j];
        acc[0][j] += a0 * bj;
        acc[1][j] += a1 * bj;
      }
    }
    ck += KS;
    if (ck >= ents[ce].k) {
      ck = 0;
      ce++;
      while (ce < task.e1 && ents[ce].k <= 0) ce++;
    }
    slot = (slot + 1) % ST;
  }
  cp_async_wait<0>();
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int r = 2 * tid + t;
    if (r >= mrows) continue;
#pragma unroll
    for (int j = 0; j < NR; j++) {
      if (j >= task.n) break;
      T* p = task.C + (m0 + r) + (i64)j * task.ldc;
      *p = (task.beta == T(0)) ? acc[t][j] : task.beta * (*p) + acc[t][j];
    }
  }
}

// FP64 variant of the streaming apply on the FP64 tensor cores (mma.sync
// m8n8k4 .f64) for 8 or 16 right-hand sides.  Same ring and cursors as
// k_stream_nn; each warp owns 32 rows x NR columns as 4 x (NR / 8) m8n8k4
// accumulators.  A slabs are stored [k][BM + 4] and B slabs [k][NR + 4]
// (doubles): the padding makes the fragment loads of a half-warp (4 k x 4
// rows or columns) hit 16 distinct bank pairs.  One MMA replaces 8 DFMA
// instructions per thread, so the apply is no longer issue-bound.
constexpr int SD_KS = 8, SD_ST = 3;

template <int NR, int BM>
constexpr size_t stream_dmma_smem() {
  return sizeof(double) * (size_t)SD_ST * SD_KS * ((BM + 4) + (NR + 4));
}

template <int NR, int BM>
__global__ void __launch_bounds__(BM, BM == 256 ? 3 : 6)
    k_stream_dmma(const GemmTask<double>* __restrict__ tasks, const GemmEntry<double>* __restrict__ ents,
                  const int2* __restrict__ tiles) {
  constexpr int NT = BM, AS = BM + 4, BS = NR + 4, NF = NR / 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* As = reinterpret_cast<double*>(smem_raw);  // [ST][KS][AS]
  double* Bs = As + (size_t)SD_ST * SD_KS * AS;       // [ST][KS][BS]
  const int2 tl = tiles[blockIdx.x];
  const GemmTask<double> task = tasks[tl.x];
  const int m0 = tl.y * BM;
  const int mrows = min(BM, task.m - m0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  int pe = task.e0, pk = 0;
  while (pe < task.e1 && ents[pe].k <= 0) pe++;
  auto issue = [&](int slot) {
    if (pe < task.e1) {
      const GemmEntry<double> en = ents[pe];
      double* as = As + (size_t)slot * SD_KS * AS;
      double* bs = Bs + (size_t)slot * SD_KS * BS;
      const bool vec = ((reinterpret_cast<uintptr_t>(en.A) & 15) == 0) && (en.lda % 2 == 0);
      if (vec) {
        for (int c = tid; c < SD_KS * (BM / 2); c += NT) {
          const int k = c / (BM / 2), r = (c % (BM / 2)) * 2;
          int valid = mrows - r;
          valid = valid < 0 ? 0 : (valid > 2 ? 2 : valid);
          if (pk + k >= en.k) valid = 0;
          const double* src = valid ? en.A + (i64)(m0 + r) + (i64)(pk + k) * en.lda : en.A;
          cp_async_16(as + k * AS + r, src, valid * 8);
        }
      } else {
        for (int c = tid; c < SD_KS * BM; c += NT) {
          const int k = c / BM, r = c % BM;
          const bool ok = r < mrows && pk + k < en.k;
          const double* src = ok ? en.A + (i64)(m0 + r) + (i64)(pk + k) * en.lda : en.A;
          cp_async_ca<8>(as + k * AS + r, src, ok ? 8 : 0);
        }
      }
      for (int c = tid; c < SD_KS * NR; c += NT) {
        const int k = c / NR, j = c % NR;
        const bool ok = j < task.n && pk + k < en.k;
        const double* src = ok ? en.B + (i64)(pk + k) + (i64)j * en.ldb : en.B;
        cp_async_ca<8>(bs + k * BS + j, src, ok ? 8 : 0);
      }
      pk += SD_KS;
      if (pk >= en.k) {
        pk = 0;
        pe++;
        while (pe < task.e1 && ents[pe].k <= 0) pe++;
      }
    }
    cp_async_commit();
  };

  double acc[4][NF][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < NF; j++) acc[i][j][0] = acc[i][j][1] = 0.;

#pragma unroll
  for (int s = 0; s < SD_ST - 1; s++) issue(s);
  int ce = task.e0, ck = 0;
  while (ce < task.e1 && ents[ce].k <= 0) ce++;
  int slot = 0;
  const int fr = lane >> 2, fk = lane & 3;
  while (ce < task.e1) {
    const double alpha = ents[ce].alpha;
    cp_async_wait<SD_ST - 2>();
    if (alpha != 1.) {
      double* bs = Bs + (size_t)slot * SD_KS * BS;
      for (int c = tid; c < SD_KS * NR; c += NT) bs[(c / NR) * BS + c % NR] *= alpha;
    }
    __syncthreads();
    issue((slot + SD_ST - 1) % SD_ST);
    const double* as = As + (size_t)slot * SD_KS * AS + fk * AS + warp * 32 + fr;
    const double* bs = Bs + (size_t)slot * SD_KS * BS + fk * BS + fr;
    // Row blocks past the task's last row hold zeros: their MMAs are skipped
    // (8-row granularity), so padded tiles cost no tensor-pipe time.
    const int mf = min(4, max(0, (mrows - warp * 32 + 7) / 8));
#pragma unroll
    for (int ks = 0; ks < SD_KS; ks += 4) {
      double a[4], b[NF];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = as[ks * AS + i * 8];
#pragma unroll
      for (int j = 0; j < NF; j++) b[j] = bs[ks * BS + j * 8];
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (i < mf)
#pragma unroll
          for (int j = 0; j < NF; j++)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                         : "+d"(acc[i][j][0]), "+d"(acc[i][j][1])
                         : "d"(a[i]), "d"(b[j]));
    }
    ck += SD_KS;
    if (ck >= ents[ce].k) {
      ck = 0;
      ce++;
      while (ce < task.e1 && ents[ce].k <= 0) ce++;
    }
    slot = (slot + 1) % SD_ST;
  }
  cp_async_wait<0>();
  // D fragment: lane holds row lane >> 2, columns 2 (lane & 3) + {0, 1}.
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = warp * 32 + i * 8 + fr;
    if (r >= mrows) continue;
#pragma unroll
    for (int j = 0; j < NF; j++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int c = j * 8 + 2 * fk + h;
        if (c < task.n) {
          double* p = task.C + (m0 + r) + (i64)c * task.ldc;
          *p = (task.beta == 0.) ? acc[i][j][h] : task.beta * (*p) + acc[i][j][h];
        }
      }
  }
}

// FP64 streaming apply, warp-specialised: one producer warp moves the A
// slabs with bulk asynchronous copies (cp.async.bulk, one per column of the
// tile, completion counted in bytes on the stage's mbarrier) and the B slabs
// with cp.async; BM / 32 consumer warps each own 32 rows x NR columns and
// only read shared memory and issue mma.sync m16n8k16 FP64.  Stages are
// handed over by mbarriers (full: the copies landed; empty: every active
// consumer warp is done with the stage), so no block barrier runs inside
// the loop.
//
// MMA row and k orders are chosen for 16-byte fragment loads: MMA row g
// (g + 8) of a 16-row block is tile row 2g (2g + 1), so a lane's two A rows
// are one 16-byte pair of the column-major slab; MMA k index t + 4j is slab
// column t + 4j.  A columns are stored BM + 4 doubles apart and B rows NR + 4
// apart, which puts the 8 lanes of an A quarter-warp load (and the 16 lanes
// of a B half-warp load) on distinct banks.
//
// Columns whose start is not 16-byte aligned (odd leading dimension or
// base) are copied element by element with cp.async by the producer lanes.
// A slab columns past the entry's K are not copied: their B rows are zero
// and the stale A values there are finite (the ring is zeroed at start), so
// they add nothing; rows past the tile's last row produce outputs that are
// not stored.  Every wait is bounded: an expired wait sets the CTA's abort
// flag and the error word, the loops end, and the producer waits (bounded)
// for its last stages' copies before the CTA exits.
constexpr int DT_KS = 16;

template <int NR, int BM, int ST>
constexpr size_t stream_dtma_smem() {
  return sizeof(double) * (size_t)ST * DT_KS * ((BM + 4) + (NR + 4)) + 16 * (size_t)(2 * ST + 2);
}

__device__ __forceinline__ void dt_arrive_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void dt_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void dt_bulk(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ bool dt_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(100000u)
      : "memory");
  return ok != 0;
}
// About two seconds of SM clock cycles.
constexpr long long DT_WAIT_CYCLES = 4000000000LL;
// Lane 0 waits for the phase (bounded; the abort flag ends the wait early),
// the warp learns the outcome.
__device__ __forceinline__ bool dt_warp_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int lane) {
  int ok = 1;
  if (lane == 0) {
    if (!dt_try(bar, parity)) {
      const long long t0 = clock64();
      while (!dt_try(bar, parity)) {
        if (*abort_flag) {
          ok = 0;
          break;
        }
        if (clock64() - t0 > DT_WAIT_CYCLES) {
          *abort_flag = 1;
          ok = 0;
          break;
        }
      }
    }
  }
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

template <int NR, int BM, int ST>
__global__ void __launch_bounds__(BM + 32) k_stream_dtma(const GemmTask<double>* __restrict__ tasks,
                                                         const GemmEntry<double>* __restrict__ ents,
                                                         const int2* __restrict__ tiles, int* __restrict__ err) {
  constexpr int NC = BM / 32, AS = BM + 4, BS = NR + 4, NF = NR / 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* As = reinterpret_cast<double*>(smem_raw);   // [ST][KS][AS]
  double* Bs = As + (size_t)ST * DT_KS * AS;          // [ST][KS][BS]
  uint64_t* full = reinterpret_cast<uint64_t*>(Bs + (size_t)ST * DT_KS * BS);
  uint64_t* empty = full + ST;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + ST);

  const int2 tl = tiles[blockIdx.x];
  const GemmTask<double> task = tasks[tl.x];
  const int m0 = tl.y * BM;
  const int mrows = min(BM, task.m - m0);
  const int nact = (mrows + 31) / 32;  // consumer warps with rows
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  for (int i = tid * 2; i < ST * DT_KS * AS; i += 2 * blockDim.x)
    *reinterpret_cast<double2*>(As + i) = make_double2(0., 0.);
  // The zeros (generic proxy) are ordered before the bulk copies (async proxy).
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (tid == 0) {
    for (int s = 0; s < ST; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 33;\n" ::"r"(smem_u32(&full[s])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&empty[s])), "r"(nact) : "memory");
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  if (warp == NC) {
    // ---- producer warp
    int pe = task.e0, pk = 0, g = 0;
    while (pe < task.e1 && ents[pe].k <= 0) pe++;
    const int rows2 = (mrows + 1) & ~1;
    while (pe < task.e1) {
      const int s = g % ST;
      if (g >= ST && !dt_warp_wait(smem_u32(&empty[s]), (uint32_t)(((g / ST) - 1) & 1), abort_flag, lane)) break;
      const GemmEntry<double> en = ents[pe];
      const int kv = min(DT_KS, en.k - pk);
      double* as = As + (size_t)s * DT_KS * AS;
      double* bs = Bs + (size_t)s * DT_KS * BS;
      const uint32_t fb = smem_u32(&full[s]);
      const bool aligned = ((reinterpret_cast<uintptr_t>(en.A) & 15) == 0) && ((en.lda & 1) == 0);
      if (aligned) {
        if (lane == 0) dt_arrive_expect(fb, (uint32_t)(kv * rows2 * 8));
        __syncwarp();
        if (lane < kv) dt_bulk(smem_u32(as + lane * AS), en.A + m0 + (i64)(pk + lane) * en.lda, (uint32_t)rows2 * 8, fb);
      } else {
        if (lane == 0) dt_arrive(fb);
        for (int c = 0; c < kv; c++)
          for (int r = lane; r < mrows; r += 32) cp_async_ca<8>(as + c * AS + r, en.A + m0 + r + (i64)(pk + c) * en.lda, 8);
      }
      for (int idx = lane; idx < DT_KS * NR; idx += 32) {
        const int k = idx % DT_KS, j = idx / DT_KS;
        const bool ok = k < kv && j < task.n;
        const double* src = ok ? en.B + (i64)(pk + k) + (i64)j * en.ldb : en.B;
        cp_async_ca<8>(bs + k * BS + j, src, ok ? 8 : 0);
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(fb) : "memory");
      g++;
      pk += DT_KS;
      if (pk >= en.k) {
        pk = 0;
        pe++;
        while (pe < task.e1 && ents[pe].k <= 0) pe++;
      }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (*abort_flag) {
      // Let the copies of the stages still in flight land before the CTA's
      // shared memory is released.
      for (int q = max(0, g - ST); q < g; q++) {
        if (lane == 0) {
          const long long t0 = clock64();
          while (!dt_try(smem_u32(&full[q % ST]), (uint32_t)((q / ST) & 1)) && clock64() - t0 < DT_WAIT_CYCLES) {
          }
        }
      }
      if (lane == 0 && err) atomicExch(err, 1);
    }
    return;
  }
  if (warp >= nact) return;

  // ---- consumer warp: rows m0 + 32 warp .. + 31
  double acc[2][NF][4];
#pragma unroll
  for (int rb = 0; rb < 2; rb++)
#pragma unroll
    for (int cb = 0; cb < NF; cb++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[rb][cb][q] = 0.;
  const int g8 = lane >> 2, t4 = lane & 3;
  const int wr = warp * 32;
  const int nrb = min(2, (mrows - wr + 15) / 16);  // 16-row blocks with rows
  int ce = task.e0, ck = 0, g = 0;
  while (ce < task.e1 && ents[ce].k <= 0) ce++;
  bool ok = true;
  while (ce < task.e1) {
    const int s = g % ST;
    if (!dt_warp_wait(smem_u32(&full[s]), (uint32_t)((g / ST) & 1), abort_flag, lane)) {
      ok = false;
      break;
    }
    const double alpha = ents[ce].alpha;
    const double* as = As + (size_t)s * DT_KS * AS + wr + 2 * g8;
    const double* bs = Bs + (size_t)s * DT_KS * BS + g8;
    double a[2][8], b[NF][4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
      for (int rb = 0; rb < 2; rb++) {
        const double2 v = *reinterpret_cast<const double2*>(as + (t4 + 4 * j) * AS + 16 * rb);
        a[rb][2 * j] = v.x;
        a[rb][2 * j + 1] = v.y;
      }
#pragma unroll
      for (int cb = 0; cb < NF; cb++) b[cb][j] = bs[(t4 + 4 * j) * BS + cb * 8];
    }
    if (alpha != 1.) {
#pragma unroll
      for (int cb = 0; cb < NF; cb++)
#pragma unroll
        for (int j = 0; j < 4; j++) b[cb][j] *= alpha;
    }
#pragma unroll
    for (int rb = 0; rb < 2; rb++)
      if (rb < nrb)
#pragma unroll
        for (int cb = 0; cb < NF; cb++)
          asm volatile(
              "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
              "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
              : "+d"(acc[rb][cb][0]), "+d"(acc[rb][cb][1]), "+d"(acc[rb][cb][2]), "+d"(acc[rb][cb][3])
              : "d"(a[rb][0]), "d"(a[rb][1]), "d"(a[rb][2]), "d"(a[rb][3]), "d"(a[rb][4]), "d"(a[rb][5]),
                "d"(a[rb][6]), "d"(a[rb][7]), "d"(b[cb][0]), "d"(b[cb][1]), "d"(b[cb][2]), "d"(b[cb][3]));
    __syncwarp();
    if (lane == 0) dt_arrive(smem_u32(&empty[s]));
    g++;
    ck += DT_KS;
    if (ck >= ents[ce].k) {
      ck = 0;
      ce++;
      while (ce < task.e1 && ents[ce].k <= 0) ce++;
    }
  }
  if (!ok) return;
  // D fragment of 16-row block rb: c[2h + q] is MMA row g8 + 8h (tile row
  // 2 g8 + h of the block), column 2 t4 + q of the column block.
#pragma unroll
  for (int rb = 0; rb < 2; rb++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = wr + 16 * rb + 2 * g8 + h;
      if (r >= mrows) continue;
#pragma unroll
      for (int cb = 0; cb < NF; cb++)
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int c = cb * 8 + 2 * t4 + q;
          if (c < task.n) {
            double* p = task.C + (m0 + r) + (i64)c * task.ldc;
            *p = (task.beta == 0.) ? acc[rb][cb][2 * h + q] : task.beta * (*p) + acc[rb][cb][2 * h + q];
          }
        }
    }
}

// FP32 variant of the streaming apply on the tensor cores through warp-level
// mma.sync m16n8k8 TF32 with the 3-term split (hi*hi + hi*lo + lo*hi, FP32
// accumulation: FP32 accuracy) for 8 or 16 right-hand sides.  Same ring and
// cursors as k_stream_nn; each warp owns 32 rows x NR columns as 2 x (NR / 8)
// m16n8 accumulators.  A slabs are stored [k][BM + 8] and B slabs [k][NR + 8]
// (floats) so each fragment load of a warp (8 rows x 4 k) hits 32 distinct
// banks.  The split happens in registers as fragments are loaded.
constexpr int SF_KS = 16, SF_ST = 3;

template <int NR, int BM>
constexpr size_t stream_tf32_smem() {
  return sizeof(float) * (size_t)SF_ST * SF_KS * ((BM + 8) + (NR + 8));
}

// hi: x as stored (the tensor core reads a TF32 operand from an FP32
// container by ignoring its 13 low mantissa bits); lo = x - trunc(x), exact.
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = __float_as_uint(x);
  lo = __float_as_uint(x - __uint_as_float(hi & 0xFFFFE000u));
}

__device__ __forceinline__ void mma_tf32_16x8x8(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <int NR, int BM>
__global__ void __launch_bounds__(BM, BM == 256 ? 3 : 6)
    k_stream_tf32(const GemmTask<float>* __restrict__ tasks, const GemmEntry<float>* __restrict__ ents,
                  const int2* __restrict__ tiles) {
  constexpr int NT = BM, AS = BM + 8, BS = NR + 8, NF = NR / 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* As = reinterpret_cast<float*>(smem_raw);  // [ST][KS][AS]
  float* Bs = As + (size_t)SF_ST * SF_KS * AS;      // [ST][KS][BS]
  const int2 tl = tiles[blockIdx.x];
  const GemmTask<float> task = tasks[tl.x];
  const int m0 = tl.y * BM;
  const int mrows = min(BM, task.m - m0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  int pe = task.e0, pk = 0;
  while (pe < task.e1 && ents[pe].k <= 0) pe++;
  auto issue = [&](int slot) {
    if (pe < task.e1) {
      const GemmEntry<float> en = ents[pe];
      float* as = As + (size_t)slot * SF_KS * AS;
      float* bs = Bs + (size_t)slot * SF_KS * BS;
      const bool vec = ((reinterpret_cast<uintptr_t>(en.A) & 15) == 0) && (en.lda % 4 == 0);
      if (vec) {
        for (int c = tid; c < SF_KS * (BM / 4); c += NT) {
          const int k = c / (BM / 4), r = (c % (BM / 4)) * 4;
          int valid = mrows - r;
          valid = valid < 0 ? 0 : (valid > 4 ? 4 : valid);
          if (pk + k >= en.k) valid = 0;
          const float* src = valid ? en.A + (i64)(m0 + r) + (i64)(pk + k) * en.lda : en.A;
          cp_async_16(as + k * AS + r, src, valid * 4);
        }
      } else {
        for (int c = tid; c < SF_KS * BM; c += NT) {
          const int k = c / BM, r = c % BM;
          const bool ok = r < mrows && pk + k < en.k;
          const float* src = ok ? en.A + (i64)(m0 + r) + (i64)(pk + k) * en.lda : en.A;
          cp_async_ca<4>(as + k * AS + r, src, ok ? 4 : 0);
        }
      }
      for (int c = tid; c < SF_KS * NR; c += NT) {
        const int k = c / NR, j = c % NR;
        const bool ok = j < task.n && pk + k < en.k;
        const float* src = ok ? en.B + (i64)(pk + k) + (i64)j * en.ldb : en.B;
        cp_async_ca<4>(bs + k * BS + j, src, ok ? 4 : 0);
      }
      pk += SF_KS;
      if (pk >= en.k) {
        pk = 0;
        pe++;
        while (pe < task.e1 && ents[pe].k <= 0) pe++;
      }
    }
    cp_async_commit();
  };

  float acc[2][NF][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < NF; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.f;

#pragma unroll
  for (int s = 0; s < SF_ST - 1; s++) issue(s);
  int ce = task.e0, ck = 0;
  while (ce < task.e1 && ents[ce].k <= 0) ce++;
  int slot = 0;
  const int g = lane >> 2, t4 = lane & 3;
  while (ce < task.e1) {
    const float alpha = ents[ce].alpha;
    cp_async_wait<SF_ST - 2>();
    if (alpha != 1.f) {
      float* bs = Bs + (size_t)slot * SF_KS * BS;
      for (int c = tid; c < SF_KS * NR; c += NT) bs[(c / NR) * BS + c % NR] *= alpha;
    }
    __syncthreads();
    issue((slot + SF_ST - 1) % SF_ST);
    const float* as = As + (size_t)slot * SF_KS * AS + warp * 32 + g;
    const float* bs = Bs + (size_t)slot * SF_KS * BS + g;
    const int mf = min(2, max(0, (mrows - warp * 32 + 15) / 16));  // live 16-row blocks
#pragma unroll
    for (int ks = 0; ks < SF_KS; ks += 8) {
      // A fragment of m16n8k8 (row): a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4).
      uint32_t ah[2][4], al[2][4];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const float* ap = as + i * 16 + (ks + t4) * AS;
        split_tf32(ap[0], ah[i][0], al[i][0]);
        split_tf32(ap[8], ah[i][1], al[i][1]);
        split_tf32(ap[4 * AS], ah[i][2], al[i][2]);
        split_tf32(ap[4 * AS + 8], ah[i][3], al[i][3]);
      }
      // B fragment (col): b0 (k = t, n = g), b1 (k = t + 4, n = g).
      uint32_t bh[NF][2], bl[NF][2];
#pragma unroll
      for (int j = 0; j < NF; j++) {
        const float* bp = bs + j * 8 + (ks + t4) * BS;
        split_tf32(bp[0], bh[j][0], bl[j][0]);
        split_tf32(bp[4 * BS], bh[j][1], bl[j][1]);
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
        if (i < mf)
#pragma unroll
          for (int j = 0; j < NF; j++) {
            mma_tf32_16x8x8(acc[i][j], al[i], bh[j]);
            mma_tf32_16x8x8(acc[i][j], ah[i], bl[j]);
            mma_tf32_16x8x8(acc[i][j], ah[i], bh[j]);
          }
    }
    ck += SF_KS;
    if (ck >= ents[ce].k) {
      ck = 0;
      ce++;
      while (ce < task.e1 && ents[ce].k <= 0) ce++;
    }
    slot = (slot + 1) % SF_ST;
  }
  cp_async_wait<0>();
  // C fragment: c0 (g, 2t), c1 (g, 2t + 1), c2 (g + 8, 2t), c3 (g + 8, 2t + 1).
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int hh = 0; hh < 2; hh++) {
      const int r = warp * 32 + i * 16 + g + 8 * hh;
      if (r >= mrows) continue;
#pragma unroll
      for (int j = 0; j < NF; j++)
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int c = j * 8 + 2 * t4 + q;
          if (c < task.n) {
            float* p = task.C + (m0 + r) + (i64)c * task.ldc;
            const float v = acc[i][j][2 * hh + q];
            *p = (task.beta == 0.f) ? v : task.beta * (*p) + v;
          }
        }
    }
}

// dst = beta * dst + sum_{p < parts} src_p, the parts of one split task
// summed in a fixed order (deterministic).  blockIdx.y strides over the
// tasks, blockIdx.x is a chunk of 1024 of a task's m x n elements
// (column-major).
template <typename T>
__global__ void __launch_bounds__(256) k_sum_parts(const SumTask<T>* __restrict__ tasks, int ntasks) {
  for (int ti = blockIdx.y; ti < ntasks; ti += gridDim.y) {
    const SumTask<T> t = tasks[ti];
    const int mn = t.m * t.n;
    const int e0 = blockIdx.x * 1024;
    if (e0 >= mn) continue;
    const int e1 = min(mn, e0 + 1024);
    for (int e = e0 + (int)threadIdx.x; e < e1; e += blockDim.x) {
      const int c = e / t.m, r = e - c * t.m;
      T s = T(0);
      for (int p = 0; p < t.parts; p++) s += t.src[(i64)p * mn + e];
      T* d = t.dst + r + (i64)c * t.ldd;
      *d = (t.beta == T(0)) ? s : t.beta * (*d) + s;
    }
  }
}

template <typename T>
cudaError_t launch_sum_parts(const SumTask<T>* d_tasks, int ntasks, int maxmn, cudaStream_t st) {
  if (ntasks == 0 || maxmn <= 0) return cudaSuccess;
  note_launch();
  const dim3 grid((maxmn + 1023) / 1024, ntasks < 65535 ? ntasks : 65535);
  k_sum_parts<T><<<grid, 256, 0, st>>>(d_tasks, ntasks);
  return cudaGetLastError();
}
template cudaError_t launch_sum_parts<double>(const SumTask<double>*, int, int, cudaStream_t);
template cudaError_t launch_sum_parts<float>(const SumTask<float>*, int, int, cudaStream_t);

}  // namespace h2b

namespace h2b {

int skinny_rows_per_cta(int wide) { return wide ? 256 : 128; }

template <typename T>
cudaError_t launch_skinny_nn(int nr, int wide, const GemmTask<T>* d_tasks, const GemmEntry<T>* d_ents,
                             const int2* d_tiles, int ntiles, cudaStream_t st, int* bulk_err) {
  if (ntiles == 0) return cudaSuccess;
  auto go_bulk = [&](auto kern, size_t smem, int threads) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    note_launch();
    kern<<<ntiles, threads, smem, st>>>(d_tasks, d_ents, d_tiles, bulk_err);
    return cudaGetLastError();
  };
  auto go = [&](auto kern, size_t smem, int threads) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    note_launch();
    kern<<<ntiles, threads, smem, st>>>(d_tasks, d_ents, d_tiles);
    return cudaGetLastError();
  };
  if constexpr (sizeof(T) == 4) {
    // FP32 with 5..16 right-hand sides: TF32 tensor-core variant (3-term split), BM threads.
    if (nr > 4 && nr <= 8) {
      if (wide) return go(k_stream_tf32<8, 256>, stream_tf32_smem<8, 256>(), 256);
      return go(k_stream_tf32<8, 128>, stream_tf32_smem<8, 128>(), 128);
    }
    if (nr > 8 && nr <= 16) {
      if (wide) return go(k_stream_tf32<16, 256>, stream_tf32_smem<16, 256>(), 256);
      return go(k_stream_tf32<16, 128>, stream_tf32_smem<16, 128>(), 128);
    }
  }
  if constexpr (sizeof(T) == 8) {
    // FP64 with 5..16 right-hand sides on the FP64 tensor cores: the
    // warp-specialised bulk-copy kernel (BM + 32 threads, three stages, two
    // CTAs per SM), or the cp.async ring (BM threads).
    if (bulk_err && nr > 4 && nr <= 16) {
      if (nr <= 8) {
        if (wide) return go_bulk(k_stream_dtma<8, 256, 3>, stream_dtma_smem<8, 256, 3>(), 288);
        return go_bulk(k_stream_dtma<8, 128, 3>, stream_dtma_smem<8, 128, 3>(), 160);
      }
      if (wide) return go_bulk(k_stream_dtma<16, 256, 3>, stream_dtma_smem<16, 256, 3>(), 288);
      return go_bulk(k_stream_dtma<16, 128, 3>, stream_dtma_smem<16, 128, 3>(), 160);
    }
    if (nr > 4 && nr <= 8) {
      if (wide) return go(k_stream_dmma<8, 256>, stream_dmma_smem<8, 256>(), 256);
      return go(k_stream_dmma<8, 128>, stream_dmma_smem<8, 128>(), 128);
    }
    if (nr > 8 && nr <= 16) {
      if (wide) return go(k_stream_dmma<16, 256>, stream_dmma_smem<16, 256>(), 256);
      return go(k_stream_dmma<16, 128>, stream_dmma_smem<16, 128>(), 128);
    }
  }
#define H2B_STREAM(NRV)                                                                  \
  if (nr <= NRV) {                                                                      \
    if (wide) return go(k_stream_nn<T, NRV, 256>, stream_smem<T, NRV, 256>(), 128);    \
    return go(k_stream_nn<T, NRV, 128>, stream_smem<T, NRV, 128>(), 64);               \
  }
  H2B_STREAM(1)
  H2B_STREAM(2)
  H2B_STREAM(4)
  H2B_STREAM(8)
  H2B_STREAM(16)
#undef H2B_STREAM
  return cudaErrorInvalidValue;
}
template cudaError_t launch_skinny_nn<double>(int, int, const GemmTask<double>*, const GemmEntry<double>*, const int2*,
                                              int, cudaStream_t, int*);
template cudaError_t launch_skinny_nn<float>(int, int, const GemmTask<float>*, const GemmEntry<float>*, const int2*,
                                             int, cudaStream_t, int*);

}  // namespace h2b
