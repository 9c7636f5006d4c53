// Full-far-field random-sign sketch for the interpolative bases
// (compute_basis, h2matrix.cpp:13-63; build extension, sampling mode 2).
//
// The reference factors the whole far block XF = K(far bodies, box bodies)
// (S x M, S up to the number of bodies) with a Householder QR and runs the
// column-pivoted QR on its R.  Capping S by strided samples keeps the cost
// down but loses accuracy on the unsampled far bodies: the nearest far boxes
// carry most of the numerical rank and a stride of 1 in 16 misses it (at
// 262,144 points, 16,000 samples leave 2e-9 relative ID error where the
// whole far field gives 3e-12).  Here every far body is used, through the
// M x M product Y = Omega XF with a random-sign Omega: Y has the column
// geometry of XF up to the sketch's distortion, so the pivoted QR of Y picks
// skeletons and interpolation coefficients of nearly whole-far-field
// accuracy (randomized ID, Halko, Martinsson and Tropp 2011), and the cost is
// one GEMM of 2 M^2 S flops per box on the FP64 tensor cores with XF never
// stored: each 16-body slab of XF is generated into shared memory next to
// the 16 x 128 slab of signs it meets.
//
// Omega(a, f) = -1 when bit (a mod 64) of mix64(body_f * MUL_F + (a div 64) *
// MUL_W + ADD) is set, else +1 (splitmix64 finaliser); body_f is the body's
// index in the tree-sorted array, so the matrix does not depend on the order
// in which a box's far list is walked.  Boxes whose far list has at most M
// bodies take XF itself (compute_basis's K == N branch).
#include "common.cuh"
#include "kernels.h"

#include <cstdint>

namespace h2b {

namespace {

constexpr int SK_TM = 128, SK_TN = 64, SK_KS = 16, SK_CS = SK_KS + 4, SK_NT = 256;

__device__ __forceinline__ unsigned long long sk_mix64(unsigned long long z) {
  z ^= z >> 30;
  z *= 0xBF58476D1CE4E5B9ull;
  z ^= z >> 27;
  z *= 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ unsigned long long sk_word(i64 body, int w) {
  return sk_mix64((unsigned long long)body * 0x9E3779B97F4A7C15ull + (unsigned long long)w * 0xD1B54A32D192ED03ull +
                  0x2545F4914F6CDD1Dull);
}

__device__ __forceinline__ void sk_dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Body index of entry f (0 <= f < S) of a box's far list: ranges r0..r1-1
// hold [rstart[r], rstart[r] + count) with rend[r] the running count; the
// walk starts at a range known to begin at or before f.
__device__ __forceinline__ i64 sk_body(i64 f, i64 from, i64 r0, const i64* __restrict__ rstart,
                                       const i64* __restrict__ rend) {
  i64 r = from;
  while (f >= rend[r]) r++;
  return rstart[r] + (f - (r == r0 ? 0 : rend[r - 1]));
}

}  // namespace

// One CTA per {box, 128-row tile, 64-column tile} of Y (row-major M x M per
// box at Rws + qoff[box], the layout k_cpqr reads).  8 warps as 4 x 2 tiles
// of 32 x 32 (4 x 4 m8n8k4 fragments each).  Per 16-body slab: every thread
// evaluates 4 entries of XF (its column fixed, so the box body stays in
// registers) into a [column][20] shared tile laid out like the fragment
// loads, 32 threads form the slab's 16 x 2 sign words, 16 threads fetch the
// next slab's far bodies; one barrier per slab with two buffers.
template <typename T>
__global__ void __launch_bounds__(SK_NT, 2)
    k_sketch(KernelParams kp, const double* __restrict__ bodies, const double* __restrict__ pts,
             const i64* __restrict__ xoff, const i64* __restrict__ dims, const i64* __restrict__ qoff,
             const i64* __restrict__ roff, const i64* __restrict__ rstart, const i64* __restrict__ rend,
             const int4* __restrict__ tiles, T* __restrict__ Rws) {
  __shared__ __align__(16) double xf[2][SK_TN * SK_CS];
  __shared__ double fc[2][SK_KS * 3];
  __shared__ i64 fb[2][SK_KS];
  __shared__ unsigned long long sw[2][SK_KS][2];

  const int4 tl = tiles[blockIdx.x];
  const int box = tl.x;
  const int M = (int)dims[box];
  const int a0 = tl.y * SK_TM, c0 = tl.z * SK_TN;
  const i64 r0 = roff[box], r1 = roff[box + 1];
  const i64 S = r1 > r0 ? rend[r1 - 1] : 0;
  T* W = Rws + qoff[box];
  const double* X = pts + 3 * xoff[box];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (M == 0 || S == 0) return;

  if (S <= (i64)M) {
    // Whole far block: rows a < S of W are K(F_a, X_c).
    for (int e = tid; e < SK_TM * SK_TN; e += SK_NT) {
      const int a = a0 + e / SK_TN, c = c0 + e % SK_TN;
      if ((i64)a >= S || c >= M) continue;
      const i64 body = sk_body(a, r0, r0, rstart, rend);
      W[(i64)a * M + c] = (T)kernel_fast_pair(kp, bodies[3 * body], bodies[3 * body + 1], bodies[3 * body + 2],
                                              X[3 * c], X[3 * c + 1], X[3 * c + 2]);
    }
    return;
  }

  const int cl = warp * 8 + (lane >> 2);
  const int c = c0 + cl;
  const bool cv = c < M;
  double x0 = 0., x1 = 0., x2 = 0.;
  if (cv) {
    x0 = X[3 * c];
    x1 = X[3 * c + 1];
    x2 = X[3 * c + 2];
  }
  const int wm = warp >> 1, wn = warp & 1;
  const int nslab = (int)((S + SK_KS - 1) / SK_KS);
  i64 cur = r0;  // uniform: a range that starts at or before the slab being fetched

  auto fetch = [&](int sl, int b) {
    const i64 k0 = (i64)sl * SK_KS;
    while (cur < r1 - 1 && rend[cur] <= k0) cur++;
    if (tid < SK_KS) {
      const i64 f = k0 + tid;
      i64 body = -1;
      if (f < S) body = sk_body(f, cur, r0, rstart, rend);
      fb[b][tid] = body;
      fc[b][3 * tid] = body >= 0 ? bodies[3 * body] : 0.;
      fc[b][3 * tid + 1] = body >= 0 ? bodies[3 * body + 1] : 0.;
      fc[b][3 * tid + 2] = body >= 0 ? bodies[3 * body + 2] : 0.;
    }
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.;

  fetch(0, 0);
  __syncthreads();
  const int wsel = wm >> 1;                       // which 64-row sign word of the 128-row tile
  const int bit0 = (wm & 1) * 32 + (lane >> 2);   // fragment row's bit in that word
  for (int sl = 0; sl < nslab; sl++) {
    const int b = sl & 1;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int fl = e * 4 + (lane & 3);
      double v = 0.;
      if (cv && fb[b][fl] >= 0)
        v = kernel_fast_pair(kp, fc[b][3 * fl], fc[b][3 * fl + 1], fc[b][3 * fl + 2], x0, x1, x2);
      xf[b][cl * SK_CS + fl] = v;
    }
    if (tid >= 32 && tid < 64) {
      const int f = (tid - 32) & 15, w = (tid - 32) >> 4;
      const i64 body = fb[b][f];
      sw[b][f][w] = body >= 0 ? sk_word(body, (a0 >> 6) + w) : 0ull;
    }
    if (sl + 1 < nslab) fetch(sl + 1, b ^ 1);
    __syncthreads();
    const double* bs = xf[b] + (wn * 32 + (lane >> 2)) * SK_CS + (lane & 3);
#pragma unroll
    for (int ks = 0; ks < SK_KS; ks += 4) {
      const unsigned long long word = sw[b][ks + (lane & 3)][wsel];
      double av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; i++) av[i] = ((word >> (bit0 + 8 * i)) & 1ull) ? -1. : 1.;
#pragma unroll
      for (int j = 0; j < 4; j++) bv[j] = bs[j * 8 * SK_CS + ks];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) sk_dmma(acc[i][j], av[i], bv[j]);
    }
  }

  // D fragment of m8n8k4: lane holds row lane >> 2, columns 2 (lane & 3) + {0, 1}.
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int a = a0 + wm * 32 + i * 8 + (lane >> 2);
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int col = c0 + wn * 32 + j * 8 + 2 * (lane & 3) + h;
        if (a < M && col < M) W[(i64)a * M + col] = (T)acc[i][j][h];
      }
  }
}

int sketch_tile_rows() { return SK_TM; }
int sketch_tile_cols() { return SK_TN; }

template <typename T>
cudaError_t launch_sketch(const KernelParams& kp, const double* bodies, const double* pts, const i64* xoff,
                          const i64* dims, const i64* qoff, const i64* roff, const i64* rstart, const i64* rend,
                          const int4* d_tiles, int ntiles, T* Rws, cudaStream_t st) {
  if (ntiles == 0) return cudaSuccess;
  note_launch();
  k_sketch<T><<<ntiles, SK_NT, 0, st>>>(kp, bodies, pts, xoff, dims, qoff, roff, rstart, rend, d_tiles, Rws);
  return cudaGetLastError();
}

template cudaError_t launch_sketch<double>(const KernelParams&, const double*, const double*, const i64*, const i64*,
                                           const i64*, const i64*, const i64*, const i64*, const int4*, int, double*,
                                           cudaStream_t);
template cudaError_t launch_sketch<float>(const KernelParams&, const double*, const double*, const i64*, const i64*,
                                          const i64*, const i64*, const i64*, const i64*, const int4*, int, float*,
                                          cudaStream_t);

}  // namespace h2b
