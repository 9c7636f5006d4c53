// Shared device helpers for the H^2 solver kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace h2b {

typedef int64_t i64;

// KERNEL_QUADRATIC, K(d) = d^2 + alpha, has exactly low-rank (<= 6)
// off-diagonal blocks; with it the ULV factorization has no dropped fill and
// must reproduce the inverse, which is how the multilevel logic is verified.
//
// KERNEL_HELMHOLTZ is the complex kernel exp(-i k d)/d (kernel.hpp:63-74)
// solved in its real symmetric form: every body appears twice, as its real
// (component 0) and imaginary (component 1) unknown, and the real matrix
// entry between component p of body a and component q of body b is
//   p == q == 0: Re K(a, b);   p != q: Im K(a, b);   p == q == 1: -Re K(a, b).
// This form is symmetric because K is complex symmetric, and it maps y =
// conj(x) to K x (Re and Im interleaved, the std::complex<double> layout).
// The component travels with the body's coordinates as bit 0 of x (see
// helm_tag), so every copy and permutation of the body arrays keeps it.
enum KernelKind { KERNEL_LAPLACE = 0, KERNEL_YUKAWA = 1, KERNEL_QUADRATIC = 2, KERNEL_HELMHOLTZ = 3 };

// K(d) for d != 0, and the value used where two bodies coincide
// (kernel.hpp:28-50: Laplace 1/d, Yukawa exp(-alpha d)/d, diagonal 1/s).
struct KernelParams {
  int kind;
  double diag;
  double alpha;
};

// Distance exactly as libstdc++'s 3-argument std::hypot forms it
// (a * sqrt((x/a)^2 + (y/a)^2 + (z/a)^2) with a the largest magnitude),
// with every operation rounded separately so the result matches the
// reference's host build bit for bit.
__device__ __forceinline__ double hypot3_exact(double dx, double dy, double dz) {
  double x = fabs(dx), y = fabs(dy), z = fabs(dz);
  double a = x < y ? (y < z ? z : y) : (x < z ? z : x);
  if (a == 0.) return 0.;
  double sx = __ddiv_rn(x, a), sy = __ddiv_rn(y, a), sz = __ddiv_rn(z, a);
  double s = __dadd_rn(__dadd_rn(__dmul_rn(sx, sx), __dmul_rn(sy, sy)), __dmul_rn(sz, sz));
  return __dmul_rn(a, __dsqrt_rn(s));
}

__device__ __forceinline__ double kernel_exact(const KernelParams& kp, double dx, double dy, double dz) {
  double d = hypot3_exact(dx, dy, dz);
  if (d == 0.) return kp.diag;
  if (kp.kind == KERNEL_LAPLACE) return __ddiv_rn(1., d);
  if (kp.kind == KERNEL_QUADRATIC) return __dadd_rn(__dmul_rn(d, d), kp.alpha);
  return __ddiv_rn(exp(__dmul_rn(-kp.alpha, d)), d);
}

// Fast form for far-field samples and the dense verifier: one rsqrt of the
// squared distance; differs from the exact form by a few ulp.
__device__ __forceinline__ double kernel_fast(const KernelParams& kp, double dx, double dy, double dz) {
  double r2 = dx * dx + dy * dy + dz * dz;
  if (r2 == 0.) return kp.diag;
  if (kp.kind == KERNEL_QUADRATIC) return r2 + kp.alpha;
  double inv = rsqrt(r2);
  if (kp.kind == KERNEL_LAPLACE) return inv;
  return exp(-kp.alpha * (r2 * inv)) * inv;
}

// Helmholtz real form.  Component tag of a body coordinate (bit 0 of x) and
// the coordinate with the tag cleared; distances are always taken between
// cleared coordinates, so the two components of one body coincide.
__device__ __forceinline__ int helm_tag(double x) { return (int)(__double_as_longlong(x) & 1LL); }
__device__ __forceinline__ double helm_clear(double x) { return __longlong_as_double(__double_as_longlong(x) & ~1LL); }

// Real-form entry for a pair of tagged bodies (wave number kp.alpha, value
// 1/s at d == 0 as Helmholtz3D::operator()).  EXACT: distance by the
// separately rounded hypot and a correctly rounded division, as the FP64
// stored blocks use; otherwise one rsqrt of the squared distance.
template <bool EXACT>
__device__ __forceinline__ double helm_entry(const KernelParams& kp, double xi, double yi, double zi, double xj,
                                             double yj, double zj) {
  const int ti = helm_tag(xi), tj = helm_tag(xj);
  const double dx = helm_clear(xi) - helm_clear(xj), dy = yi - yj, dz = zi - zj;
  double re, im;
  if (EXACT) {
    const double d = hypot3_exact(dx, dy, dz);
    if (d == 0.) {
      re = kp.diag;
      im = 0.;
    } else {
      double s, c;
      sincos(kp.alpha * d, &s, &c);
      re = __ddiv_rn(c, d);
      im = -__ddiv_rn(s, d);
    }
  } else {
    const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
    if (r2 == 0.) {
      re = kp.diag;
      im = 0.;
    } else {
      const double inv = rsqrt(r2);
      double s, c;
      sincos(kp.alpha * (r2 * inv), &s, &c);
      re = c * inv;
      im = -s * inv;
    }
  }
  return ti != tj ? im : (ti ? -re : re);
}

// kernel_fast for a pair of bodies given by their coordinates (kind chosen
// at run time): the real kernels take the differences exactly as
// kernel_fast does; Helmholtz reads the component tags.
__device__ __forceinline__ double kernel_fast_pair(const KernelParams& kp, double xi, double yi, double zi,
                                                   double xj, double yj, double zj) {
  if (kp.kind == KERNEL_HELMHOLTZ) return helm_entry<false>(kp, xi, yi, zi, xj, yj, zj);
  return kernel_fast(kp, xi - xj, yi - yj, zi - zj);
}

// K(d) with the kernel kind fixed at compile time (no per-pair dispatch),
// for the matrix-free applies: one reciprocal square root per pair (the
// library's FP64 rsqrt measured faster on B200 than an FP32 seed refined by
// Newton steps, and is correctly rounded to about 1 ulp).
template <int KIND>
__device__ __forceinline__ double kernel_eval(const KernelParams& kp, double dx, double dy, double dz) {
  const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
  if (r2 == 0.) return kp.diag;
  if constexpr (KIND == KERNEL_QUADRATIC) return r2 + kp.alpha;
  const double inv = rsqrt(r2);
  if constexpr (KIND == KERNEL_LAPLACE) return inv;
  return exp(-kp.alpha * (r2 * inv)) * inv;
}

// kernel_eval for a pair of bodies given by their coordinates.
template <int KIND>
__device__ __forceinline__ double kernel_eval_pair(const KernelParams& kp, double xi, double yi, double zi, double xj,
                                                   double yj, double zj) {
  if constexpr (KIND == KERNEL_HELMHOLTZ) return helm_entry<false>(kp, xi, yi, zi, xj, yj, zj);
  return kernel_eval<KIND>(kp, xi - xj, yi - yj, zi - zj);
}

// Calls f(r, c, e) for every element e = r + c m of an m x n column-major
// range (m n < 2^31), consecutive threads of the CTA on consecutive rows:
// one division per thread, then division-free stepping.
template <typename F>
__device__ __forceinline__ void for_each_rc(int m, int n, F f) {
  if (m <= 0 || n <= 0) return;
  const int stride = (int)blockDim.x, total = m * n;
  const int dq = stride / m, dr = stride - dq * m;
  int e = (int)threadIdx.x;
  if (e >= total) return;
  int c = e / m, r = e - c * m;
  for (; e < total; e += stride) {
    f(r, c, e);
    r += dr;
    c += dq;
    if (r >= m) {
      r -= m;
      c++;
    }
  }
}

template <typename T>
struct BlockReduce {
  // Sum over a whole CTA (blockDim.x a multiple of 32, <= 1024).
  static __device__ T sum(T v, T* sbuf) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sbuf[w] = v;
    __syncthreads();
    int nw = blockDim.x >> 5;
    T r = (threadIdx.x < nw) ? sbuf[threadIdx.x] : T(0);
    if (w == 0)
      for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (threadIdx.x == 0) sbuf[0] = r;
    __syncthreads();
    T out = sbuf[0];
    __syncthreads();
    return out;
  }
};

// CTA-wide argmax of a double with the first index winning ties.
__device__ __forceinline__ void argmax_first(double& v, int& idx, double* sv, int* si) {
  for (int o = 16; o > 0; o >>= 1) {
    double ov = __shfl_xor_sync(0xffffffffu, v, o);
    int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
  }
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) { sv[w] = v; si[w] = idx; }
  __syncthreads();
  int nw = blockDim.x >> 5;
  if (w == 0) {
    double rv = (l < nw) ? sv[l] : -1.0;
    int ri = (l < nw) ? si[l] : 0x7fffffff;
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_xor_sync(0xffffffffu, rv, o);
      int oi = __shfl_xor_sync(0xffffffffu, ri, o);
      if (ov > rv || (ov == rv && oi < ri)) { rv = ov; ri = oi; }
    }
    if (l == 0) { sv[0] = rv; si[0] = ri; }
  }
  __syncthreads();
  v = sv[0];
  idx = si[0];
  __syncthreads();
}

// Host-side count of kernel launches made by this library (process-wide);
// every launcher calls note_launch() once per kernel it launches.
void note_launch();
long long launch_count();

}  // namespace h2b
