// Launch interfaces of the device kernels (host-callable, no torch types).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace h2b {

// ---------------------------------------------------------------- gen
struct GenTask {
  const double* bi;  // m bodies, xyz interleaved
  const double* bj;  // n bodies
  int m, n;
  i64 out_off;  // element offset of the column-major m x n output
  i64 ld;
};
// max_m: the largest task row count (one CTA per 256 rows of a task); fast:
// rsqrt of the squared distance instead of the std::hypot-exact form; err:
// device int set if a CTA's bounded wait on its bulk copy expired (then the
// CTA fell back to plain loads, and the result is still complete).
template <typename T>
cudaError_t launch_gen_blocks(const KernelParams& kp, const GenTask* d_tasks, int ntasks, i64 max_m, T* out,
                              cudaStream_t st, int fast = 0, int* err = nullptr);
cudaError_t launch_dense_matvec(const KernelParams& kp, const double* bodies, i64 n, const double* X, i64 ldx,
                                double* Y, i64 ldy, int nrhs, cudaStream_t st);

// ---------------------------------------------------------------- basis
template <typename T>
cudaError_t launch_sample_tsqr(const KernelParams& kp, const double* bodies, const double* pts, const i64* xoff,
                               const i64* dims, const int* sidx, const i64* soff, T* Rws, const i64* qoff,
                               int nboxes, int maxM, cudaStream_t st);
// Full-far-field sketch (k_sketch.cu): Rws[box] (row-major M x M) = Omega XF
// over every far body (ranges roff[box]..roff[box+1]-1 of rstart / rend), or
// the first S rows = XF when S <= M.  tiles: {box, row tile, column tile}.
template <typename T>
cudaError_t launch_sketch(const KernelParams& kp, const double* bodies, const double* pts, const i64* xoff,
                          const i64* dims, const i64* qoff, const i64* roff, const i64* rstart, const i64* rend,
                          const int4* d_tiles, int ntiles, T* Rws, cudaStream_t st);
int sketch_tile_rows();
int sketch_tile_cols();
template <typename T>
cudaError_t launch_cpqr(const i64* dims, const i64* krows, T* Rws, const i64* qoff, int* perm, const i64* xoff,
                        double* maxpiv, int* nonzero, i64 step_cap, int nboxes, int maxM, cudaStream_t st);
template <typename T>
cudaError_t launch_basis_finish(const i64* dims, const i64* krows, T* Rws, T* Q, T* R, const i64* qoff,
                                const int* perm, const i64* xoff, const double* maxpiv, const int* nonzero,
                                double* pts, i64* ranks, double epi, int orth, int qin_identity, int nboxes,
                                int maxM, cudaStream_t st, T* wy_taus = nullptr);
// Compact-WY T matrix per box (see k_wy_t).
template <typename T>
struct WyTask {
  const T* S;     // r x r, V^T V
  const T* taus;  // r
  T* Tm;          // r x r output (upper triangular)
  int r;
};
// One Householder panel per box (k_qr_panel).
template <typename T>
struct QrPanelTask {
  T* W;      // M x rank, column-major (ld M)
  T* Vp;     // (M - k0) x nb explicit V of the panel
  T* Tp;     // nb x nb
  T* taus;   // per box, indexed by column
  int M, k0, nb;
};
template <typename T>
cudaError_t launch_qr_panel(const QrPanelTask<T>* d_tasks, int ntasks, int maxm, int nb, cudaStream_t st);
template <typename T>
struct QrExtractTask {
  T* W;
  T* R;
  T* Q;
  int M, rank;
};
template <typename T>
cudaError_t launch_qr_extract(const QrExtractTask<T>* d_tasks, int ntasks, cudaStream_t st);
template <typename T>
cudaError_t launch_wy_t(const WyTask<T>* d_tasks, int ntasks, int maxr, cudaStream_t st);

// Blocked pivoted Cholesky: one panel of nb pivots starting at k0 for every
// box (steps_box[i] pivots in all); state holds 3 doubles per box.
cudaError_t launch_pivchol_panel(const i64* dims, const i64* steps_box, double* G, double* Rws, const i64* qoff,
                                 int* perm, const i64* xoff, double* state, int k0, int nb, int nboxes, int maxM,
                                 cudaStream_t st);
cudaError_t launch_gather_points(const double* bodies, const int* idx, i64 n, double* out, cudaStream_t st);
// Gram matrix G = X^T X of one box (k_gram): X is S x M column-major.
struct GramTask {
  const double* X;
  i64 ld;
  int S, M;
  double* G;
  i64 ldg;
};
// tiles: {task, tile row, tile col} with tile row <= tile col, gram_tile() wide.
cudaError_t launch_gram(const GramTask* d_tasks, const int4* d_tiles, int ntiles, cudaStream_t st);
int gram_tile();

// ---------------------------------------------------------------- gemm
// C_task = beta * C_task + sum_{e in task} alpha_e * op(A_e) * op(B_e)
template <typename T>
struct GemmEntry {
  const T* A;
  const T* B;
  i64 lda, ldb;
  int k;
  int opA, opB;  // 0: as stored (column-major), 1: transposed
  T alpha;
};
template <typename T>
struct GemmTask {
  T* C;
  i64 ldc;
  int m, n;
  int e0, e1;
  T beta;
};
struct TileRef {
  int task, tm, tn;
};
enum GemmShape { GEMM_BIG = 0, GEMM_SKINNY = 1, GEMM_TC = 2 };
template <typename T>
cudaError_t launch_seg_gemm(int shape, const GemmTask<T>* d_tasks, const GemmEntry<T>* d_ents, const TileRef* d_tiles,
                            int ntiles, cudaStream_t st);
int gemm_tile_m(int shape);
// Plans whose entries all use A and B as stored and whose outputs have at
// most 16 columns: A streamed from HBM through a shared-memory ring, one CTA
// per skinny_rows_per_cta(wide) rows of a task (tile = {task, row block});
// wide = 0 for tasks of at most 128 rows, 1 otherwise.  FP64 plans with 5-16
// columns given bulk_err (a device int) run the warp-specialised bulk-copy
// kernel, which wants every A column start 16-byte aligned for full speed
// and sets *bulk_err when one of its mbarrier waits expires; without
// bulk_err they run the cp.async ring.
template <typename T>
cudaError_t launch_skinny_nn(int nr, int wide, const GemmTask<T>* d_tasks, const GemmEntry<T>* d_ents,
                             const int2* d_tiles, int ntiles, cudaStream_t st, int* bulk_err = nullptr);
int skinny_rows_per_cta(int wide);
// Reduction of a split task: dst (m x n, ld ldd) = beta dst + sum of `parts`
// consecutive m x n partial results at src.
template <typename T>
struct SumTask {
  T* dst;
  i64 ldd;
  const T* src;
  int m, n, parts;
  T beta;
};
template <typename T>
cudaError_t launch_sum_parts(const SumTask<T>* d_tasks, int ntasks, int maxmn, cudaStream_t st);
int gemm_tile_n(int shape);
// FP32 segmented GEMM on the tcgen05 tensor cores, 128 x 128 output tiles
// (TileRef over tc_gemm_tile()-sized tiles); split = 1: 3-term TF32 split
// (FP32 accuracy), 0: one TF32 product.  A CTA whose bounded wait expired
// sets *err to 1 (err: a device int owned by the caller, may be null).
cudaError_t launch_tc_gemm(const GemmTask<float>* d_tasks, const GemmEntry<float>* d_ents, const TileRef* d_tiles,
                           int ntiles, int split, int* err, cudaStream_t st);
int tc_gemm_tile();
// FP64 segmented GEMM on the FP64 tensor cores (mma.sync m8n8k4), 64 x 64
// output tiles (TileRef over dgemm_tile()-sized tiles).
cudaError_t launch_dgemm(const GemmTask<double>* d_tasks, const GemmEntry<double>* d_ents, const TileRef* d_tiles,
                         int ntiles, cudaStream_t st);
int dgemm_tile();

// Matrix-free block apply (k_mf.cu), FP64: C = beta C + sum over the task's
// entries of alpha K(pts_task, pts_entry) B (m x nr output, ld ldc; B k x nr,
// ld ldb; points xyz-interleaved).  tiles: {task, block of
// mf_rows_per_cta(rpt) rows}; nr <= 16.  With rpt 1 and nr > 4 the block is
// generated into FP64 tensor-core fragments (k_mf_dmma, tiles of
// mf_dmma_rows_per_cta() rows), otherwise each thread accumulates rpt rows
// on the FP64 FMA pipe.
struct MfTask {
  const double* pts;
  int m;
  double* C;
  i64 ldc;
  int e0, e1;
  double beta;
};
struct MfEntry {
  const double* pts;
  int k;
  const double* B;
  i64 ldb;
  double alpha;
};
cudaError_t launch_mf_apply(const KernelParams& kp, int nr, int rpt, const MfTask* d_tasks, const MfEntry* d_ents,
                            const int2* d_tiles, int ntiles, cudaStream_t st);
// Rows of a task one CTA covers with rpt (1 or 2) rows per thread.
int mf_rows_per_cta(int rpt);
int mf_dmma_rows_per_cta();

// BF16 substitution blocks (k_bf16.cu).  Pack: dst (m x k, ld ldd, a
// multiple of 8) = bf16(src / s), s = 2^ceil(log2 max |src|) written to
// *scale.  Apply: GemmTask<float> tasks with BfEntry entries, C = beta C +
// sum_e (alpha_e *scale_e) A_e B_e (A_e BF16 packed, B_e FP32 k x n);
// tiles {task, block of bf16_rows_per_cta() rows}; n <= 16.
struct BfPackTask {
  const float* src;
  i64 lds;
  int m, k;
  __nv_bfloat16* dst;
  i64 ldd;
  float* scale;
};
struct BfEntry {
  const __nv_bfloat16* A;
  i64 lda;
  const float* B;
  i64 ldb;
  int k;
  float alpha;
  const float* scale;
};
cudaError_t launch_bf16_pack(const BfPackTask* d_tasks, int ntasks, cudaStream_t st);
// 5-16 right-hand sides run on the BF16 tensor cores (k_stream_bf16_mma),
// 1-4 on the FMA pipe.
cudaError_t launch_stream_bf16(int nr, const GemmTask<float>* d_tasks, const BfEntry* d_ents, const int2* d_tiles,
                               int ntiles, cudaStream_t st);
int bf16_rows_per_cta();

template <typename T>
struct CopyEntry {
  const T* src;
  T* dst;
  i64 lds, ldd;
  int m, n;
  int trans;  // dst(r, c) = trans ? src(c, r) : src(r, c)
};
template <typename T>
cudaError_t launch_batched_copy(const CopyEntry<T>* d_ents, int n, cudaStream_t st);
template <typename T>
cudaError_t launch_set_identity(T* base, const i64* qoff, const i64* dims, int nboxes, cudaStream_t st);

// ---------------------------------------------------------------- lu
template <typename T>
struct LuTask {
  T* A;      // n x n column-major (read only)
  i64 lda;
  int n;
  T* invT;   // receives A^{-1} transposed (column-major, ld = ldinv)
  i64 ldinv;
  int* ipiv;  // n
  int* info;  // 1 when |det| <= DBL_MIN (h2matrix.cpp:384)
};
template <typename T>
cudaError_t launch_lu_inverse(const LuTask<T>* d_tasks, int ntasks, int maxn, cudaStream_t st);
// PartialPivLU of A (n x n) and X = A^{-1} B for m right-hand sides stored
// row by row: B[c + r ldb], X[c + r ldx] (r < n, c < m).  work: n x n scratch
// (ld n) used when the factor does not fit in shared memory.
template <typename T>
struct LuSolveTask {
  const T* A;
  i64 lda;
  int n;
  const T* B;
  i64 ldb;
  int m;
  T* X;
  i64 ldx;
  T* work;
  int* ipiv;
  int* info;
};
template <typename T>
cudaError_t launch_lu_solve(const LuSolveTask<T>* d_tasks, int ntasks, int maxn, cudaStream_t st);

// ---------------------------------------------------------------- vectors
template <typename Ts, typename Td>
cudaError_t launch_convert(const Ts* src, Td* dst, i64 n, cudaStream_t st);
cudaError_t launch_dots(const double* V, i64 vstride, int kvec, const double* w, i64 n, int nrhs, double* partial,
                        int nchunks, double* out, cudaStream_t st);
int dots_chunks(i64 n);
cudaError_t launch_gs_update(double* w, const double* V, i64 vstride, const double* h, i64 hstride, int kvec, i64 n,
                             int nrhs, double sign, const int* active, cudaStream_t st, const int* kdev = nullptr);
cudaError_t launch_dots_strided(const double* V, i64 vstride, int kvec, const double* w, i64 n, int nrhs,
                                double* partial, int nchunks, double* out, i64 ostride, cudaStream_t st);
// Device-side GMRES control (k_vec.cu); ctl = {used, stop, cycles, again}.
cudaError_t launch_gmres_init(int* act, int* it, double* resh, int outer, double tol, int nrhs, int* ctl,
                              cudaStream_t st);
cudaError_t launch_gmres_cycle_begin(int* ctl, int inner, cudaStream_t st);
cudaError_t launch_gmres_estimate(const double* H, int ldh, int inner, int i, const double* beta, const double* normb,
                                  const int* act, int nrhs, double tol, int* ctl, cudaStream_t st);
cudaError_t launch_gmres_cycle_end(const double* rvec, int* act, int* it, double* resh, int outer, double tol,
                                   int nrhs, int* ctl, cudaStream_t st);
// ctl[4] = some active column needs its true residual (recurrence residual below tol, or last cycle).
cudaError_t launch_gmres_need_true(const double* rvec, const int* act, const int* it, int outer, int nrhs, double tol,
                                   int* ctl, cudaStream_t st);
// Conditional node value of a captured graph = (*word != 0) xor invert.
cudaError_t launch_graph_condition(cudaGraphConditionalHandle handle, const int* word, int invert, cudaStream_t st);
cudaError_t launch_scale_by_norm(const double* w, double* vout, const double* nrm2, double* hout, i64 hstride,
                                 i64 n, int nrhs, cudaStream_t st);
cudaError_t launch_gmres_ls(const double* H, int ld, int inner, const double* beta, double* y, int nrhs,
                            cudaStream_t st, const int* used = nullptr);
// Helmholtz real form: tagged bodies (comps = 2: 2n x 3, both components; 1: n x 3, real part only).
cudaError_t launch_helm_expand(const double* bodies, i64 n, int comps, double* out, cudaStream_t st);
// Complex conjugate of a column-major array of interleaved (re, im) pairs (n doubles per column).
cudaError_t launch_conj_interleaved(double* X, i64 n, i64 ld, int nrhs, cudaStream_t st);
// Complex GMRES (interleaved vectors of nc complex entries per column; H and y complex pairs).
int cdots_chunks(i64 nc);
cudaError_t launch_cdots_strided(const double* V, i64 vstride, int kvec, const double* w, i64 nc, int nrhs,
                                 double* partial, int nchunks, double* out, i64 ostride, cudaStream_t st);
cudaError_t launch_cgs_update(double* w, const double* V, i64 vstride, const double* h, i64 hstride, int kvec, i64 nc,
                              int nrhs, double sign, const int* active, cudaStream_t st, const int* kdev = nullptr);
cudaError_t launch_cgmres_ls(const double* H, int ld, int inner, const double* beta, double* y, int nrhs,
                             cudaStream_t st, const int* used = nullptr);
cudaError_t launch_cgmres_estimate(const double* H, int ldh, int inner, int i, const double* beta, const double* normb,
                                   const int* act, int nrhs, double tol, int* ctl, cudaStream_t st);
cudaError_t launch_axpby(double* y, const double* x, double a, double b, i64 n, cudaStream_t st);
cudaError_t launch_residual_norm_finish(const double* nrm2, const double* normb, double* resid, int nrhs,
                                        cudaStream_t st);

i64 relerr_chunks(i64 n);
// partial: 2 * relerr_chunks(n) * nrhs doubles of scratch; out: nrhs doubles (device)
cudaError_t launch_relerr(const double* X, const double* ref, i64 n, i64 ld, int nrhs, double* partial, double* out,
                          cudaStream_t st);
cudaError_t launch_fma_probe(int precision, int blocks, int iters, void* out, cudaStream_t st);

}  // namespace h2b
