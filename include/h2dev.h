/*
 * h2dev.h — C ABI of the B200-native H^2 solver (libmxcb200.so).
 *
 * Plain pointers and sizes only.  Every entry point returns an int status
 * (H2DEV_OK on success).  "Host" arrays are caller-owned host memory; the
 * *_device variants take device pointers on the solver's device.  All
 * vectors are column-major n x nrhs with leading dimension ld >= n, in the
 * tree-sorted body order produced by h2_build_tree (the order the reference
 * uses for every vector, solver.hpp:23).  One solver object per host thread
 * at a time; calls on one handle are ordered on the handle's stream.
 */
#ifndef H2DEV_H
#define H2DEV_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct h2dev_handle_s* h2dev_handle_t;
typedef struct h2dev_solver_s* h2dev_solver_t;

enum {
  H2DEV_OK = 0,
  H2DEV_ERR_ARG = 1,      /* invalid argument or size */
  H2DEV_ERR_CUDA = 2,     /* CUDA runtime error (h2dev_last_error_message has it) */
  H2DEV_ERR_OOM = 3,      /* device allocation failed */
  H2DEV_ERR_STATE = 4,    /* call out of order (e.g. solve before factorize) */
  H2DEV_ERR_SINGULAR = 5, /* a redundant block had |det| <= DBL_MIN (info > 0) */
  H2DEV_ERR_NOCONV = 6    /* GMRES stopped at outer_iters above tol */
};

/* Laplace3D 1/d and Yukawa3D exp(-alpha d)/d (kernel.hpp:28-50); QUADRATIC
 * d^2 + alpha has exactly low-rank off-diagonal blocks (no counterpart in the
 * reference: used to verify that the ULV factorization is an exact inverse
 * when no fill is dropped).  Every kernel takes the value 1/s at d == 0.
 *
 * HELMHOLTZ is Helmholtz3D exp(-i alpha d)/d (kernel.hpp:63-74, the
 * reference's default, main.cpp:62), complex valued.  Its vectors are
 * complex: each column holds n complex values as 2n doubles with real and
 * imaginary parts interleaved (the std::complex<double> layout), so lenX,
 * ld and every vector length count 2 doubles per body.  The solver stores the
 * real symmetric form S = [[Re K, Im K], [Im K, -Re K]] over two real
 * unknowns per body (S conj(x) = K x) and runs every kernel of the real
 * path on it; matvec, precondition and the dense matvec conjugate their
 * vectors, and GMRES runs in complex arithmetic (as solver.cpp:144-201), so
 * that callers see K itself.  rank, leveled_rank and
 * samples are given per body as for the reference (complex degrees of
 * freedom) and doubled for the real form; level dims and ranks report real
 * unknowns.  Bodies' x coordinates are used with bit 0 cleared (a change of
 * at most one ulp), which carries the component tag internally. */
enum { H2DEV_KERNEL_LAPLACE = 0, H2DEV_KERNEL_YUKAWA = 1, H2DEV_KERNEL_QUADRATIC = 2, H2DEV_KERNEL_HELMHOLTZ = 3 };
enum { H2DEV_FP64 = 0, H2DEV_FP32 = 1 };

/* ---- host helpers (no device work) ---------------------------------- */

/* test_funcs.hpp:31-41 uniform_unit_cube_rnd: std::mt19937(seed) bodies. */
int h2_uniform_unit_cube_rnd(double* bodies, int64_t nbodies, double diameter, int64_t dim, unsigned seed);
/* main.cpp:73-76: default-seeded std::mt19937_64 uniform[0,1) vector. */
int h2_uniform_rhs(double* x, int64_t n);
/* build_tree.cpp:67-99 buildBinaryTree: sorts bodies (n x 3) in place and
 * fills 2^(levels+1)-1 cells: child[2], body[2] (int64) and R[3], C[3]. */
int h2_build_tree(double* bodies, int64_t nbodies, int64_t levels, int64_t* cell_child, int64_t* cell_body,
                  double* cell_R, double* cell_C);
/* No counterpart in the reference (whose median split always gives equal
 * leaves): the same tree with each cell cut where its bounding box is halved
 * along the longest extent, the cut clamped so every leaf ends with
 * leaf_min..leaf_max bodies (requires leaf_min 2^levels <= nbodies <=
 * leaf_max 2^levels).  For strongly non-uniform bodies (clustered
 * mixtures), where median cuts give elongated boxes. */
int h2_build_tree_capped(double* bodies, int64_t nbodies, int64_t levels, int64_t leaf_min, int64_t leaf_max,
                         int64_t* cell_child, int64_t* cell_body, double* cell_R, double* cell_C);
/* build_tree.cpp:41-58 CSR::CSR: kind 'N' (near) or 'F' (far) pair list over
 * all cells.  row receives ncells+1 offsets; col up to cap column indices;
 * *nnz the list length (call with col = NULL to size it). */
int h2_pair_csr(char kind, int64_t ncells, const int64_t* cell_child, const int64_t* cell_body, const double* cell_R,
                const double* cell_C, double theta, int64_t* row, int64_t* col, int64_t cap, int64_t* nnz);
/* main.cpp:54-55: levels = floor(log2(N / min(N, leaf))). */
int64_t h2_levels_for(int64_t nbodies, int64_t leaf);

/* ---- device handle (gpu_handles.cu:54-62 initGpuEnvs / finalizeGpuEnvs) */
int h2dev_handle_create(int device, h2dev_handle_t* out);
int h2dev_handle_destroy(h2dev_handle_t h);
int h2dev_handle_synchronize(h2dev_handle_t h);
/* Device memory of the handle: bytes held by its live solvers, plans and
 * temporaries, and bytes freed into its cache for reuse (no reference
 * counterpart; used for HBM-budget admission by a serving loop). */
int h2dev_handle_memory(h2dev_handle_t h, int64_t* live_bytes, int64_t* cached_bytes);
/* Returns the handle's cached (free) device blocks to the driver. */
int h2dev_handle_trim(h2dev_handle_t h);
/* High-water mark of the live bytes (blocks handed out by the handle's
 * cache) since the handle was created or the mark last reset; reset != 0
 * restarts it from the current live bytes.  No reference counterpart
 * (memory planning for resident systems). */
int h2dev_handle_memory_peak(h2dev_handle_t h, int64_t* peak_live_bytes, int reset);
/* Handle options (apply to solvers created afterwards on this handle).
 * H2DEV_OPT_BASIS: 0 (default) forms fixed-rank orthogonal bases from the
 * Gram matrix of the far samples with a pivoted Cholesky (same pivots and R
 * as the column-pivoted QR in exact arithmetic); 1 uses the Householder
 * sample-tile QR + Eigen-rule column-pivoted QR for every basis, the
 * reference's own sequence (h2matrix.cpp:19-32).  Threshold (operator) bases
 * always use the Householder path, or the sketch (H2DEV_OPT_SAMPLING = 2). */
/* H2DEV_OPT_SKINNY_TILED: 1 makes plans built afterwards (in this process)
 * run every multi-right-hand-side apply on the tiled segmented GEMM instead
 * of the register-streaming kernel; 0 (default) restores the latter. */
/* H2DEV_OPT_SAMPLING: how `samples` caps a box's far list.  0 (default):
 * rows floor(j * total / samples) of the whole list.  1: level-geometric —
 * the far boxes of the box's own level (the nearest) get half of the budget,
 * each level further out half of what remains, each group strided as in 0.
 * 2: sketch — `samples` is ignored and every far body is used, as the
 * reference does, but the column-pivoted QR runs on the M x M product of a
 * random-sign matrix with the whole far block instead of on R of its QR
 * (randomized interpolative decomposition; one FP64 tensor-core GEMM per box,
 * the far block is never stored).  Boxes whose far list has at most M bodies
 * use the far block itself, as the reference does. */
/* H2DEV_OPT_TENSOR_CORES: 1 (default) runs the FP32 block contractions of
 * plans built afterwards (in this process) on the tcgen05 tensor cores with
 * a 3-term TF32 split (FP32 accuracy); 2 with one TF32 product (about 1e-3
 * relative, for accuracy ablations); 0 runs them on the SIMT kernel. */
/* H2DEV_OPT_MATRIX_FREE: 1 makes operator-mode (epi > 0) FP64 solvers
 * created afterwards matrix-free: in interpolative mode every block the
 * matvec reads is the kernel evaluated on two point sets (leaf near blocks on
 * the box bodies, couplings on the skeleton bodies), so those blocks are
 * evaluated inside the matvec instead of stored, and the upper-level near
 * blocks (read only by a factorization) are not assembled.  Such a solver
 * holds only its bases and points; h2dev_factorize on it returns
 * H2DEV_ERR_STATE and exporting its A or C yields nothing.  0 (default)
 * stores every block as the reference does. */
/* H2DEV_OPT_PRECOND_BF16: 1 makes FP32 solvers created afterwards apply
 * their ULV substitution (solvePrecondition) from BF16 copies of the blocks
 * it streams, each scaled by a power of two so its entries lie in [-1, 1],
 * with FP32 arithmetic: half the bytes of the FP32 apply, 8 significand
 * bits instead of 24.  The factorization itself stays FP32.  0 (default):
 * FP32 blocks. */
/* H2DEV_OPT_GRAPH_SOLVE: 1 runs every GMRES solve on this handle as one
 * CUDA graph: the solve is captured once per call (a WHILE node over restart
 * cycles, an IF node around each Arnoldi step, the convergence decisions made
 * by kernels on the device) and launched once, with no host round trip until
 * it ends.  0 (default): the same kernels launched step by step, the host
 * reading the device's convergence flags between steps. */
/* H2DEV_OPT_AUTOTUNE: 1 (default) lets the handle time, once per plan shape
 * bucket, each launch variant a block-apply plan admits (row tilings of the
 * streaming applies, rows per thread of the matrix-free apply) on the plan's
 * own data and keep the fastest for later plans of the bucket; the variants
 * give identical results.  0: the fixed default variants. */
enum {
  H2DEV_OPT_BASIS = 0,
  H2DEV_OPT_SKINNY_TILED = 1,
  H2DEV_OPT_SAMPLING = 2,
  H2DEV_OPT_TENSOR_CORES = 3,
  H2DEV_OPT_MATRIX_FREE = 4,
  H2DEV_OPT_PRECOND_BF16 = 5,
  H2DEV_OPT_GRAPH_SOLVE = 6,
  H2DEV_OPT_AUTOTUNE = 7
};
int h2dev_set_option(h2dev_handle_t h, int option, int64_t value);

/* ---- solver (solver.hpp:11-47 H2MatrixSolver) ------------------------ */

/* H2MatrixSolver::H2MatrixSolver (solver.cpp:12-41): builds the tree lists,
 * the shared bases (compute_basis, h2matrix.cpp:13-63), near blocks and
 * couplings of every level on the device.  epi > 0: operator mode (ID basis
 * with relative threshold epi); epi == 0: fixed-rank orthogonal preconditioner
 * mode with rank (levels - l) * leveled_rank + rank at level l and far lists
 * from weak admissibility.  samples > 0 caps each box's far list (build
 * extension); samples <= 0 uses every far body as the reference does.
 * precision: H2DEV_FP64 or H2DEV_FP32 storage/arithmetic for this matrix.
 * bodies: tree-sorted nbodies x 3 host array (as left by h2_build_tree). */
int h2dev_solver_create(h2dev_handle_t h, int kernel, double singularity, double alpha, double epi, int64_t rank,
                        int64_t leveled_rank, int64_t ncells, const int64_t* cell_child, const int64_t* cell_body,
                        const double* cell_R, const double* cell_C, double theta, const double* bodies,
                        int64_t nbodies, int64_t levels, int64_t samples, int precision, h2dev_solver_t* out);
int h2dev_solver_destroy(h2dev_solver_t s);
/* levels and lenX (= local_bodies.second - local_bodies.first). */
int h2dev_solver_shape(h2dev_solver_t s, int64_t* levels, int64_t* lenX);
/* Dims / DimsLr of one level (h2matrix.hpp:27-28), 2^level entries each. */
int h2dev_solver_level_dims(h2dev_solver_t s, int64_t level, int64_t* dims, int64_t* ranks);

/* matVecMul (solver.cpp:76-88): X <- A_H2 X, in place. */
int h2dev_matvec(h2dev_solver_t s, int64_t nrhs, double* X, int64_t ldx);
int h2dev_matvec_device(h2dev_solver_t s, int64_t nrhs, double* dX, int64_t ldx);

/* factorizeM (solver.cpp:90-100): multilevel ULV factorization.
 * info_per_level (optional, levels+1 ints) receives the singular-block
 * count of each level; returns H2DEV_ERR_SINGULAR when any is nonzero. */
int h2dev_factorize(h2dev_solver_t s, int* info_per_level);

/* solvePrecondition (solver.cpp:121-132): X <- M^{-1} X, in place. */
int h2dev_solve_precondition(h2dev_solver_t s, int64_t nrhs, double* X, int64_t ldx);
int h2dev_solve_precondition_device(h2dev_solver_t s, int64_t nrhs, double* dX, int64_t ldx);

/* solveGMRES (solver.cpp:144-201), one independent restarted GMRES per
 * right-hand side: left preconditioner M (factored), true residual with A.
 * X is the initial guess on entry and the solution on return.  resid
 * ((outer+1) x nrhs, column-major) receives the relative residual history and
 * iters (nrhs) the restart cycles taken.  early_exit != 0 ends a cycle's
 * Arnoldi loop once every active Hessenberg residual estimate is below tol
 * (the reference always runs inner steps); 0 reproduces the reference. */
int h2dev_solve_gmres(h2dev_solver_t A, h2dev_solver_t M, double tol, int64_t nrhs, double* X, const double* B,
                      int64_t ld, int64_t inner, int64_t outer, int early_exit, double* resid, int64_t* iters);
int h2dev_solve_gmres_device(h2dev_solver_t A, h2dev_solver_t M, double tol, int64_t nrhs, double* dX,
                             const double* dB, int64_t ld, int64_t inner, int64_t outer, int early_exit,
                             double* resid, int64_t* iters);

/* H2MatrixSolver::solveRelErr (solver.cpp:229-238) for each of nrhs
 * columns of device arrays X and ref (leading dimension ld):
 * err[c] = sqrt(sum (x - ref)^2 / sum ref^2), written to host memory.  The
 * per-chunk partial sums live in a device scratch buffer allocated per call. */
int h2dev_solve_rel_err_device(h2dev_handle_t h, int64_t n, int64_t nrhs, const double* dX, const double* dRef,
                               int64_t ld, double* err);

/* No counterpart in the reference.  The same relative errors as
 * h2dev_solve_rel_err_device, for callers that must not allocate device
 * memory: a serving loop whose HBM is handed out entirely by its own budgeted
 * pool (an allocation behind its back can fail or break the budget), or a
 * latency-critical path that cannot take the device-wide synchronisation
 * cudaMalloc / cudaFree may imply.  Nothing is allocated: the partial sums go
 * to a fixed 16384-double (128 KiB) device array inside the library, held by
 * every GPU that loads it until the process exits, and err[c] is written to
 * the caller's device array dErr (nrhs doubles) asynchronously on the
 * handle's stream.  Limit: 2 * ceil(n / 16384) * nrhs <= 16384 (for example
 * n up to 134,217,728 with one column, 8,388,608 with 16); larger requests
 * return H2DEV_ERR_ARG.  The first call on a device looks up the array's
 * device address, so make it before any stream capture; the address is kept
 * for the life of the process, so do not call this after cudaDeviceReset.
 * All calls share the array: calls whose work overlaps on the GPU (two
 * streams at once) race. */
int h2dev_solve_rel_err_device_noalloc(h2dev_handle_t h, int64_t n, int64_t nrhs, const double* dX,
                                       const double* dRef, int64_t ld, double* dErr);

/* ---- dense kernel access (kernel.cpp:71-85 gen_matrix; main.cpp:83-84) */

/* out (m x n column-major) = K(bi, bj), bodies xyz-interleaved host arrays;
 * distances formed exactly as the reference's std::hypot.  HELMHOLTZ: the
 * complex block, 2m doubles per column (interleaved real/imaginary parts). */
int h2dev_gen_block(h2dev_handle_t h, int kernel, double singularity, double alpha, const double* bi, int64_t m,
                    const double* bj, int64_t n, double* out);
/* Y = A_dense X without storing A (host arrays, FP64).  HELMHOLTZ: X and Y
 * complex, 2n doubles per column (ld >= 2n). */
int h2dev_dense_matvec(h2dev_handle_t h, int kernel, double singularity, double alpha, const double* bodies,
                       int64_t n, int64_t nrhs, const double* X, double* Y, int64_t ld);
int h2dev_dense_matvec_device(h2dev_handle_t h, int kernel, double singularity, double alpha,
                              const double* dbodies, int64_t n, int64_t nrhs, const double* dX, double* dY,
                              int64_t ld);

/* ---- inspection (parity tests) -------------------------------------- */

enum { H2DEV_EXPORT_S = 0, H2DEV_EXPORT_Q = 1, H2DEV_EXPORT_R = 2, H2DEV_EXPORT_A = 3, H2DEV_EXPORT_C = 4 };
/* Number of doubles h2dev_solver_export writes for (level, what). */
int h2dev_solver_export_size(h2dev_solver_t s, int64_t level, int what, int64_t* count);
/* Copies one level's container (S: skeleton-ordered bodies, Q, R (V after
 * factorize, stored transposed), A near blocks, C couplings) in box /
 * block order, each block column-major, converted to double.  After
 * factorize, the redundant x redundant part of an off-diagonal near block
 * keeps its pre-transform values: the factorization never forms it (the
 * reference drops that fill and never reads it). */
int h2dev_solver_export(h2dev_solver_t s, int64_t level, int what, double* out);

/* ---- instrumentation (CUDA events on the handle's stream) ------------ */

/* Turns per-launch timing on/off (clears earlier records).  While on, every
 * kernel launch is bracketed by a pair of events; MPI_Wtime phase timers and
 * the comm stopwatch (main.cpp, comm-mpi.cpp:247-262) have no other analogue. */
int h2dev_profile_enable(h2dev_handle_t h, int on);
/* Aggregates the records by kernel name: up to cap rows of names (48 bytes
 * each), launch counts, total device ms, algorithmic FLOPs and bytes;
 * *count receives the number of distinct kernels. */
int h2dev_profile_report(h2dev_handle_t h, int64_t cap, char* names, int64_t* launches, double* ms, double* flops,
                         double* bytes, int64_t* count);
/* Strided-batched GEMM through the solver's segmented-GEMM engine (device
 * pointers, column-major, element type by `precision`): for b < batch,
 * C_b = beta C_b + alpha sum_{t < nterms} op(A_{b,t}) op(B_{b,t}), where
 * X_{b,t} = X + (b * nterms + t) * strideX, op(X) = X (op 0) or X^T (op 1),
 * op(A) m x k, op(B) k x n.  The contraction engine of the factorization,
 * exposed for testing and reuse; no reference counterpart. */
int h2dev_batched_gemm_device(h2dev_handle_t h, int precision, int64_t batch, int64_t nterms, int64_t m, int64_t n,
                              int64_t k, int opA, int opB, double alpha, const void* A, int64_t lda, int64_t strideA,
                              const void* B, int64_t ldb, int64_t strideB, double beta, void* C, int64_t ldc,
                              int64_t strideC);
/* Per-launch records since profiling was enabled, in launch order: names
 * (48 bytes each), start (ms after the first record's start) and device
 * duration; idle gaps between records show host-side stalls.  *count
 * receives the number of records. */
int h2dev_profile_timeline(h2dev_handle_t h, int64_t cap, char* names, double* start_ms, double* dur_ms,
                           int64_t* count);
/* Decisions of the handle's autotuner, in the order they were made: up to
 * cap bucket keys (64 bytes each), the chosen variant and the device ms of
 * each variant when it was timed (3 per key, -1 where a plan has fewer
 * variants); *count receives the number of decisions.  No reference
 * counterpart. */
int h2dev_autotune_report(h2dev_handle_t h, int64_t cap, char* keys, int* choice, double* ms, int64_t* count);
/* Number of kernels this library has launched in this process so far (all
 * handles); the difference across a region counts its launches. */
int h2dev_launch_count(int64_t* count);
/* Measured FMA throughput (TFLOP/s, 2 flops per FMA) of plain FP64 or FP32
 * SIMT code on this device: the denominator for the FP64/FP32 kernels. */
int h2dev_probe_fma_peak(h2dev_handle_t h, int precision, double* tflops);
/* Event pair on the handle's stream: device time between start and stop. */
int h2dev_timer_start(h2dev_handle_t h);
int h2dev_timer_stop(h2dev_handle_t h, double* ms);

const char* h2dev_last_error_message(void);

#ifdef __cplusplus
}
#endif

#endif /* H2DEV_H */
