/*
 * evd_b200.h — C ABI of the B200-native two-stage symmetric eigensolver.
 *
 * Every entry point is `extern "C"`, takes plain device pointers, 64-bit sizes
 * and leading dimensions (column-major FP64, as the reference), and a CUDA
 * stream (NULL = legacy default stream, which is what every reference routine
 * uses).  Each returns an int status (EVD_SUCCESS or a negative EVD_ERR_*).
 * No entry point allocates device memory unless its comment says so; the
 * caller passes workspaces sized by the matching *_work_size query.
 *
 * Synchronisation: entry points whose kernels report through a device error
 * word (bounded waits, convergence) read it before returning and therefore
 * synchronise `stream`: evd_bulge_chase(_noalloc), evd_stedc, evd_syevd,
 * evd_syevd_values, evd_tc_syr2k, evd_syr2k_lower_h, the metrics, the FP64
 * peak probe and the file functions.  All others only enqueue work on
 * `stream`.
 *
 * The comment on each function names the reference interface it replaces
 * (paths relative to the hansheng1001/EVD4SC2025 source tree).  The reference
 * functions take cuBLAS/cuSOLVER handles; this library uses none, so the C++
 * shims in evd_b200_compat.hpp accept and ignore them.
 */
#ifndef EVD_B200_H
#define EVD_B200_H

#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define EVD_SUCCESS 0
#define EVD_ERR_INVALID_ARG (-1)   /* bad size / leading dimension / pointer     */
#define EVD_ERR_CUDA (-2)          /* a CUDA runtime call failed                  */
#define EVD_ERR_TIMEOUT (-3)       /* a bounded device-side wait ran out          */
#define EVD_ERR_NO_CONVERGENCE (-4)/* an iterative solver did not converge        */
#define EVD_ERR_WORKSPACE (-5)     /* workspace smaller than the size query says  */
#define EVD_ERR_IO (-6)            /* a file could not be opened, read or written */
#define EVD_ERR_HOST (-7)          /* a host resource failed (threads, host memory) */

/* Human-readable text for a status code (static storage). */
const char* evd_status_string(int status);

/* Library version string, e.g. "evd_b200 0.1 sm_100a". */
const char* evd_version(void);

/* Number of kernel launches this library has issued since it was loaded (host
 * counter; a measurement aid with no counterpart in the reference). */
long evd_launch_count(void);

/* Measured FP64 DMMA throughput of the current GPU in TFLOP/s (a short
 * microbenchmark; the roofline denominator for the FP64 kernels; no
 * counterpart in the reference).  Synchronises `stream`. */
int evd_fp64_peak_probe(double* tflops, cudaStream_t stream);

/* ---- FP64 GEMM / SYR2K building blocks --------------------------------- */

/* C = alpha*op(A)*op(B) + beta*C, op = N ('n') or T ('t'); FP64 on DMMA.
 * Replaces the cublasGemmEx / cublasDgemm (CUBLAS_COMPUTE_64F) calls the
 * reference issues throughout (e.g. api/zy_zy_sy2sb.cu:134-347,
 * src/EVD/myEVD.cu:227-232, :564). */
int evd_dgemm(char transa, char transb, long m, long n, long k, double alpha,
              const double* A, long lda, const double* B, long ldb, double beta,
              double* C, long ldc, cudaStream_t stream);

/* Strided-batched variant (replaces cublasGemmStridedBatchedEx in
 * api/inc/TallShinnyQR.h:72-98 and src/EVD/myEVD.cu:151-206). */
int evd_dgemm_strided_batched(char transa, char transb, long m, long n, long k,
                              double alpha, const double* A, long lda, long strideA,
                              const double* B, long ldb, long strideB, double beta,
                              double* C, long ldc, long strideC, long batch,
                              cudaStream_t stream);

/* Lower-triangular SYR2K with mirrored upper triangle:
 *   C = alpha*(A*B^T + B*A^T) + beta*C   (n x n, A and B n x k)
 * then C(upper) = C(lower)^T.  Replaces tc_ozimmu_syr2k<double>
 * (api/inc/tc_ozimmu_syr2k.h:6-18, api/TCblas/tc_ozimmu_syr2k.cu:631-681)
 * followed by copyMatrixL2U (api/zy_zy_sy2sb.cu:436).  `nb` is accepted for
 * signature parity and ignored (the tile schedule does not need it). */
int evd_syr2k_lower_mirror(long n, long k, double alpha, const double* A, long lda,
                           const double* B, long ldb, double beta, double* C, long ldc,
                           long nb, cudaStream_t stream);

/* ---- Stage 1: full -> band (ZY) ---------------------------------------- */

/* Workspace (in doubles) needed by evd_tsqr / evd_panel_qr for an m x n panel. */
long evd_panel_qr_work_size(long m, long n);

/* Tall-skinny QR with explicit Q: A (m x n, n == 32) is overwritten by the
 * explicit thin Q, R (n x n) receives the triangular factor.  Tiles of 128
 * rows, reduction tree of fan-in 4, as hou_tsqr_panel<double,128,32>
 * (api/inc/TallShinnyQR.h:9-133, util/inc/kernelQR.h:215-414).
 * Requires (m % 128) % n == 0 like the reference (TallShinnyQR.h:37-41). */
int evd_tsqr(long m, long n, double* A, long lda, double* R, long ldr,
             double* work, long lwork, cudaStream_t stream);

/* Panel QR in compact form Q = I - W*Y^T: A (m x n) is overwritten by Y
 * (unit lower trapezoidal), W (m x n) and R (n x n) are written.  Replaces
 * panelQR<double> (api/inc/PanelQR.h:7-18, api/panelQR.cu:20-246): TSQR,
 * then the unpivoted LU of (I - Q) and W = (I - Q) * L1^{-T}. */
int evd_panel_qr(long m, long n, double* A, long lda, double* W, long ldw, double* R,
                 long ldr, double* work, long lwork, cudaStream_t stream);

/* Workspace (doubles) for evd_sy2sb. */
long evd_sy2sb_work_size(long M, long b, long nb);

/* Full-to-band reduction with the ZY update.  Argument meaning as
 * my_ZY_ZY_SBR_Vector<double> (api/inc/zy_zy_sy2sb.h:5-24,
 * api/zy_zy_sy2sb.cu:24-486): dOriA holds the full symmetric matrix and is
 * destroyed; dA receives the band matrix (lower band, R blocks); the W and Y
 * factors of each b-wide panel are left at (i, i-b) of dW / dY; dZ (M x nb)
 * and dR (M x nb) are scratch.  On return dA is symmetric (both triangles),
 * as after the reference's copyMatrixL2U (src/EVD/myEVD.cu:346).
 * Requires b == 32, M == N, M % nb == 0, nb % b == 0. */
int evd_sy2sb(long M, long N, long b, long nb, double* dOriA, long ldOriA, double* dA,
              long ldA, double* dW, long ldW, double* dY, long ldY, double* dZ, long ldZ,
              double* dR, long ldR, double* work, long lwork, cudaStream_t stream);

/* ---- Stage 2: band -> tridiagonal (bulge chasing) ----------------------- */

/* Pack the lower band of dA into band storage sub(i + j*ldSub) = A(j+i, j),
 * i < 2b, zero below the band (kernel_bugle_chasing_cpydA2dSubA,
 * src/EVD/myEVD.cu:53-78). */
int evd_band_pack(long n, long b, const double* dA, long ldA, double* dSub, long ldSub,
                  cudaStream_t stream);

/* Bytes of int scratch needed by evd_bulge_chase (progress flags + counters). */
long evd_bulge_chase_iwork_size(long n);

/* Band -> tridiagonal.  dSub is band storage with ldSub == 2b exactly (each
 * column contiguous) and 16-byte alignment; it is overwritten;
 * every Householder vector (||u||^2 = 2) is written into dU column s (sweep s),
 * 32-row segments starting at row s+1, exactly where chasing_kernel_one_timeV10
 * writes them (util/inc/bugle_chasingV10.h:21-392, launched at
 * src/EVD/myEVD.cu:383-439).  dU must have ldU >= n and is NOT cleared here
 * (clear it first, as the reference does at src/EVD/myEVD.cu:413).  d (n) and
 * e (n-1) receive the tridiagonal (kernel_bugle_chasing_cpydSubA2dA +
 * cpyATr2Vector, src/EVD/myEVD.cu:105-123, :477-480).  iwork: evd_bulge_chase_iwork_size
 * bytes of device memory.  b must be 32.  dU may be NULL: the reflectors are
 * then not stored (eigenvalues-only use). */
int evd_bulge_chase(long n, long b, double* dSub, long ldSub, double* dU, long ldU,
                    double* d, double* e, int* iwork, cudaStream_t stream);

/* Same as evd_bulge_chase, but allocates nothing and takes no scratch: for
 * callers that cannot obtain device memory where they run the chase (no
 * cudaMalloc allowed there: a fixed memory footprint, or a host framework that
 * owns the allocator).  This entry point has no counterpart in the reference.
 * Its scratch is a file-scope device array of the library, sized for
 * n <= 65536 (256 KB per GPU that loads the library, kept until exit); larger
 * n is rejected with EVD_ERR_INVALID_ARG and a message on stderr.  The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress);
 * make that first call before any stream capture.  Every call shares the one
 * array and clears it first, so calls that overlap on the GPU (other streams,
 * other host threads) race: serialise them.  Synchronises `stream`. */
int evd_bulge_chase_noalloc(long n, long b, double* dSub, long ldSub, double* dU, long ldU,
                            double* d, double* e, cudaStream_t stream);

/* ---- Tridiagonal eigensolver (device divide and conquer) ---------------- */

long evd_stedc_work_size(long n);   /* doubles */
long evd_stedc_iwork_size(long n);  /* ints    */

/* All eigenvalues (ascending, into d) and eigenvectors (Z, n x n) of the
 * symmetric tridiagonal (d, e).  Replaces the host LAPACKE_dstedc('I') call of
 * the reference driver (src/EVD/myEVD.cu:529) with a device divide and
 * conquer.  d and e are device arrays; e is destroyed. */
int evd_stedc(long n, double* d, double* e, double* Z, long ldz, double* work, long lwork,
              int* iwork, long liwork, cudaStream_t stream);

/* All eigenvalues (ascending, into w) of the symmetric tridiagonal (d, e), no
 * vectors: Sturm-count multisection with the pivot rule of LAPACK dstebz.  The
 * eigenvalues-only counterpart of the reference's LAPACKE_dstedc('I') call
 * (src/EVD/myEVD.cu:529), which always forms vectors.  work: evd_stebz_work_size
 * doubles.  d and e are not modified. */
long evd_stebz_work_size(long n);
int evd_stebz(long n, const double* d, const double* e, double* w, double* work, long lwork,
              cudaStream_t stream);

/* ---- Back transformations ----------------------------------------------- */

/* Q <- Q2^T * Q, Q2 = product of the chasing reflectors stored in U (generation
 * order).  Same signature and meaning as my_BC_back_trans_v8_10_noBandU
 * (api/inc/BC_backTrans.h:3, api/BC_backTransV8_10_noBandU.cu:234-313).  Q has
 * n rows (rows >= n are neither read nor written, so no padding is needed);
 * U is the chasing output (ldU >= n).  Returns 0 on success. */
int evd_bc_back(double* Q, long ldQ, const double* U, long ldU, long n, int b,
                cudaStream_t stream);

/* X <- Q2 * X for an n x ncols block X (the eigenvector direction: reflectors
 * applied in reverse generation order; the reference applies Q2 through
 * my_SBRBack_BCBack, src/EVD/myEVD.cu:135-249).  `work` (16-byte aligned,
 * evd_bc_back_work_size(n) doubles, about 5 n^2/8) receives the compact-WY
 * factors V = Y T of the reflector groups, built once for all columns; with
 * work == NULL the T factors are rebuilt inside the apply kernel (slower). */
long evd_bc_back_work_size(long n);
int evd_bc_back_apply(long n, long ncols, const double* U, long ldU, double* X, long ldX,
                      int b, double* work, long lwork, cudaStream_t stream);

/* Merge the b-wide compact-WY slides of an M x N block into one compact WY:
 * W[:, i-b:i] -= W[:, 0:i-b] * (Y[:, 0:i-b]^T * W[:, i-b:i]) for i = 2b..N.
 * Same as computerWYFromSlide (api/inc/computerWYFromSlide.h:4,
 * api/computerWYFromSlide.cu:5-25); work >= M*b doubles (the reference's
 * (i-b) x b product with leading dimension M). */
int evd_wy_from_slide(long M, long N, long slideWidth, double* dW, long ldW,
                      const double* dY, long ldY, double* work, cudaStream_t stream);

/* Q = I - W*Y^T (M x M), as computerQFromWY (api/inc/computerQFromWY.h:4,
 * api/computerQFromWY.cu:5-17). */
int evd_q_from_wy(long M, long N, double* dQ, long ldQ, const double* dW, long ldW,
                  const double* dY, long ldY, cudaStream_t stream);

/* Workspace (doubles) for evd_sbr_back. */
long evd_sbr_back_work_size(long n, long b, long nk);

/* X <- Q1 * X with Q1 = prod_p (I - W_p Y_p^T) over the b-wide panels left by
 * evd_sy2sb in dW/dY (panel p at rows/cols (p+1)b.., p*b..).  Panels are merged
 * into nk-wide slabs first (the inline merge of my_SBRBack_BCBack,
 * src/EVD/myEVD.cu:148-207; dW is overwritten by the merged W), then each slab
 * is applied to X.  The reference instead forms Q1 from I
 * (src/EVD/myEVD.cu:213-233) and multiplies by Z afterwards (:564). */
int evd_sbr_back(long n, long b, long nk, double* dW, long ldW, const double* dY,
                 long ldY, double* X, long ldX, long ncols, double* work, long lwork,
                 cudaStream_t stream);

/* ---- Metrics (a13) --------------------------------------------------------- */

/* result[0] = ||A^T B - I||_F / M  (checkOrthogonality,
 * util/tool/checkMetric.cu:5-24, which prints instead of returning).
 * A and B are N x M.  work >= M*M doubles (as the reference); result is a
 * HOST pointer (the call synchronises `stream`). */
int evd_check_orthogonality(long M, long N, const double* dA, long ldA, const double* dB,
                            long ldB, double* work, double* result, cudaStream_t stream);

/* result[0] = ||A X - X diag(w)||_F / (n ||A||_F), result[1] = ||X^T X - I||_F / n.
 * work >= n*n doubles; result is a HOST pointer (synchronises `stream`). */
int evd_check_eig(long n, const double* A, long lda, const double* w, const double* X,
                  long ldX, double* work, double* result, cudaStream_t stream);

/* ---- Whole solver ------------------------------------------------------- */

/* Bytes of device workspace for evd_syevd and evd_syevd_values (0 for an
 * unsupported shape: b != 32, nb not 32 * 2^k, n < 1).  Any n >= 1 is accepted;
 * when n % nb != 0 the workspace also holds the padded copies (see evd_syevd). */
long evd_syevd_work_size(long n, long b, long nb);

/* Stage timings (milliseconds, CUDA events) of the last evd_syevd call on this
 * host thread: [0] sy2sb, [1] bulge chasing, [2] tridiagonal D&C,
 * [3] stage-2 back transformation, [4] stage-1 back transformation, [5] total. */
void evd_syevd_last_timings(double out_ms[6]);

/* Eigenvalues w (ascending, device, n) and eigenvectors X (n x n, device) of the
 * symmetric A (device, full storage; A is not modified).  The plain-FP64
 * two-stage pipeline of the reference driver `myEVD n b nb`
 * (src/EVD/myEVD.cu:251-706): sy2sb -> bulge chasing -> tridiagonal D&C ->
 * stage-2 then stage-1 back transformation.  work: evd_syevd_work_size bytes.
 * The reference requires n % nb == 0; here any n >= 1 is accepted: A is embedded
 * in A' = [A 0; 0 D] of order n' = nb * ceil(n / nb), D = diag(2s + s k / (n' - n)),
 * s = ||A||_1 computed on the device (no host synchronisation), so A's
 * eigenvalues are the n smallest of A' and the leading n x n block of A''s
 * eigenvectors holds A's.  Stage timings then refer to the order-n' solve. */
int evd_syevd(long n, long b, long nb, const double* A, long lda, double* w, double* X,
              long ldX, void* work, long lwork_bytes, int timed, cudaStream_t stream);

/* Eigenvalues only (ascending, device, n) of the symmetric A: sy2sb, the chase
 * without storing reflectors, and evd_stebz; no back transformation.  The
 * reference driver has no such mode (its eigenvalues come from the full
 * dstedc at src/EVD/myEVD.cu:465-491).  work: evd_syevd_work_size bytes;
 * evd_syevd_last_timings gives [0] sy2sb, [1] chasing, [2] tridiagonal
 * eigenvalues, [5] total.  Any n >= 1, padded as in evd_syevd. */
int evd_syevd_values(long n, long b, long nb, const double* A, long lda, double* w, void* work,
                     long lwork_bytes, int timed, cudaStream_t stream);

/* ---- Batched solves of uneven orders ------------------------------------ */

/* No counterpart in the reference (one matrix per process, myEVD.cu:251-706).
 * Eigenpairs of `count` symmetric matrices of any orders n[i] >= 1: A[i]
 * (n[i] x n[i], lda[i]), w[i] (n[i]), X[i] (n[i] x n[i], ldX[i]), all device
 * pointers; the pointer and size arrays are HOST arrays.  The solves run on
 * min(nstreams, count) internal streams (one host thread each, largest
 * matrices first), after the work already enqueued on `stream`, which waits
 * for all of them; nb per matrix: the largest 32 * 2^k (<= 1024) dividing
 * 32 * ceil(n / 32).  work: evd_syevd_batched_work_size bytes (one solver
 * workspace of the largest order per stream).  nstreams <= 64.  Returns the
 * first failing solve's status.  Synchronises the internal streams. */
long evd_syevd_batched_work_size(long count, const long* n, int nstreams);
int evd_syevd_batched(long count, const long* n, const double* const* A, const long* lda,
                      double* const* w, double* const* X, const long* ldX, int nstreams,
                      void* work, long lwork_bytes, cudaStream_t stream);

/* ---- Mixed form of the solve -------------------------------------------- */

/* Same pipeline and outputs as evd_syevd (the reference's myEVD,
 * src/EVD/myEVD.cu:251-706), with the big contractions on the integer tensor
 * cores.  These are emulated products with `moduli` moduli
 * (evd_dgemm_ozaki; 14 give FP64-level operands, fewer are faster and less
 * accurate):
 *  - the stage-1 trailing SYR2K (the reference's tc_ozimmu_syr2k,
 *    api/TCblas/tc_ozimmu_syr2k.cu:631-681);
 *  - Q1, formed explicitly (myEVD.cu:135-249 forms it from I);
 *  - the large divide-and-conquer merges;
 *  - Q2^T = B A, Q^T = Q2^T Q1^T (the reference's Q, myEVD.cu:563-565) and
 *    X = Q Z.
 * Then `refine_iters` Ogita-Aishima iterations with FP64-level emulated
 * products win FP64 accuracy back (the X E update uses `moduli_update`,
 * <= 14).
 * The chase runs as consecutive sweep ranges.  The DMMA stage-2 kernel
 * accumulates A (the reflectors of the sweeps below 0.39 n) and B (the rest)
 * from the identity on side streams, one range behind the chase.  The Q1
 * formation and the divide and conquer run beside them.  Up to n = 24576
 * the work size includes an n x n buffer and integer workspaces of their own
 * for the divide and conquer and the Q1 formation.  The panels, the chase,
 * the divide and conquer and the stage-2 reflectors are the plain FP64
 * kernels.
 * refine_iters > 0 needs n <= 65535 (padded order).  work:
 * evd_syevd_mixed_work_size bytes.  Synchronises `stream`. */
long evd_syevd_mixed_work_size(long n, long b, long nb, int moduli, int refine_iters);
/* The smallest workspace evd_syevd_mixed accepts (no counterpart in the
 * reference): with less than evd_syevd_mixed_work_size bytes it runs one
 * stage-2 chain and the divide and conquer after the Q1 formation, the
 * schedule of orders above 24576 (slower, about 2.4 n^2 + n^2 doubles less). */
long evd_syevd_mixed_work_size_min(long n, long b, long nb, int moduli, int refine_iters);
int evd_syevd_mixed(long n, long b, long nb, const double* A, long lda, double* w, double* X,
                    long ldX, int moduli, int refine_iters, int moduli_update, void* work,
                    long lwork_bytes, int timed, cudaStream_t stream);
/* refinement time (ms) of the last timed evd_syevd_mixed call on this thread
 * (evd_syevd_last_timings holds its other stages and, at index 5, the total) */
double evd_syevd_last_refine_ms(void);
/* stages (ms) of the last timed evd_syevd_mixed call on this thread: sy2sb,
 * chase, divide and conquer (from the end of the chase), Q1 formation, the
 * stage-2 chains (from their start to the end of the later one), the final
 * products (from the end of the divide and conquer to X), refinement, total.
 * The Q1 formation and the stage-2 chains run on side streams beside the
 * chase and the divide and conquer. */
void evd_syevd_mixed_last_timings(double out_ms[8]);

/* ---- FP32 solve ---------------------------------------------------------- */

/* The reference's driver is FP64 only (myEVD.cu:251-706); its FP32 pieces are
 * panelQR<float> (api/panelQR.cu:262-464) and tc_ozimmu_syr2k<float>
 * (api/TCblas/tc_ozimmu_syr2k.cu:343-629).  All eigenpairs of the symmetric
 * FP32 matrix A (n x n, lda; any n >= 1): w (n, ascending) and X (n x n, ldX),
 * FP32, device pointers.  The solve is evd_syevd_mixed with 8 moduli (30-bit
 * operands) and no refinement: the dominant contractions run on the integer
 * tensor cores at the accuracy FP32 needs, while the latency-bound stages
 * (panels, chase, divide and conquer) stay FP64.  Residual and orthogonality
 * (1/n normalised) are FP32-level or better.  work: evd_syevd_s_work_size
 * bytes (FP64 copies of A, w and X plus the mixed form's workspace).
 * Synchronises `stream`. */
long evd_syevd_s_work_size(long n, long b, long nb);
int evd_syevd_s(long n, long b, long nb, const float* A, long lda, float* w, float* X, long ldX,
                void* work, long lwork_bytes, cudaStream_t stream);

/* ---- Iterative refinement of eigenpairs -------------------------------- */

/* No counterpart in the reference.  Ogita-Aishima refinement (RefSyEv,
 * JJIAM 35 (2018), Algorithm 1) of approximate eigenpairs of the symmetric A:
 * each iteration forms R = I - X^T X and S = X^T A X with FP64 DMMA GEMMs,
 * l_i = s_ii / (1 - r_ii), the correction E (clustered pairs, |l_i - l_j| <=
 * delta, get r_ij / 2) and X <- X + X E; w receives the l_i of the last
 * iteration (in the column order of X).  The error of X falls quadratically
 * while it is well below the eigenvalue gaps; 8 n^3 flops per iteration.
 * n <= 65535; work: evd_refine_syev_work_size(n) doubles (3 n^2 + O(n)). */
long evd_refine_syev_work_size(long n);
int evd_refine_syev(long n, const double* A, long lda, double* w, double* X, long ldX, int iters,
                    double* work, long lwork, cudaStream_t stream);

/* The same iteration with every product emulated on the integer tensor cores
 * (evd_dgemm_ozaki's scheme): A X, X^T X and X^T A X with `moduli` moduli (14:
 * FP64-level operands), X E with `moduli_update` (<= moduli; E is of the size
 * of X's error, so fewer bits of it give the same absolute accuracy).  The
 * symmetric products multiply only their lower tiles.  n <= 65535; work:
 * evd_refine_syev_ozaki_work_size(n, moduli) BYTES.  Synchronises `stream`. */
long evd_refine_syev_ozaki_work_size(long n, int moduli);
int evd_refine_syev_ozaki(long n, const double* A, long lda, double* w, double* X, long ldX,
                          int iters, int moduli, int moduli_update, void* work,
                          long lwork_bytes, cudaStream_t stream);

/* ---- Emulated FP64 products on the integer tensor cores ---------------- */

/* Replaces the FP64 cuBLAS products of the reference's trailing update
 * (api/TCblas/tc_ozimmu_syr2k.cu:54-192, cublasDgemm) with an Ozaki-II
 * emulation: C = alpha op(A) op(B) + beta C, where every row of op(A) and
 * column of op(B) is scaled to integers of at most P bits (2-norm), the
 * product is formed exactly modulo `moduli` pairwise coprime numbers <= 256 by
 * tcgen05 kind::i8 GEMMs with INT32 accumulation, and rebuilt by the Chinese
 * remainder theorem.  Error <= ~sqrt(k) 2^-P ||row_i(op A)|| ||col_j(op B)||;
 * P = evd_ozaki_bits(moduli, k) (53 for 14 moduli).  4 <= moduli <= 20,
 * k <= 65536; C must not alias A or B.  work: evd_dgemm_ozaki_work_size
 * bytes (moduli x (m + n + m n) k-ish bytes).  Synchronises `stream` (reads
 * the error word of the bounded tensor-core waits). */
long evd_dgemm_ozaki_work_size(char transa, char transb, long m, long n, long k, int moduli);
int evd_dgemm_ozaki(char transa, char transb, long m, long n, long k, double alpha,
                    const double* A, long lda, const double* B, long ldb, double beta, double* C,
                    long ldc, int moduli, void* work, long lwork_bytes, cudaStream_t stream);
int evd_ozaki_bits(int moduli, long k);

/* ---- FP32 / FP16 entry points of the reference's API -------------------- */

/* The reference instantiates panelQR and tc_ozimmu_syr2k for float and half
 * (api/panelQR.cu:262-701, api/TCblas/tc_ozimmu_syr2k.cu:343-629, :683-720)
 * and has tc_syr2k (api/inc/tc_syr2k.h:6-18, api/TCblas/tc_syr2k.cu:144-330).
 * FP16 matrices are passed as void* holding IEEE binary16 values. */

/* Bytes of workspace for evd_panel_qr_s/_h and evd_tsqr_s/_h (m x 32 panel). */
long evd_panel_qr_lp_work_size(long m, long n);
/* panelQR<float> / panelQR<half> (api/inc/PanelQR.h:7-18), n == 32: A <- Y,
 * W, R as evd_panel_qr.  Computed in FP64 on converted copies, rounded back. */
int evd_panel_qr_s(long m, long n, float* A, long lda, float* W, long ldw, float* R, long ldr,
                   void* work, long lwork_bytes, cudaStream_t stream);
int evd_panel_qr_h(long m, long n, void* A, long lda, void* W, long ldw, void* R, long ldr,
                   void* work, long lwork_bytes, cudaStream_t stream);
/* hou_tsqr_panel<float/half, 128, 32>: A <- explicit thin Q, R. */
int evd_tsqr_s(long m, long n, float* A, long lda, float* R, long ldr, void* work,
               long lwork_bytes, cudaStream_t stream);
int evd_tsqr_h(long m, long n, void* A, long lda, void* R, long ldr, void* work,
               long lwork_bytes, cudaStream_t stream);
/* tc_ozimmu_syr2k<float>: C(lower) = alpha (A B^T + B A^T) + beta C in FP32
 * arithmetic (SIMT FP32 FMA; CUBLAS_COMPUTE_32F in the reference).  Only the
 * lower triangle (with the diagonal) is written; beta == 0 does not read C. */
int evd_syr2k_lower_s(long n, long k, float alpha, const float* A, long lda, const float* B,
                      long ldb, float beta, float* C, long ldc, long nb, cudaStream_t stream);
/* tc_syr2k: as above with A and B rounded to FP16 and the products summed in
 * FP32 on the tcgen05 tensor cores.  `hwork` (2 n k halves, as the reference)
 * receives the packed FP16 operands when k % 8 == 0; with hwork == NULL or
 * another k the library uses a buffer from its own stream-ordered memory pool.  nb is
 * accepted and not needed. */
int evd_tc_syr2k(long n, long k, float alpha, const float* A, long lda, const float* B, long ldb,
                 float beta, float* C, long ldc, void* hwork, long nb, cudaStream_t stream);
/* tc_ozimmu_syr2k<half>: FP16 A, B, C; FP32 accumulation on the tensor cores
 * (the reference accumulates in FP16, CUBLAS_COMPUTE_16F); alpha, beta as float.
 * Packs the operands into a buffer of 2 n k halves from the library's pool. */
int evd_syr2k_lower_h(long n, long k, float alpha, const void* A, long lda, const void* B,
                      long ldb, float beta, void* C, long ldc, long nb, cudaStream_t stream);

/* ---- Matrix and eigenpair files ----------------------------------------- */

/* The reference has CSV only (writeMatrixToCsvV2, util/inc/fileOpTool.h:51-80;
 * readMatrixFromFile + fillMatrix, util/tool/fileOpTool.cu:127-174).  Binary
 * files here are a sequence of records: a 32-byte little-endian header
 * {"EVDM", u32 version = 1, u32 elem_bytes = 8, u32 0, i64 rows, i64 cols}
 * then rows * cols FP64 values, column-major.  Matrix pointers may be device
 * or host memory.  Errors: EVD_ERR_IO (open/read/write failure, bad header,
 * missing record), EVD_ERR_INVALID_ARG (bad size, or a shape that does not
 * match the record). */
int evd_write_matrix_bin(const char* path, int append, long rows, long cols, const double* A,
                         long ldA);
/* Number of records in the file (negative status on error). */
long evd_matrix_bin_count(const char* path);
int evd_matrix_bin_shape(const char* path, long index, long* rows, long* cols);
int evd_read_matrix_bin(const char* path, long index, long rows, long cols, double* A, long ldA);
/* Eigenpair file: record 0 = w (n x 1), record 1 = X (n x n). */
int evd_write_eigenpairs_bin(const char* path, long n, const double* w, const double* X,
                             long ldX);
int evd_read_eigenpairs_bin(const char* path, long n, double* w, double* X, long ldX);
/* CSV in the reference's layout (one matrix row per line, comma separated,
 * %.17g).  evd_read_matrix_csv with A == NULL returns the shape in *rows,
 * *cols; with A it checks the shape and reads. */
int evd_write_matrix_csv(const char* path, long rows, long cols, const double* A, long ldA);
int evd_read_matrix_csv(const char* path, long* rows, long* cols, double* A, long ldA);

#ifdef __cplusplus
}
#endif

#endif /* EVD_B200_H */
