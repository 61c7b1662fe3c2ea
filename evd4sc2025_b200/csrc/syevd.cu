// Whole two-stage eigensolver (plain FP64): the pipeline of the reference
// driver `myEVD n b nb` (src/EVD/myEVD.cu:251-706) behind one C entry point.
//
//   A -> [sy2sb] band B, W, Y -> [band pack + bulge chasing] T = (d, e), U
//     -> [device D&C] T = Z diag(w) Z^T
//     -> X = Q2 Z [stage-2 back transformation, reflectors from U]
//     -> X = Q1 X [stage-1 back transformation, slab-merged WY from W, Y]
//
// Differences from the reference driver: the tridiagonal solve runs on the GPU
// (the reference copies T to the host for MKL dstedc and overlaps it with the
// back transformation on a second host thread); Q1 and Q2 are applied to the
// eigenvectors directly instead of forming Q = Q2^T Q1^T explicitly and
// multiplying by Z in a final GEMM (saves 4n^3 flops); one process can call it
// any number of times (the reference's chasing kernel keeps a global flag that
// makes a second call return early).
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "common.cuh"
#include "gemm_f64.cuh"
#include "ozaki.cuh"

namespace evd {

long sy2sb_ws_doubles(long M, long b, long nb);
int sy2sb(long M, long N, long b, long nb, double* OA, long ldOA, double* dA, long ldA,
          double* dW, long ldW, double* dY, long ldY, double* dZ, long ldZ, double* dR, long ldR,
          double* work, long lwork, cudaStream_t st, const OzWork* oz);
int copy_matrix(long m, long n, const double* src, long lds, double* dst, long ldd,
                cudaStream_t st);
int band_pack(long n, long b, const double* dA, long ldA, double* dSub, long ldSub,
              cudaStream_t st);
long chase_iwork_ints(long n);
int bulge_chase_async(long n, long b, double* dSub, long ldSub, double* dU, long ldU, double* d,
                      double* e, int* iwork, cudaStream_t st);
long stedc_ws_doubles(long n);
int stebz(long n, const double* d, const double* e, double* w, double* work, cudaStream_t st);
long stedc_ws_ints(long n);
int stedc(long n, double* d, double* e, double* Z, long ldz, double* work, long lwork, int* iwork,
          long liwork, cudaStream_t st, const OzWork* oz);
long q2_tbuf_doubles(long n);
int q2_apply(bool forward, long n, long ncols, const double* U, long ldU, double* X, long ldX,
             double* tbuf, cudaStream_t st);
long sbr_back_ws_doubles(long n, long b, long nk);
int wy_merge_slabs(long n, long b, long nk, long ncolsWY, double* dW, long ldW, const double* dY,
                   long ldY, double* work, cudaStream_t st);
int sbr_apply_slabs(long n, long b, long nk, const double* dW, long ldW, const double* dY,
                    long ldY, double* X, long ldX, long ncols, double* work, size_t work_n,
                    cudaStream_t st);
long sbr_form_oz_bytes(long n, long nk, int nmod);
int sbr_form_q1(long n, long b, long nk, const double* dW, long ldW, const double* dY, long ldY,
                double* M, long ldM, double* work, size_t work_n, cudaStream_t st,
                const OzWork* oz, bool lean);
int oz_transpose(long m, long n, const double* A, long lda, double* B, long ldb, cudaStream_t st);
long refine_ws_doubles(long n);
long refine_oz_int_bytes(long n, int moduli);
int refine_syev_oz_split(long n, const double* A, long lda, double* w, double* X, long ldX,
                         int iters, int moduli, int moduli_update, double* f64, uint8_t* iwork,
                         cudaStream_t st);

// The mixed form of the solve: the big contractions (the trailing SYR2K of
// stage 1 and both products of every stage-1 back-transformation slab) as
// emulated products on the integer tensor cores with `nmod` moduli, then
// `refine_iters` Ogita-Aishima iterations with FP64-level emulated products
// (moduli kOzFp64Mod, the X E update with `moduli_update`).
struct MixedOpts {
  int nmod;
  int refine_iters;
  int moduli_update;
  uint8_t* oz;
  long oz_bytes;
};

// integer workspace of the mixed solve for order n (padded)
long mixed_oz_bytes(long n, long nb, int nmod, int refine_iters) {
  long need = std::max(oz_syr2k_ws_bytes(std::max(n - nb, 1L), nb, nmod),
                       sbr_form_oz_bytes(n, nb, nmod));
  // X = Q Z, and the divide and conquer's largest merge products (their
  // left operand is transposed first)
  need = std::max(need, oz_layout(n, n, n, nmod, true).bytes);
  if (refine_iters > 0) need = std::max(need, refine_oz_int_bytes(n, kOzFp64Mod));
  return need + 512;
}

namespace {

struct SyevdLayout {
  long nb_eff;
  size_t oOA, oA, oW, oY, oZ, oR, oS, oSub, oU, oD, oE, oStedc, oSbr, end_d;  // doubles
  size_t oIchase, oIstedc, end_i;                                          // ints
  size_t bytes;
};

SyevdLayout layout(long n, long b, long nb) {
  SyevdLayout L{};
  auto al = [](size_t x) { return (x + 31) / 32 * 32; };
  size_t o = 0;
  const size_t nn = (size_t)n * n;
  L.oOA = o; o = al(o + nn);
  L.oA = o; o = al(o + nn);
  L.oW = o; o = al(o + nn);
  L.oY = o; o = al(o + nn);
  L.oZ = o; o = al(o + (size_t)n * nb);
  L.oR = o; o = al(o + (size_t)n * nb);
  L.oS = o; o = al(o + sy2sb_ws_doubles(n, b, nb));
  L.oSub = o; o = al(o + (size_t)2 * b * n);
  L.oU = o; o = al(o + nn);
  L.oD = o; o = al(o + n);
  L.oE = o; o = al(o + n);
  L.oStedc = o; o = al(o + stedc_ws_doubles(n));
  L.oSbr = o; o = al(o + sbr_back_ws_doubles(n, b, nb));
  L.end_d = o;
  size_t q = 0;
  L.oIchase = q; q = al(q + chase_iwork_ints(n));
  L.oIstedc = q; q = al(q + stedc_ws_ints(n));
  L.end_i = q;
  L.bytes = L.end_d * sizeof(double) + L.end_i * sizeof(int) + 256;
  return L;
}

thread_local double g_timings[6] = {0, 0, 0, 0, 0, 0};
thread_local double g_refine_ms = 0.0;  // refinement time of the last timed mixed solve
// stages of the last timed mixed solve: sy2sb, chase, divide and conquer, Q1
// formation, stage-2 application, X = Q Z, refinement, total (the Q1 and
// stage-2 times overlap the chase and the divide and conquer)
thread_local double g_mixed[8] = {0, 0, 0, 0, 0, 0, 0, 0};

// A second stream for the work that overlaps the main stream inside one
// call, and the events that order the two; destroyed (after the side stream
// has drained, also on error paths) when the call returns.
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t ev[12] = {};
  int nev = 0;
  bool timing = false;
  ~SideStream() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
    for (int i = 0; i < nev; ++i) cudaEventDestroy(ev[i]);
  }
  int init(bool timed) {
    timing = timed;
    EVD_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    for (nev = 0; nev < 12; ++nev)
      EVD_CUDA_TRY(cudaEventCreateWithFlags(&ev[nev], timed ? cudaEventDefault
                                                            : cudaEventDisableTiming));
    return EVD_SUCCESS;
  }
};

// NVTX range per stage (a profiler's timeline shows the stages by name; the
// range closes on every return path)
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace

// err_out != nullptr: the chase's error word is not read here; its address is
// returned so the caller can enqueue more work before the one host read.
static int syevd_core(long n, long b, long nb, const double* A, long lda, double* w, double* X,
                      long ldX, void* work, long lwork_bytes, int timed, cudaStream_t st,
                      const int** err_out = nullptr) {
  if (n <= 0 || b != 32 || nb <= 0 || nb % b != 0 || n % nb != 0) return EVD_ERR_INVALID_ARG;
  long q = nb / b;
  if (q & (q - 1)) return EVD_ERR_INVALID_ARG;  // slab merge needs nb = b * 2^k
  if (lda < n || ldX < n || !A || !w || !X || !work) return EVD_ERR_INVALID_ARG;
  SyevdLayout L = layout(n, b, nb);
  if ((size_t)lwork_bytes < L.bytes) return EVD_ERR_WORKSPACE;
  double* base = reinterpret_cast<double*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
  int* ibase = reinterpret_cast<int*>(base + L.end_d);
  double *OA = base + L.oOA, *dA = base + L.oA, *W = base + L.oW, *Y = base + L.oY,
         *Z = base + L.oZ, *R = base + L.oR, *S = base + L.oS, *sub = base + L.oSub,
         *U = base + L.oU, *d = base + L.oD, *e = base + L.oE, *SW = base + L.oStedc,
         *SB = base + L.oSbr;
  int* ich = ibase + L.oIchase;
  int* ist = ibase + L.oIstedc;

  cudaEvent_t ev[6];
  if (timed) {
    for (auto& x : ev) EVD_CUDA_TRY(cudaEventCreate(&x));
    EVD_CUDA_TRY(cudaEventRecord(ev[0], st));
  }
  {  // ---- stage 1: full -> band ----
    NvtxRange r("evd_b200 sy2sb");
    EVD_TRY(copy_matrix(n, n, A, lda, OA, n, st));
    EVD_TRY(copy_matrix(n, n, A, lda, dA, n, st));
    EVD_CUDA_TRY(cudaMemsetAsync(W, 0, sizeof(double) * n * n, st));
    EVD_CUDA_TRY(cudaMemsetAsync(Y, 0, sizeof(double) * n * n, st));
    EVD_TRY(sy2sb(n, n, b, nb, OA, n, dA, n, W, n, Y, n, Z, n, R, n, S,
                  (long)sy2sb_ws_doubles(n, b, nb), st, nullptr));
  }
  if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[1], st));
  {  // ---- stage 2: band -> tridiagonal ----
    NvtxRange r("evd_b200 bulge chasing");
    EVD_TRY(band_pack(n, b, dA, n, sub, 2 * b, st));
    EVD_CUDA_TRY(cudaMemsetAsync(U, 0, sizeof(double) * n * n, st));
    EVD_TRY(bulge_chase_async(n, b, sub, 2 * b, U, n, d, e, ich, st));
  }
  if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[2], st));
  {  // ---- tridiagonal D&C (eigenvectors straight into X) ----
    NvtxRange r("evd_b200 tridiagonal divide and conquer");
    EVD_TRY(
        stedc(n, d, e, X, ldX, SW, (long)stedc_ws_doubles(n), ist, (long)stedc_ws_ints(n), st,
              nullptr));
  }
  if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[3], st));
  {  // ---- back transformations ----
    NvtxRange r("evd_b200 stage-2 back transformation");
    // the T factors of the chasing reflectors go into OA (free after stage 1);
    // for very small n they do not fit and the kernel rebuilds them itself
    double* tbuf = ((size_t)q2_tbuf_doubles(n) <= (size_t)n * n) ? OA : nullptr;
    EVD_TRY(q2_apply(false, n, n, U, n, X, ldX, tbuf, st));
  }
  if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[4], st));
  {
    NvtxRange r("evd_b200 stage-1 back transformation");
    const long npcols = ((n - 1) / b) * b;
    EVD_TRY(wy_merge_slabs(n, b, nb, npcols, W, n, Y, n, SB, st));
    EVD_TRY(sbr_apply_slabs(n, b, nb, W, n, Y, n, X, ldX, n, SB,
                            (size_t)sbr_back_ws_doubles(n, b, nb), st));
  }
  EVD_CUDA_TRY(cudaMemcpyAsync(w, d, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  if (timed) {
    EVD_CUDA_TRY(cudaEventRecord(ev[5], st));
    EVD_CUDA_TRY(cudaEventSynchronize(ev[5]));
    float ms;
    for (int i = 0; i < 5; ++i) {
      EVD_CUDA_TRY(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
      g_timings[i] = ms;
    }
    EVD_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[5]));
    g_timings[5] = ms;
    for (auto& x : ev) cudaEventDestroy(x);
  }
  // chasing error word (bounded waits) is checked once at the end
  if (err_out) {
    *err_out = ich + n + 32;
    return EVD_SUCCESS;
  }
  return read_device_error(ich + n + 32, st);
}

size_t syevd_ws_bytes(long n, long b, long nb) { return layout(n, b, nb).bytes; }

// The mixed form, scheduled on two streams (the reference overlaps its host
// divide and conquer with the back transformation in the same spirit,
// src/EVD/myEVD.cu:503-561):
//   main:  sy2sb (emulated trailing SYR2K) -> band pack -> chase -> D&C (Z
//          into W) -> X = Q Z (one emulated product) -> refinement
//   side:  after the band pack: slab merge, Q1 formed explicitly (emulated
//          products, the lean integer GEMM beside the chase), Q1^T;
//          after the chase: Q^T = Q2^T Q1^T (the DMMA stage-2 kernel, beside
//          the D&C)
// Buffers: Q1 in dA (free after the band pack), Q1^T and then Q^T in Y (free
// after the formation), the stage-2 T factors in OA, Z in W (the main stream
// waits for the formation before the D&C writes it).
static int syevd_mixed_core(long n, long b, long nb, const double* A, long lda, double* w,
                            double* X, long ldX, void* work, long lwork_bytes, int timed,
                            cudaStream_t st, const int** err_out, const MixedOpts* mx) {
  if (n <= 0 || b != 32 || nb <= 0 || nb % b != 0 || n % nb != 0) return EVD_ERR_INVALID_ARG;
  long q = nb / b;
  if (q & (q - 1)) return EVD_ERR_INVALID_ARG;
  if (lda < n || ldX < n || !A || !w || !X || !work || !mx) return EVD_ERR_INVALID_ARG;
  SyevdLayout L = layout(n, b, nb);
  if ((size_t)lwork_bytes < L.bytes) return EVD_ERR_WORKSPACE;
  double* base = reinterpret_cast<double*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
  int* ibase = reinterpret_cast<int*>(base + L.end_d);
  double *OA = base + L.oOA, *dA = base + L.oA, *W = base + L.oW, *Y = base + L.oY,
         *Z = base + L.oZ, *R = base + L.oR, *S = base + L.oS, *sub = base + L.oSub,
         *U = base + L.oU, *d = base + L.oD, *e = base + L.oE, *SW = base + L.oStedc,
         *SB = base + L.oSbr;
  int* ich = ibase + L.oIchase;
  int* ist = ibase + L.oIstedc;
  const OzWork oz{mx->nmod, mx->oz, mx->oz_bytes};
  SideStream side;
  EVD_TRY(side.init(timed != 0));
  cudaStream_t sb = side.s;
  // events: 0 start, 1 sy2sb done, 2 band packed, 3 Q1^T ready, 4 chase done,
  // 5 Q^T ready, 6 D&C done, 7 X done, 8 refined, 9 side start of stage 2
  cudaEvent_t* ev = side.ev;
  if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[0], st));
  {
    NvtxRange r("evd_b200 sy2sb (emulated trailing update)");
    EVD_TRY(copy_matrix(n, n, A, lda, OA, n, st));
    EVD_TRY(copy_matrix(n, n, A, lda, dA, n, st));
    EVD_CUDA_TRY(cudaMemsetAsync(W, 0, sizeof(double) * n * n, st));
    EVD_CUDA_TRY(cudaMemsetAsync(Y, 0, sizeof(double) * n * n, st));
    EVD_TRY(sy2sb(n, n, b, nb, OA, n, dA, n, W, n, Y, n, Z, n, R, n, S,
                  (long)sy2sb_ws_doubles(n, b, nb), st, &oz));
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[1], st));
  EVD_TRY(band_pack(n, b, dA, n, sub, 2 * b, st));
  EVD_CUDA_TRY(cudaEventRecord(ev[2], st));
  // ---- side: Q1 formation beside the chase ----
  EVD_CUDA_TRY(cudaStreamWaitEvent(sb, ev[2], 0));
  {
    NvtxRange r("evd_b200 Q1 formation (side stream)");
    const long npcols = ((n - 1) / b) * b;
    EVD_TRY(wy_merge_slabs(n, b, nb, npcols, W, n, Y, n, SB, sb));
    EVD_TRY(sbr_form_q1(n, b, nb, W, n, Y, n, dA, n, SB, (size_t)sbr_back_ws_doubles(n, b, nb),
                        sb, &oz, true));
    EVD_TRY(oz_transpose(n, n, dA, n, Y, n, sb));  // Q1^T
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[3], sb));
  {
    NvtxRange r("evd_b200 bulge chasing");
    EVD_CUDA_TRY(cudaMemsetAsync(U, 0, sizeof(double) * n * n, st));
    EVD_TRY(bulge_chase_async(n, b, sub, 2 * b, U, n, d, e, ich, st));
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[4], st));
  // ---- side: Q^T = Q2^T Q1^T beside the D&C ----
  EVD_CUDA_TRY(cudaStreamWaitEvent(sb, ev[4], 0));
  if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[9], sb));
  {
    NvtxRange r("evd_b200 stage-2 application to Q1^T (side stream)");
    double* tbuf = ((size_t)q2_tbuf_doubles(n) <= (size_t)n * n) ? OA : nullptr;
    EVD_TRY(q2_apply(true, n, n, U, n, Y, n, tbuf, sb));
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[5], sb));
  // ---- main: D&C (Z into W once the formation no longer reads W) ----
  EVD_CUDA_TRY(cudaStreamWaitEvent(st, ev[3], 0));
  {
    NvtxRange r("evd_b200 tridiagonal divide and conquer");
    EVD_TRY(stedc(n, d, e, W, n, SW, (long)stedc_ws_doubles(n), ist, (long)stedc_ws_ints(n), st,
                  &oz));
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[6], st));
  EVD_CUDA_TRY(cudaStreamWaitEvent(st, ev[5], 0));
  {
    NvtxRange r("evd_b200 X = Q Z (emulated)");
    EVD_TRY(oz_gemm('t', 'n', n, n, n, 1.0, Y, n, W, n, 0.0, nullptr, n, 0.0, X, ldX, mx->nmod,
                    false, mx->oz, mx->oz_bytes, st));
  }
  EVD_CUDA_TRY(cudaMemcpyAsync(w, d, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  EVD_CUDA_TRY(cudaEventRecord(ev[7], st));
  if (mx->refine_iters > 0) {
    NvtxRange r("evd_b200 eigenpair refinement");
    if ((size_t)refine_ws_doubles(n) > L.oY + (size_t)n * n) return EVD_ERR_WORKSPACE;
    EVD_TRY(refine_syev_oz_split(n, A, lda, w, X, ldX, mx->refine_iters, kOzFp64Mod,
                                 mx->moduli_update, OA, mx->oz, st));
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[8], st));
  if (timed) {
    EVD_CUDA_TRY(cudaEventSynchronize(ev[8]));
    float ms;
    auto el = [&](int a, int z) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[a], ev[z]);
      return (double)t;
    };
    g_mixed[0] = el(0, 1);
    g_mixed[1] = el(1, 4);
    g_mixed[2] = el(4, 6);
    g_mixed[3] = el(2, 3);
    g_mixed[4] = el(9, 5);
    g_mixed[5] = el(6, 7);
    g_mixed[6] = el(7, 8);
    g_mixed[7] = el(0, 8);
    g_refine_ms = g_mixed[6];
    g_timings[0] = g_mixed[0];
    g_timings[1] = g_mixed[1];
    g_timings[2] = g_mixed[2];
    g_timings[3] = g_mixed[4];
    g_timings[4] = g_mixed[3];
    g_timings[5] = g_mixed[7];
    (void)ms;
  }
  if (err_out) {
    *err_out = ich + n + 32;
    return EVD_SUCCESS;
  }
  return read_device_error(ich + n + 32, st);
}

// Eigenvalues only: stage 1, the chase without storing reflectors, and
// Sturm-count multisection on the tridiagonal (no vectors, no back
// transformation).  Same workspace as syevd.
static int values_core(long n, long b, long nb, const double* A, long lda, double* w,
                       void* work, long lwork_bytes, int timed, cudaStream_t st,
                       const int** err_out = nullptr) {
  if (n <= 0 || b != 32 || nb <= 0 || nb % b != 0 || n % nb != 0) return EVD_ERR_INVALID_ARG;
  if (lda < n || !A || !w || !work) return EVD_ERR_INVALID_ARG;
  SyevdLayout L = layout(n, b, nb);
  if ((size_t)lwork_bytes < L.bytes) return EVD_ERR_WORKSPACE;
  double* base = reinterpret_cast<double*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
  int* ibase = reinterpret_cast<int*>(base + L.end_d);
  double *OA = base + L.oOA, *dA = base + L.oA, *W = base + L.oW, *Y = base + L.oY,
         *Z = base + L.oZ, *R = base + L.oR, *S = base + L.oS, *sub = base + L.oSub,
         *d = base + L.oD, *e = base + L.oE, *SW = base + L.oStedc;
  int* ich = ibase + L.oIchase;
  cudaEvent_t ev[4];
  if (timed) {
    for (auto& x : ev) EVD_CUDA_TRY(cudaEventCreate(&x));
    EVD_CUDA_TRY(cudaEventRecord(ev[0], st));
  }
  EVD_TRY(copy_matrix(n, n, A, lda, OA, n, st));
  EVD_TRY(copy_matrix(n, n, A, lda, dA, n, st));
  EVD_CUDA_TRY(cudaMemsetAsync(W, 0, sizeof(double) * n * n, st));
  EVD_CUDA_TRY(cudaMemsetAsync(Y, 0, sizeof(double) * n * n, st));
  EVD_TRY(sy2sb(n, n, b, nb, OA, n, dA, n, W, n, Y, n, Z, n, R, n, S,
                (long)sy2sb_ws_doubles(n, b, nb), st, nullptr));
  if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[1], st));
  EVD_TRY(band_pack(n, b, dA, n, sub, 2 * b, st));
  EVD_TRY(bulge_chase_async(n, b, sub, 2 * b, nullptr, n, d, e, ich, st));
  if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[2], st));
  EVD_TRY(stebz(n, d, e, w, SW, st));
  if (timed) {
    EVD_CUDA_TRY(cudaEventRecord(ev[3], st));
    EVD_CUDA_TRY(cudaEventSynchronize(ev[3]));
    float ms;
    for (int i = 0; i < 3; ++i) {
      EVD_CUDA_TRY(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
      g_timings[i] = ms;
    }
    g_timings[3] = g_timings[4] = 0.0;
    EVD_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[3]));
    g_timings[5] = ms;
    for (auto& x : ev) cudaEventDestroy(x);
  }
  if (err_out) {
    *err_out = ich + n + 32;
    return EVD_SUCCESS;
  }
  return read_device_error(ich + n + 32, st);
}

}  // namespace evd

namespace evd {
namespace {

// ---- any order n: padding to a multiple of nb ----
// A of order n is embedded in A' = [A 0; 0 D] of order n' = nb * ceil(n / nb),
// D = diag(2s + s k / (n'-n)), s >= ||A||_1 >= ||A||_2 (computed on the device).
// A' is block diagonal, so its n smallest eigenvalues are A's, and the
// leading n x n block of its eigenvectors holds A's eigenvectors.

__global__ void col_abs_sum_kernel(long n, const double* __restrict__ A, long lda,
                                   double* __restrict__ cs) {
  __shared__ double red[32];
  const long j = blockIdx.x;
  double acc = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) acc += fabs(A[i + j * lda]);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
    cs[j] = t;
  }
}

__global__ void pad_fill_kernel(long n, long np, const double* __restrict__ cs,
                                double* __restrict__ Ap, long ldp) {
  // s = max column sum (every block recomputes it: n <= a few 10^5 reads)
  __shared__ double red[32];
  double m = 0.0;
  for (long j = threadIdx.x; j < n; j += blockDim.x) m = fmax(m, cs[j]);
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  double sv = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) sv = fmax(sv, red[k]);
  if (!(sv > 0.0)) sv = 1.0;  // zero matrix: pad values 2 .. 3 sit above its eigenvalues
  const long kpad = np - n;
  // column c of A' outside A's block: zero, with the pad value on the diagonal;
  // rows n.. of A's columns: zero
  for (long c = blockIdx.x; c < np; c += gridDim.x) {
    if (c < n) {
      for (long i = n + threadIdx.x; i < np; i += blockDim.x) Ap[i + c * ldp] = 0.0;
    } else {
      const double dv = 2.0 * sv + sv * (double)(c - n) / (double)kpad;
      for (long i = threadIdx.x; i < np; i += blockDim.x) Ap[i + c * ldp] = (i == c) ? dv : 0.0;
    }
  }
}

// at least 64 (two b = 32 panels), so the smallest problems take the same path
long padded_order(long n, long nb) { return std::max<long>((n + nb - 1) / nb * nb, 64); }
bool needs_pad(long n, long nb) { return n % nb != 0 || n < 64; }

struct PadLayout {
  long np;
  size_t core_bytes, oAp, oXp, owp, ocs, bytes;  // offsets in doubles after the core part
};

PadLayout pad_layout(long n, long b, long nb) {
  PadLayout P{};
  P.np = padded_order(n, nb);
  P.core_bytes = syevd_ws_bytes(P.np, b, nb);
  const size_t base = (P.core_bytes + 255) / 8 + 32;  // doubles, past the core region
  auto al = [](size_t x) { return (x + 31) / 32 * 32; };
  size_t o = al(base);
  P.oAp = o; o = al(o + (size_t)P.np * P.np);
  P.oXp = o; o = al(o + (size_t)P.np * P.np);
  P.owp = o; o = al(o + P.np);
  P.ocs = o; o = al(o + n);
  P.bytes = o * sizeof(double) + 256;
  return P;
}

int pad_prepare(long n, const double* A, long lda, const PadLayout& P, double* base,
                cudaStream_t st) {
  double* Ap = base + P.oAp;
  double* cs = base + P.ocs;
  col_abs_sum_kernel<<<(unsigned)n, 256, 0, st>>>(n, A, lda, cs);
  EVD_LAUNCHED();
  EVD_TRY(copy_matrix(n, n, A, lda, Ap, P.np, st));
  pad_fill_kernel<<<(unsigned)std::min<long>(P.np, 4096), 256, 0, st>>>(n, P.np, cs, Ap, P.np);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

bool shape_ok(long n, long b, long nb) {
  return n > 0 && b == 32 && nb > 0 && nb % b == 0 && ((nb / b) & (nb / b - 1)) == 0;
}

}  // namespace

size_t syevd_any_ws_bytes(long n, long b, long nb) {
  if (!needs_pad(n, nb)) return syevd_ws_bytes(n, b, nb);
  return pad_layout(n, b, nb).bytes;
}

int syevd(long n, long b, long nb, const double* A, long lda, double* w, double* X, long ldX,
          void* work, long lwork_bytes, int timed, cudaStream_t st) {
  if (!shape_ok(n, b, nb)) return EVD_ERR_INVALID_ARG;
  if (!needs_pad(n, nb)) return syevd_core(n, b, nb, A, lda, w, X, ldX, work, lwork_bytes, timed, st);
  if (lda < n || ldX < n || !A || !w || !X || !work) return EVD_ERR_INVALID_ARG;
  const PadLayout P = pad_layout(n, b, nb);
  if ((size_t)lwork_bytes < P.bytes) return EVD_ERR_WORKSPACE;
  double* base = reinterpret_cast<double*>(work);
  EVD_TRY(pad_prepare(n, A, lda, P, base, st));
  const int* err = nullptr;
  EVD_TRY(syevd_core(P.np, b, nb, base + P.oAp, P.np, base + P.owp, base + P.oXp, P.np, work,
                     (long)P.core_bytes, timed, st, &err));
  EVD_CUDA_TRY(cudaMemcpyAsync(w, base + P.owp, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  EVD_TRY(copy_matrix(n, n, base + P.oXp, P.np, X, ldX, st));
  return read_device_error(err, st);
}

// Mixed form: workspace = the plain solve's (any order) + the integer part.
size_t syevd_mixed_ws_bytes(long n, long b, long nb, int nmod, int refine_iters) {
  const size_t plain = (syevd_any_ws_bytes(n, b, nb) + 255) / 256 * 256;
  return plain + (size_t)mixed_oz_bytes(padded_order(n, nb), nb, nmod, refine_iters) + 256;
}

int syevd_mixed(long n, long b, long nb, const double* A, long lda, double* w, double* X,
                long ldX, int nmod, int refine_iters, int moduli_update, void* work,
                long lwork_bytes, int timed, cudaStream_t st) {
  if (!shape_ok(n, b, nb)) return EVD_ERR_INVALID_ARG;
  if (nmod < kOzMinMod || nmod > kOzMaxMod || refine_iters < 0 || refine_iters > 16 ||
      moduli_update < kOzMinMod || moduli_update > kOzFp64Mod)
    return EVD_ERR_INVALID_ARG;
  const long np = padded_order(n, nb);
  if (refine_iters > 0 && np > 65535) return EVD_ERR_INVALID_ARG;
  if (lda < n || ldX < n || !A || !w || !X || !work) return EVD_ERR_INVALID_ARG;
  if ((size_t)lwork_bytes < syevd_mixed_ws_bytes(n, b, nb, nmod, refine_iters))
    return EVD_ERR_WORKSPACE;
  const size_t plain = (syevd_any_ws_bytes(n, b, nb) + 255) / 256 * 256;
  uint8_t* wb = reinterpret_cast<uint8_t*>(work);
  uint8_t* ozb = reinterpret_cast<uint8_t*>(((uintptr_t)(wb + plain) + 255) & ~(uintptr_t)255);
  MixedOpts mx{nmod, refine_iters, moduli_update, ozb,
               mixed_oz_bytes(np, nb, nmod, refine_iters)};
  const int* err = nullptr;
  if (!needs_pad(n, nb)) {
    EVD_TRY(syevd_mixed_core(n, b, nb, A, lda, w, X, ldX, work, (long)plain, timed, st, &err, &mx));
  } else {
    const PadLayout P = pad_layout(n, b, nb);
    double* base = reinterpret_cast<double*>(work);
    EVD_TRY(pad_prepare(n, A, lda, P, base, st));
    EVD_TRY(syevd_mixed_core(P.np, b, nb, base + P.oAp, P.np, base + P.owp, base + P.oXp, P.np,
                             work, (long)P.core_bytes, timed, st, &err, &mx));
    EVD_CUDA_TRY(
        cudaMemcpyAsync(w, base + P.owp, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    EVD_TRY(copy_matrix(n, n, base + P.oXp, P.np, X, ldX, st));
  }
  EVD_TRY(read_device_error(err, st));
  return oz_check_err(st);
}

int syevd_values(long n, long b, long nb, const double* A, long lda, double* w, void* work,
                 long lwork_bytes, int timed, cudaStream_t st) {
  if (!shape_ok(n, b, nb)) return EVD_ERR_INVALID_ARG;
  if (!needs_pad(n, nb)) return values_core(n, b, nb, A, lda, w, work, lwork_bytes, timed, st);
  if (lda < n || !A || !w || !work) return EVD_ERR_INVALID_ARG;
  const PadLayout P = pad_layout(n, b, nb);
  if ((size_t)lwork_bytes < P.bytes) return EVD_ERR_WORKSPACE;
  double* base = reinterpret_cast<double*>(work);
  EVD_TRY(pad_prepare(n, A, lda, P, base, st));
  const int* err = nullptr;
  EVD_TRY(values_core(P.np, b, nb, base + P.oAp, P.np, base + P.owp, work, (long)P.core_bytes,
                      timed, st, &err));
  EVD_CUDA_TRY(cudaMemcpyAsync(w, base + P.owp, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  return read_device_error(err, st);
}

}  // namespace evd

extern "C" long evd_syevd_work_size(long n, long b, long nb) {
  if (!evd::shape_ok(n, b, nb)) return 0;
  return (long)evd::syevd_any_ws_bytes(n, b, nb);
}

extern "C" void evd_syevd_last_timings(double out_ms[6]) {
  for (int i = 0; i < 6; ++i) out_ms[i] = evd::g_timings[i];
}

extern "C" int evd_syevd_values(long n, long b, long nb, const double* A, long lda, double* w,
                                void* work, long lwork_bytes, int timed, cudaStream_t stream) {
  return evd::syevd_values(n, b, nb, A, lda, w, work, lwork_bytes, timed, stream);
}

extern "C" int evd_syevd(long n, long b, long nb, const double* A, long lda, double* w, double* X,
                         long ldX, void* work, long lwork_bytes, int timed, cudaStream_t stream) {
  return evd::syevd(n, b, nb, A, lda, w, X, ldX, work, lwork_bytes, timed, stream);
}

extern "C" long evd_syevd_mixed_work_size(long n, long b, long nb, int moduli, int refine_iters) {
  if (!evd::shape_ok(n, b, nb) || moduli < evd::kOzMinMod || moduli > evd::kOzMaxMod ||
      refine_iters < 0)
    return 0;
  return (long)evd::syevd_mixed_ws_bytes(n, b, nb, moduli, refine_iters);
}

extern "C" int evd_syevd_mixed(long n, long b, long nb, const double* A, long lda, double* w,
                               double* X, long ldX, int moduli, int refine_iters,
                               int moduli_update, void* work, long lwork_bytes, int timed,
                               cudaStream_t stream) {
  try {
    return evd::syevd_mixed(n, b, nb, A, lda, w, X, ldX, moduli, refine_iters, moduli_update,
                            work, lwork_bytes, timed, stream);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

extern "C" double evd_syevd_last_refine_ms(void) { return evd::g_refine_ms; }

extern "C" void evd_syevd_mixed_last_timings(double out_ms[8]) {
  for (int i = 0; i < 8; ++i) out_ms[i] = evd::g_mixed[i];
}
