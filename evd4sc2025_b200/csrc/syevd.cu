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
#include <cstdlib>
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
          long liwork, cudaStream_t st, const OzWork* oz, cudaEvent_t out_after = nullptr);
long stedc_oz_bytes(long n, int nmod);
long q2_tbuf_doubles(long n);
int q2_apply(bool forward, long n, long ncols, const double* U, long ldU, double* X, long ldX,
             double* tbuf, cudaStream_t st);
int q2_apply_range(bool forward, long n, long ncols, const double* U, long ldU, double* X,
                   long ldX, double* tbuf, long h0, long h1, long ident_k, cudaStream_t st);
int chase_part_async(long n, long b, double* dSub, long ldSub, double* dU, long ldU, int* iwork,
                     long s0, long s1, int part, cudaStream_t st);
int chase_tridiag(long n, const double* dSub, long ldSub, double* d, double* e, cudaStream_t st);
int set_identity(long m, long n, double* Q, long ldq, cudaStream_t st);
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
  uint8_t* oz_dc;  // the divide and conquer's own integer workspace, or nullptr
  long oz_dc_bytes;
  uint8_t* oz_q1;  // the Q1 formation's own integer workspace, or nullptr
  long oz_q1_bytes;
  double* split_buf;  // an n x n buffer for the second stage-2 chain, or nullptr
};

// Orders up to this one get a separate integer workspace for the divide and
// conquer's emulated merges (about 2.4 n^2 doubles), so that it can run while
// the Q1 formation still uses the main one; above it (32768: 21 GB more on top
// of about 140 GB) the divide and conquer waits for the formation instead.
constexpr long kMixedDcOwnMax = 24576;
// The separate regions of orders up to kMixedDcOwnMax (bytes, each 256-byte
// aligned): the D&C's integer workspace, the Q1 formation's, and the n x n
// buffer of the second stage-2 chain; zero sizes above it.
struct MixedExtra {
  long dc, q1, split, total;
};
MixedExtra mixed_extra(long np, long nb, int nmod) {
  MixedExtra x{};
  if (np > kMixedDcOwnMax) return x;
  auto al = [](long v) { return (v + 255) / 256 * 256; };
  x.dc = al(stedc_oz_bytes(np, nmod) + 512);
  x.q1 = al(sbr_form_oz_bytes(np, nb, nmod) + 512);
  x.split = al(np * np * 8);
  x.total = x.dc + x.q1 + x.split + 256;
  return x;
}

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
  cudaEvent_t ev[40] = {};
  int nev = 0;
  bool timing = false;
  ~SideStream() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
    for (int i = 0; i < nev; ++i) cudaEventDestroy(ev[i]);
  }
  int init(bool timed, int prio = 0) {
    timing = timed;
    EVD_CUDA_TRY(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, prio));
    for (nev = 0; nev < 40; ++nev)
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

// Sweep ranges of the pipelined chase.  Below the split sweep k (a multiple
// of 8): [0, 512), [512, 1536), ... doubling, the last one ending at k; from k
// on: ranges of max(2048, (n - 2 - k) / 16) sweeps (rounded up to a multiple
// of 8), the last one ending at sweep n - 2.  k = 0: no lower part.  Returns
// the number of ranges r (at most 32); range i is [bounds[i], bounds[i+1]).
static int chase_ranges(long n, long k, long bounds[34]) {
  const long S = std::max(n - 2, 0L);
  int c = 0;
  bounds[c++] = 0;
  long s = 0, len = 512;
  while (s + len < k) {
    s += len;
    bounds[c++] = s;
    len *= 2;
  }
  if (k > 0 && k < S) bounds[c++] = k;
  s = std::max(k, 0L);
  const long step = std::max(2048L, ((S - s) / 16 + 7) / 8 * 8);
  while (s + step < S) {
    s += step;
    bounds[c++] = s;
  }
  bounds[c] = S;
  return c;
}

// The mixed form with the stage-2 reflectors applied while the chase runs.
// Q2^T = B A with A = the reflectors of the sweeps [0, k) and B those of the
// sweeps [k, n - 2), each accumulated from the identity by the DMMA stage-2
// kernel one chase range behind the chase (a CTA skips the strips that are
// still zero below its columns).  The kernel's dependency chain (strips x
// blocks of 8 sweeps per column) is the longest path of the solve; splitting
// it at k = 0.39 n into two chains that run side by side about halves it
// (A starts after the first range, B once the chase has passed k).
//   main:   sy2sb (emulated trailing SYR2K) -> band pack -> chase, one launch
//           per sweep range -> D&C (own integer workspace; Z into W once the
//           Q1 formation no longer reads W)
//   side B: slab merge, Q1 formed explicitly (emulated)
//   side A: A = I, the ranges below k; T1 = A Q1^T; Q^T = B T1;
//           X = Q Z (emulated, the main integer workspace)
//   side C: B = I, the ranges from k
// Without the extra n x n buffer (orders above kMixedDcOwnMax) there is one
// chain, P = Q2^T in X, then Y2 = P^T Z and X = Q1 Y2.
// Buffers: A in the extra buffer (then Q^T), B (or P) in X, Q1 in dA, T1 (or
// Y2) in Y, Z in W, the stage-2 T factors in OA.
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
  const OzWork ozdc{mx->nmod, mx->oz_dc, mx->oz_dc_bytes};
  const OzWork ozq1{mx->nmod, mx->oz_q1, mx->oz_q1_bytes};
  const bool dc_own = mx->oz_dc != nullptr;
  // the chains' T factors go into OA (free after stage 1); for very small n
  // they do not fit and the stage-2 kernel rebuilds them itself
  double* tbuf = ((size_t)q2_tbuf_doubles(n) <= (size_t)n * n) ? OA : nullptr;
  double* XA = mx->split_buf;  // chain A, then Q^T
  const bool split = XA != nullptr && n > 64;
  const long k = split ? std::max(8L, (long)(0.39 * (double)n) / 8 * 8) : 0;
  SideStream sideA, sideB, sideC;
  EVD_TRY(sideA.init(timed != 0));
  EVD_TRY(sideB.init(timed != 0));
  EVD_TRY(sideC.init(timed != 0));
  cudaStream_t sa = sideA.s, sb = sideB.s, sc = sideC.s;
  // events: 0 start, 1 sy2sb done, 2 band packed, 3 Q1 ready, 4 chase done,
  // 5 chain A (or P) done, 6 D&C done, 7 X done, 8 refined, 9 side A start,
  // 10 chain B done, 11 products done, 12 first product done;
  // sideB.ev[i]: chase range i done
  cudaEvent_t* ev = sideA.ev;
  cudaEvent_t* evr = sideB.ev;
  long bounds[34];
  const int nr = chase_ranges(n, k, bounds);
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
  // ---- side B: Q1 formation ----
  EVD_CUDA_TRY(cudaStreamWaitEvent(sb, ev[2], 0));
  {
    NvtxRange r("evd_b200 Q1 formation (side stream)");
    const long npcols = ((n - 1) / b) * b;
    EVD_TRY(wy_merge_slabs(n, b, nb, npcols, W, n, Y, n, SB, sb));
    // the 4-stage integer GEMM beside the two chains (measured faster there);
    // the 2-stage one beside the single chain, whose CTAs it shares SMs with
    EVD_TRY(sbr_form_q1(n, b, nb, W, n, Y, n, dA, n, SB, (size_t)sbr_back_ws_doubles(n, b, nb),
                        sb, mx->oz_q1 ? &ozq1 : &oz, /*lean=*/!split));
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[3], sb));
  // ---- side A / side C: the chains start from the identity (OA holds the
  // stage-2 T factors from here on) ----
  double* PA = split ? XA : X;
  const long ldPA = split ? n : ldX;
  EVD_CUDA_TRY(cudaStreamWaitEvent(sa, ev[2], 0));
  if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[9], sa));
  EVD_TRY(set_identity(n, n, PA, ldPA, sa));
  if (split) {
    EVD_CUDA_TRY(cudaStreamWaitEvent(sc, ev[2], 0));
    EVD_TRY(set_identity(n, n, X, ldX, sc));
  }
  // ---- main: the chase, one launch per sweep range ----
  {
    NvtxRange r("evd_b200 bulge chasing");
    EVD_CUDA_TRY(cudaMemsetAsync(U, 0, sizeof(double) * n * n, st));
    for (int i = 0; i < nr; ++i) {
      EVD_TRY(chase_part_async(n, b, sub, 2 * b, U, n, ich, bounds[i], bounds[i + 1], i, st));
      EVD_CUDA_TRY(cudaEventRecord(evr[i], st));
    }
    EVD_TRY(chase_tridiag(n, sub, 2 * b, d, e, st));
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[4], st));
  // ---- the chains, range by range behind the chase ----
  {
    NvtxRange r("evd_b200 stage-2 reflectors beside the chase (side streams)");
    for (int i = 0; i < nr; ++i) {
      const bool in_b = split && bounds[i] >= k;
      cudaStream_t s2 = in_b ? sc : sa;
      EVD_CUDA_TRY(cudaStreamWaitEvent(s2, evr[i], 0));
      EVD_TRY(q2_apply_range(true, n, n, U, n, in_b ? X : PA, in_b ? ldX : ldPA, tbuf,
                             bounds[i], bounds[i + 1], in_b ? k : 0, s2));
    }
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[5], sa));
  EVD_CUDA_TRY(cudaEventRecord(ev[10], split ? sc : sa));
  // ---- main: D&C; Z goes into W once the Q1 formation no longer reads W.
  // With its own integer workspace the D&C starts right after the chase and
  // waits for the formation only before its last kernel writes Z; otherwise
  // it shares the formation's workspace and waits for the formation first.
  if (!dc_own) EVD_CUDA_TRY(cudaStreamWaitEvent(st, ev[3], 0));
  {
    NvtxRange r("evd_b200 tridiagonal divide and conquer");
    EVD_TRY(stedc(n, d, e, W, n, SW, (long)stedc_ws_doubles(n), ist, (long)stedc_ws_ints(n), st,
                  dc_own ? &ozdc : &oz, dc_own ? ev[3] : nullptr));
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[6], st));
  // ---- side A: the products (emulated, the main integer workspace; the Q1
  // formation has its own when the split buffer exists) ----
  if (split) {
    NvtxRange r("evd_b200 P = B A, Q^T = P Q1^T, X = Q Z (emulated, side stream)");
    // P = B A into U (the reflectors are dead once both chains are done); B
    // is the identity in its first k + 1 rows and columns
    EVD_CUDA_TRY(cudaStreamWaitEvent(sa, ev[10], 0));
    const long m = n - k - 1;
    EVD_TRY(copy_matrix(k + 1, n, XA, n, U, n, sa));
    EVD_TRY(oz_gemm('n', 'n', m, n, m, 1.0, X + (k + 1) + (k + 1) * ldX, ldX, XA + (k + 1), n,
                    0.0, nullptr, n, 0.0, U + (k + 1), n, mx->nmod, false, mx->oz, mx->oz_bytes,
                    sa));
    if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[12], sa));
    // Q^T = P Q1^T into the chain-A buffer
    EVD_CUDA_TRY(cudaStreamWaitEvent(sa, ev[3], 0));
    EVD_TRY(oz_gemm('n', 't', n, n, n, 1.0, U, n, dA, n, 0.0, nullptr, n, 0.0, XA, n, mx->nmod,
                    false, mx->oz, mx->oz_bytes, sa));
    // X = Q Z
    EVD_CUDA_TRY(cudaStreamWaitEvent(sa, ev[6], 0));
    EVD_TRY(oz_gemm('t', 'n', n, n, n, 1.0, XA, n, W, n, 0.0, nullptr, n, 0.0, X, ldX, mx->nmod,
                    false, mx->oz, mx->oz_bytes, sa));
  } else {
    NvtxRange r("evd_b200 X = Q1 (P^T Z) (emulated, side stream)");
    EVD_CUDA_TRY(cudaStreamWaitEvent(sa, ev[3], 0));
    EVD_CUDA_TRY(cudaStreamWaitEvent(sa, ev[6], 0));
    EVD_TRY(oz_gemm('t', 'n', n, n, n, 1.0, X, ldX, W, n, 0.0, nullptr, n, 0.0, Y, n, mx->nmod,
                    false, mx->oz, mx->oz_bytes, sa));
    if (timed) EVD_CUDA_TRY(cudaEventRecord(ev[12], sa));
    EVD_TRY(oz_gemm('n', 'n', n, n, n, 1.0, dA, n, Y, n, 0.0, nullptr, n, 0.0, X, ldX, mx->nmod,
                    false, mx->oz, mx->oz_bytes, sa));
  }
  EVD_CUDA_TRY(cudaEventRecord(ev[11], sa));
  EVD_CUDA_TRY(cudaStreamWaitEvent(st, ev[11], 0));
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
    auto el = [&](cudaEvent_t a, cudaEvent_t z) {
      float t = 0.f;
      // an event that this schedule did not record reads as 0 (and its
      // error must not reach the next launch check)
      if (cudaEventElapsedTime(&t, a, z) != cudaSuccess) {
        (void)cudaGetLastError();
        t = 0.f;
      }
      return (double)t;
    };
    g_mixed[0] = el(ev[0], ev[1]);
    g_mixed[1] = el(ev[1], ev[4]);
    g_mixed[2] = el(ev[4], ev[6]);
    g_mixed[3] = el(ev[2], ev[3]);
    g_mixed[4] = std::max(el(ev[9], ev[5]), el(ev[9], ev[10]));
    g_mixed[5] = el(ev[6], ev[7]);
    g_mixed[6] = el(ev[7], ev[8]);
    g_mixed[7] = el(ev[0], ev[8]);
    g_refine_ms = g_mixed[6];
    g_timings[0] = g_mixed[0];
    g_timings[1] = g_mixed[1];
    g_timings[2] = g_mixed[2];
    g_timings[3] = g_mixed[4];
    g_timings[4] = g_mixed[3];
    g_timings[5] = g_mixed[7];
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
// The full workspace (with the split buffer and the own integer workspaces
// up to kMixedDcOwnMax) and the minimum one (one stage-2 chain, the D&C after
// the Q1 formation), for callers short of device memory.
size_t syevd_mixed_ws_min_bytes(long n, long b, long nb, int nmod, int refine_iters) {
  const size_t plain = (syevd_any_ws_bytes(n, b, nb) + 255) / 256 * 256;
  const long np = padded_order(n, nb);
  return plain + (size_t)mixed_oz_bytes(np, nb, nmod, refine_iters) + 256;
}
size_t syevd_mixed_ws_bytes(long n, long b, long nb, int nmod, int refine_iters) {
  return syevd_mixed_ws_min_bytes(n, b, nb, nmod, refine_iters) +
         (size_t)mixed_extra(padded_order(n, nb), nb, nmod).total;
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
  if ((size_t)lwork_bytes < syevd_mixed_ws_min_bytes(n, b, nb, nmod, refine_iters))
    return EVD_ERR_WORKSPACE;
  const bool full = (size_t)lwork_bytes >= syevd_mixed_ws_bytes(n, b, nb, nmod, refine_iters);
  const size_t plain = (syevd_any_ws_bytes(n, b, nb) + 255) / 256 * 256;
  uint8_t* wb = reinterpret_cast<uint8_t*>(work);
  uint8_t* ozb = reinterpret_cast<uint8_t*>(((uintptr_t)(wb + plain) + 255) & ~(uintptr_t)255);
  const long ozn = mixed_oz_bytes(np, nb, nmod, refine_iters);
  const MixedExtra xt = mixed_extra(np, nb, nmod);
  uint8_t* xb = reinterpret_cast<uint8_t*>(((uintptr_t)(ozb + ozn) + 255) & ~(uintptr_t)255);
  MixedOpts mx{nmod, refine_iters, moduli_update, ozb, ozn, nullptr, 0, nullptr, 0, nullptr};
  if (full && xt.total > 0) {
    mx.oz_dc = xb;
    mx.oz_dc_bytes = xt.dc;
    mx.oz_q1 = xb + xt.dc;
    mx.oz_q1_bytes = xt.q1;
    mx.split_buf = reinterpret_cast<double*>(xb + xt.dc + xt.q1);
  }
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

extern "C" long evd_syevd_mixed_work_size_min(long n, long b, long nb, int moduli,
                                              int refine_iters) {
  if (!evd::shape_ok(n, b, nb) || moduli < evd::kOzMinMod || moduli > evd::kOzMaxMod ||
      refine_iters < 0)
    return 0;
  return (long)evd::syevd_mixed_ws_min_bytes(n, b, nb, moduli, refine_iters);
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

// ---- FP32 solve ----
// FP32 matrices in and out.  The contractions that dominate the work (the
// stage-1 trailing SYR2K, the Q1 formation, the large merges and the products
// that form X) run as emulated products with kFp32Moduli moduli (30-bit
// operands, no refinement), i.e. the mixed form at the accuracy FP32 needs;
// the panels, the chase and the divide and conquer stay FP64: they are
// latency-bound, so narrower arithmetic would not make them faster.  The
// workspace holds FP64 copies of A, w and X before the mixed form's own.
namespace evd {
namespace {

constexpr int kFp32Moduli = 8;

template <typename S, typename D>
__global__ void convert_kernel(long m, long n, const S* __restrict__ src, long lds,
                               D* __restrict__ dst, long ldd) {
  for (long j = blockIdx.y; j < n; j += gridDim.y)
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m;
         i += (long)gridDim.x * blockDim.x)
      dst[i + j * ldd] = (D)src[i + j * lds];
}

template <typename S, typename D>
int convert(long m, long n, const S* src, long lds, D* dst, long ldd, cudaStream_t st) {
  if (m <= 0 || n <= 0) return EVD_SUCCESS;
  dim3 grid(ceil_div_i(m, 256), (unsigned)std::min<long>(n, 65535));
  convert_kernel<S, D><<<grid, 256, 0, st>>>(m, n, src, lds, dst, ldd);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

size_t al256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

size_t syevd_s_ws_bytes(long n, long b, long nb) {
  const size_t sq = al256(sizeof(double) * (size_t)n * n);
  return 2 * sq + al256(sizeof(double) * (size_t)n) +
         syevd_mixed_ws_bytes(n, b, nb, kFp32Moduli, 0) + 256;
}

int syevd_s(long n, long b, long nb, const float* A, long lda, float* w, float* X, long ldX,
            void* work, long lwork_bytes, cudaStream_t st) {
  if (!shape_ok(n, b, nb)) return EVD_ERR_INVALID_ARG;
  if (lda < n || ldX < n || !A || !w || !X || !work) return EVD_ERR_INVALID_ARG;
  if ((size_t)lwork_bytes < syevd_s_ws_bytes(n, b, nb)) return EVD_ERR_WORKSPACE;
  uint8_t* p = reinterpret_cast<uint8_t*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
  const size_t sq = al256(sizeof(double) * (size_t)n * n);
  double* Ad = reinterpret_cast<double*>(p);
  double* Xd = reinterpret_cast<double*>(p + sq);
  double* wd = reinterpret_cast<double*>(p + 2 * sq);
  uint8_t* mw = p + 2 * sq + al256(sizeof(double) * (size_t)n);
  const size_t mbytes = syevd_mixed_ws_bytes(n, b, nb, kFp32Moduli, 0);
  EVD_TRY(convert(n, n, A, lda, Ad, n, st));
  EVD_TRY(syevd_mixed(n, b, nb, Ad, n, wd, Xd, n, kFp32Moduli, 0, kFp32Moduli, mw, (long)mbytes,
                      0, st));
  EVD_TRY(convert(n, 1, wd, n, w, n, st));
  EVD_TRY(convert(n, n, Xd, n, X, ldX, st));
  EVD_CUDA_TRY(cudaStreamSynchronize(st));
  return EVD_SUCCESS;
}

}  // namespace evd

extern "C" long evd_syevd_s_work_size(long n, long b, long nb) {
  if (!evd::shape_ok(n, b, nb)) return 0;
  return (long)evd::syevd_s_ws_bytes(n, b, nb);
}

extern "C" int evd_syevd_s(long n, long b, long nb, const float* A, long lda, float* w, float* X,
                           long ldX, void* work, long lwork_bytes, cudaStream_t stream) {
  try {
    return evd::syevd_s(n, b, nb, A, lda, w, X, ldX, work, lwork_bytes, stream);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

extern "C" double evd_syevd_last_refine_ms(void) { return evd::g_refine_ms; }


extern "C" void evd_syevd_mixed_last_timings(double out_ms[8]) {
  for (int i = 0; i < 8; ++i) out_ms[i] = evd::g_mixed[i];
}
