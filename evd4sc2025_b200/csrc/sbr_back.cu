// Stage-1 back transformation and the compact-WY utilities.
//
// Q1 = prod_p (I - W_p Y_p^T) over the b-wide panels of stage 1 (panel p at
// rows (p+1)b.., columns pb..pb+b-1 of dW/dY, zero elsewhere).
//
// evd_sbr_back: X <- Q1 X.  Panels are first merged into nk-wide slabs
// (I - W_s Y_s^T = product of the slab's panels) by recursive doubling, the
// same batched merge as my_SBRBack_BCBack (src/EVD/myEVD.cu:148-207); then
// the slabs are applied last to first: T = Y_s^T X, X -= W_s T.  The
// reference instead builds Q1 explicitly from I (4n^3 flops, :213-233),
// transposes it (:235-239) and multiplies by Z at the end (:564, 2n^3); the
// application here is 2 n^2 ncols flops on the vectors directly.
//
// evd_wy_from_slide: computerWYFromSlide (api/computerWYFromSlide.cu:5-25).
// evd_q_from_wy:     computerQFromWY (api/computerQFromWY.cu:5-17).
#include "common.cuh"
#include "gemm_f64.cuh"
#include "ozaki.cuh"

namespace evd {

namespace {

__global__ void set_identity_kernel(long m, long n, double* Q, long ldq) {
  for (long j = blockIdx.y; j < n; j += gridDim.y)
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m;
         i += (long)gridDim.x * blockDim.x)
      Q[i + j * ldq] = (i == j) ? 1.0 : 0.0;
}

}  // namespace

int set_identity(long m, long n, double* Q, long ldq, cudaStream_t st) {
  if (m <= 0 || n <= 0) return EVD_SUCCESS;
  dim3 grid(ceil_div_i(m, 256), (unsigned)std::min<long>(n, 65535));
  set_identity_kernel<<<grid, 256, 0, st>>>(m, n, Q, ldq);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

// In-place merge of the panels of every nk-wide slab (recursive doubling over
// widths b, 2b, ..., nk/2).  dW/dY: n x ncolsWY (ncolsWY = number of panel
// columns), rows b..n-1 used.  work: >= n * nk / 2 doubles.
int wy_merge_slabs(long n, long b, long nk, long ncolsWY, double* dW, long ldW, const double* dY,
                   long ldY, double* work, cudaStream_t st) {
  const long rows = n - b;
  if (rows <= 0) return EVD_SUCCESS;
  for (long c = b; c < nk; c *= 2) {
    // pairs (L, R) of width c: L = cols [2jc, 2jc+c), R = [2jc+c, 2jc+2c)
    long npairs = ncolsWY / (2 * c);
    long rem = ncolsWY - npairs * 2 * c;  // a trailing partial pair (last slab)
    if (npairs > 0) {
      // T_j = Y_L^T W_R (c x c), W_R -= W_L T_j
      EVD_TRY(dgemm_batched('t', 'n', c, c, rows, 1.0, dY + b, ldY, 2 * c * ldY,
                            dW + b + c * ldW, ldW, 2 * c * ldW, 0.0, work, c, c * c, npairs,
                            st));
      EVD_TRY(dgemm_batched('n', 'n', rows, c, c, -1.0, dW + b, ldW, 2 * c * ldW, work, c, c * c,
                            1.0, dW + b + c * ldW, ldW, 2 * c * ldW, npairs, st));
    }
    if (rem > c) {
      // partial pair at the end: L has width c, R has width rem - c
      long j0 = npairs * 2 * c;
      long cr = rem - c;
      EVD_TRY(dgemm('t', 'n', c, cr, rows, 1.0, dY + b + j0 * ldY, ldY, dW + b + (j0 + c) * ldW,
                    ldW, 0.0, work, c, st));
      EVD_TRY(dgemm('n', 'n', rows, cr, c, -1.0, dW + b + j0 * ldW, ldW, work, c, 1.0,
                    dW + b + (j0 + c) * ldW, ldW, st));
    }
  }
  return EVD_SUCCESS;
}

long sbr_back_ws_doubles(long n, long b, long nk) {
  (void)b;
  return std::max(n * nk / 2, nk * n) + 64;
}

// Emulated-product workspace of sbr_form_q1 (bytes): the larger of its two
// products' (T = Y_s^T M with K = rows, M -= W_s T with K = nk).
long sbr_form_oz_bytes(long n, long nk, int nmod) {
  return std::max(oz_layout(nk, n, n, nmod, false).bytes, oz_layout(n, n, nk, nmod, true).bytes);
}

// X <- Q1 X using slab-merged W (call wy_merge_slabs first).
int sbr_apply_slabs(long n, long b, long nk, const double* dW, long ldW, const double* dY,
                    long ldY, double* X, long ldX, long ncols, double* work, size_t work_n,
                    cudaStream_t st) {
  const long npcols = ((n - 1) / b) * b;  // panel columns (stage 1 leaves the last b-block)
  if (npcols <= 0 || ncols <= 0) return EVD_SUCCESS;
  const long nslabs = (npcols + nk - 1) / nk;
  for (long s = nslabs - 1; s >= 0; --s) {
    const long c0 = s * nk;
    const long w = std::min(nk, npcols - c0);
    const long r0 = c0 + b;  // first row with panel data in this slab
    const long m = n - r0;
    if (m <= 0 || w <= 0) continue;
    // T = Y_s^T X[r0:, :]  (w x ncols), then X[r0:, :] -= W_s T
    if ((size_t)(w * ncols) > work_n) return EVD_ERR_WORKSPACE;
    EVD_TRY(dgemm('t', 'n', w, ncols, m, 1.0, dY + r0 + c0 * ldY, ldY, X + r0, ldX, 0.0, work, w,
                  st));
    EVD_TRY(dgemm('n', 'n', m, ncols, w, -1.0, dW + r0 + c0 * ldW, ldW, work, w, 1.0, X + r0,
                  ldX, st));
  }
  return EVD_SUCCESS;
}

// Q1 = prod_p (I - W_p Y_p^T) formed explicitly into M (slab-merged W, Y:
// call wy_merge_slabs first).  M = I, then for the slabs last to first
//   M[r0:, r0:] -= W_s (Y_s^T M[r0:, r0:])
// where r0 is the slab's first row: outside rows and columns r0.. M is still
// the identity, so the products shrink with the slab index and the whole
// formation costs (4/3) n^3 flops instead of 2 n^3 (the reference forms Q1
// from I the same way, src/EVD/myEVD.cu:213-233, over the full matrix).
// oz != nullptr: emulated products (lean: the 2-stage integer GEMM, which
// shares SMs with the bulge chase running beside it).
int sbr_form_q1(long n, long b, long nk, const double* dW, long ldW, const double* dY, long ldY,
                double* M, long ldM, double* work, size_t work_n, cudaStream_t st,
                const OzWork* oz, bool lean) {
  EVD_TRY(set_identity(n, n, M, ldM, st));
  const long npcols = ((n - 1) / b) * b;
  if (npcols <= 0) return EVD_SUCCESS;
  const long nslabs = (npcols + nk - 1) / nk;
  for (long s = nslabs - 1; s >= 0; --s) {
    const long c0 = s * nk;
    const long w = std::min(nk, npcols - c0);
    const long r0 = c0 + b;
    const long m = n - r0;
    if (m <= 0 || w <= 0) continue;
    if ((size_t)(w * m) > work_n) return EVD_ERR_WORKSPACE;
    double* Mb = M + r0 + r0 * ldM;
    if (oz) {
      EVD_TRY(oz_gemm('t', 'n', w, m, m, 1.0, dY + r0 + c0 * ldY, ldY, Mb, ldM, 0.0, nullptr, w,
                      0.0, work, w, oz->nmod, false, oz->ws, oz->bytes, st, lean));
      EVD_TRY(oz_gemm('n', 'n', m, m, w, -1.0, dW + r0 + c0 * ldW, ldW, work, w, 1.0, Mb, ldM,
                      0.0, Mb, ldM, oz->nmod, false, oz->ws, oz->bytes, st, lean));
    } else {
      EVD_TRY(dgemm('t', 'n', w, m, m, 1.0, dY + r0 + c0 * ldY, ldY, Mb, ldM, 0.0, work, w, st));
      EVD_TRY(dgemm('n', 'n', m, m, w, -1.0, dW + r0 + c0 * ldW, ldW, work, w, 1.0, Mb, ldM, st));
    }
  }
  return EVD_SUCCESS;
}

}  // namespace evd

extern "C" long evd_sbr_back_work_size(long n, long b, long nk) {
  if (n <= 0 || b <= 0 || nk <= 0) return 0;
  return evd::sbr_back_ws_doubles(n, b, nk);
}

extern "C" int evd_sbr_back(long n, long b, long nk, double* dW, long ldW, const double* dY,
                            long ldY, double* X, long ldX, long ncols, double* work, long lwork,
                            cudaStream_t stream) {
  if (n < 0 || b <= 0 || nk < b || (nk % b) != 0 || ldW < n || ldY < n || ldX < n || ncols < 0)
    return EVD_ERR_INVALID_ARG;
  // slab width must be b times a power of two (recursive doubling)
  long q = nk / b;
  if (q & (q - 1)) return EVD_ERR_INVALID_ARG;
  if (n == 0 || ncols == 0) return EVD_SUCCESS;
  if (!dW || !dY || !X || !work) return EVD_ERR_INVALID_ARG;
  if (lwork < evd::sbr_back_ws_doubles(n, b, nk)) return EVD_ERR_WORKSPACE;
  const long npcols = ((n - 1) / b) * b;
  EVD_TRY(evd::wy_merge_slabs(n, b, nk, npcols, dW, ldW, dY, ldY, work, stream));
  return evd::sbr_apply_slabs(n, b, nk, dW, ldW, dY, ldY, X, ldX, ncols, work, (size_t)lwork,
                              stream);
}

extern "C" int evd_wy_from_slide(long M, long N, long slideWidth, double* dW, long ldW,
                                 const double* dY, long ldY, double* work, cudaStream_t stream) {
  const long b = slideWidth;
  if (M < 0 || N < 0 || b <= 0 || ldW < M || ldY < M) return EVD_ERR_INVALID_ARG;
  if (M == 0 || N <= b) return EVD_SUCCESS;
  if (!dW || !dY || !work) return EVD_ERR_INVALID_ARG;
  // work: (i-b) x b with leading dimension M, as the reference (ldWork = M)
  for (long i = 2 * b; i <= N; i += b) {
    EVD_TRY(evd::dgemm('t', 'n', i - b, b, M, 1.0, dY, ldY, dW + (i - b) * ldW, ldW, 0.0, work, M,
                       stream));
    EVD_TRY(evd::dgemm('n', 'n', M, b, i - b, -1.0, dW, ldW, work, M, 1.0, dW + (i - b) * ldW,
                       ldW, stream));
  }
  return EVD_SUCCESS;
}

extern "C" int evd_q_from_wy(long M, long N, double* dQ, long ldQ, const double* dW, long ldW,
                             const double* dY, long ldY, cudaStream_t stream) {
  if (M < 0 || N < 0 || ldQ < M || ldW < M || ldY < M) return EVD_ERR_INVALID_ARG;
  if (M == 0) return EVD_SUCCESS;
  if (!dQ || (N > 0 && (!dW || !dY))) return EVD_ERR_INVALID_ARG;
  EVD_TRY(evd::set_identity(M, M, dQ, ldQ, stream));
  return evd::dgemm('n', 't', M, M, N, -1.0, dW, ldW, dY, ldY, 1.0, dQ, ldQ, stream);
}
