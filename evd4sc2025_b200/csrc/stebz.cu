// Eigenvalues of a symmetric tridiagonal matrix by Sturm-count multisection
// (the eigenvalues-only path; the reference always computes vectors, through
// LAPACKE_dstedc('I') at src/EVD/myEVD.cu:529).
//
// Count(x) = number of eigenvalues < x, from the LDL^T pivots in the form of
// LAPACK's dstebz/dlaebz:  q_0 = d_0 - x,  q_i = d_i - x - e_{i-1}^2 / q_{i-1},
// a pivot of magnitude <= pivmin replaced by -pivmin, count = number of
// negative pivots.  The matrix is first scaled by its largest entry.
//
// B200 layout: 8 lanes per eigenvalue (4 eigenvalues per warp).  Each pass the
// 8 lanes evaluate Count at 8 interior points of the current interval, so the
// interval shrinks 9x per pass (17 passes for 53 bits instead of 53 bisection
// steps): the pass is a chain of n dependent divisions, so fewer passes is
// what shortens the run; d and e^2 are read through the read-only path, the
// same address for the whole warp.
#include <math.h>

#include "common.cuh"

namespace evd {

namespace {

constexpr int kGroup = 8;  // lanes per eigenvalue

__global__ void stebz_prep_kernel(long n, const double* __restrict__ d,
                                  const double* __restrict__ e, double* __restrict__ ws) {
  // ws[0] = scale = max |d|, |e|; ws[1] = gl, ws[2] = gu (Gershgorin, scaled);
  // ws[3] = pivmin; ws[4 ..] = d/scale, then e^2/scale^2
  __shared__ double red[3][32];
  double m = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    m = fmax(m, fabs(d[i]));
    if (i < n - 1) m = fmax(m, fabs(e[i]));
  }
  m = warp_max(m);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[0][w] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s = fmax(s, red[0][k]);
    ws[0] = (s > 0.0) ? s : 1.0;
  }
  __syncthreads();
  const double inv = 1.0 / ws[0];
  double* ds = ws + 4;
  double* e2 = ws + 4 + n;
  double lo = 1e300, hi = -1e300, emax2 = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    const double di = d[i] * inv;
    const double el = (i > 0) ? fabs(e[i - 1]) * inv : 0.0;
    const double er = (i < n - 1) ? fabs(e[i]) * inv : 0.0;
    ds[i] = di;
    if (i < n - 1) {
      e2[i] = er * er;
      emax2 = fmax(emax2, er * er);
    }
    lo = fmin(lo, di - el - er);
    hi = fmax(hi, di + el + er);
  }
  lo = -warp_max(-lo);
  hi = warp_max(hi);
  emax2 = warp_max(emax2);
  if (lane == 0) {
    red[0][w] = lo;
    red[1][w] = hi;
    red[2][w] = emax2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 1e300, b = -1e300, c = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      a = fmin(a, red[0][k]);
      b = fmax(b, red[1][k]);
      c = fmax(c, red[2][k]);
    }
    const double pad = 2.0 * 2.220446049250313e-16 * fmax(fabs(a), fabs(b)) * (double)n + 1e-300;
    ws[1] = a - pad;
    ws[2] = b + pad;
    ws[3] = 2.2250738585072014e-308 * fmax(1.0, c);  // LAPACK pivmin = safmin * max(1, e^2)
  }
}

// Number of eigenvalues < x.
__device__ __forceinline__ int sturm_count(long n, const double* __restrict__ ds,
                                           const double* __restrict__ e2, double pivmin, double x) {
  double q = __ldg(ds) - x;
  if (fabs(q) <= pivmin) q = -pivmin;
  int c = (q < 0.0);
  for (long i = 1; i < n; ++i) {
    q = (__ldg(ds + i) - x) - __ldg(e2 + i - 1) / q;
    if (fabs(q) <= pivmin) q = -pivmin;
    c += (q < 0.0);
  }
  return c;
}

__global__ void stebz_kernel(long n, const double* __restrict__ ws, double* __restrict__ w) {
  const long gid = (blockIdx.x * (long)blockDim.x + threadIdx.x);
  const long k = gid / kGroup;  // eigenvalue index (ascending)
  const int j = threadIdx.x & (kGroup - 1);
  const int lane = threadIdx.x & 31;
  const unsigned gmask = 0xffu << (lane & ~(kGroup - 1));
  if (k >= n) return;  // whole groups leave together (n * kGroup threads used)
  const double scale = ws[0];
  const double pivmin = ws[3];
  const double* ds = ws + 4;
  const double* e2 = ws + 4 + n;
  double lo = ws[1], hi = ws[2];
  const double tol = 4.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi));
  for (int pass = 0; pass < 64 && hi - lo > tol; ++pass) {
    const double h = (hi - lo) / (kGroup + 1);
    const double x = lo + h * (j + 1);
    const int c = sturm_count(n, ds, e2, pivmin, x);
    // lanes whose point lies right of eigenvalue k (count > k)
    const unsigned right = __ballot_sync(gmask, c > k) & gmask;
    const int first = right ? (__ffs(right) - 1 - (lane & ~(kGroup - 1))) : kGroup;
    const double xl = __shfl_sync(gmask, x, (lane & ~(kGroup - 1)) + max(first - 1, 0));
    const double xr = __shfl_sync(gmask, x, (lane & ~(kGroup - 1)) + min(first, kGroup - 1));
    if (first < kGroup) hi = xr;
    if (first > 0) lo = xl;
  }
  if (j == 0) w[k] = 0.5 * (lo + hi) * scale;
}

}  // namespace

long stebz_ws_doubles(long n) { return 2 * n + 8; }

int stebz(long n, const double* d, const double* e, double* w, double* work, cudaStream_t st) {
  if (n < 0) return EVD_ERR_INVALID_ARG;
  if (n == 0) return EVD_SUCCESS;
  if (!d || !w || !work || (n > 1 && !e)) return EVD_ERR_INVALID_ARG;
  if (n > (1L << 26)) return EVD_ERR_INVALID_ARG;
  if (n == 1) {  // the eigenvalue is d_0, exactly
    EVD_CUDA_TRY(cudaMemcpyAsync(w, d, sizeof(double), cudaMemcpyDeviceToDevice, st));
    return EVD_SUCCESS;
  }
  stebz_prep_kernel<<<1, 1024, 0, st>>>(n, d, e, work);
  EVD_LAUNCHED();
  const long threads = n * kGroup;
  stebz_kernel<<<ceil_div_i(threads, 128), 128, 0, st>>>(n, work, w);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

}  // namespace evd

extern "C" long evd_stebz_work_size(long n) { return evd::stebz_ws_doubles(n < 0 ? 0 : n); }

extern "C" int evd_stebz(long n, const double* d, const double* e, double* w, double* work,
                         long lwork, cudaStream_t stream) {
  if (lwork < evd::stebz_ws_doubles(n < 0 ? 0 : n)) return EVD_ERR_WORKSPACE;
  return evd::stebz(n, d, e, w, work, stream);
}
