// Iterative refinement of a symmetric eigendecomposition (Ogita & Aishima,
// "Iterative refinement for symmetric eigenvalue decomposition", Japan J.
// Indust. Appl. Math. 35 (2018), Algorithm 1, RefSyEv).  The reference has no
// refinement; this is the step a mixed-precision solver uses to win FP64
// accuracy back from eigenpairs computed in lower precision.
//
// One iteration, for A (n x n, symmetric) and an approximate eigenvector
// matrix X:
//   R = I - X^T X,  S = X^T A X           (three FP64 DMMA GEMMs)
//   l_i = s_ii / (1 - r_ii)
//   delta = 2 (||S - diag(l)||_2 + ||A||_2 ||R||_2), floored at the level
//           where the rounding noise of S would dominate a correction
//   E_ij = (s_ij + l_j r_ij) / (l_j - l_i)  if |l_i - l_j| > delta,
//          r_ij / 2                          otherwise (clustered pairs)
//   X <- X + X E                           (one FP64 GEMM)
// The error in X falls quadratically while it is well below the eigenvalue
// gaps.  ||A||_2 is taken as max |l_i|; ||S - diag(l)||_2 and ||R||_2 are
// estimated by power iteration (10 steps, result scaled by 1.5) on the
// device, so an iteration needs no host synchronisation.
#include <math.h>

#include "common.cuh"
#include "gemm_f64.cuh"
#include "ozaki.cuh"

namespace evd {

int copy_matrix(long m, long n, const double* src, long lds, double* dst, long ldd,
                cudaStream_t st);

namespace {

constexpr int kPowerSteps = 10;

// scal[0] = ||A||_2 estimate, [1] = ||S - D||_2, [2] = ||R||_2, [3] = delta,
// [4..5] = running norms of the two power iterations
struct RefineLayout {
  size_t AX, S, R, lam, v0, v1, y0, y1, scal, end;
};

RefineLayout refine_layout(long n) {
  auto al = [](size_t x) { return (x + 31) / 32 * 32; };
  RefineLayout L{};
  size_t o = 0;
  const size_t nn = (size_t)n * n;
  L.AX = o; o = al(o + nn);
  L.S = o; o = al(o + nn);
  L.R = o; o = al(o + nn);
  L.lam = o; o = al(o + n);
  L.v0 = o; o = al(o + n);
  L.v1 = o; o = al(o + n);
  L.y0 = o; o = al(o + n);
  L.y1 = o; o = al(o + n);
  L.scal = o; o = al(o + 32);
  L.end = o + 32;  // room for aligning the base
  return L;
}

__device__ __forceinline__ void atomic_max_nonneg(double* p, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

// R_ii += 1; l_i = S_ii / (1 - R_ii); scal[0] = max |l_i|; start vectors
__global__ void lambda_kernel(long n, const double* __restrict__ S, long lds, double* __restrict__ R,
                              long ldr, double* __restrict__ lam, double* __restrict__ v0,
                              double* __restrict__ v1, double* scal) {
  double m = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double r = R[i + i * ldr] + 1.0;
    R[i + i * ldr] = r;
    const double l = S[i + i * lds] / (1.0 - r);
    lam[i] = l;
    m = fmax(m, fabs(l));
    // deterministic pseudo-random start vectors (unnormalised: the first
    // power step normalises)
    unsigned long long h = (unsigned long long)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    h ^= h >> 29;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 32;
    const double u = (double)(h >> 11) * (1.0 / 9007199254740992.0) - 0.5;
    v0[i] = u;
    v1[i] = 0.5 - u * u;
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(scal, m);
}

// y = M v for M = S - diag(lam) (which = 0) or M = R (which = 1); one warp per
// column j (M symmetric: y_j = column j . v), coalesced column reads.
__global__ void symv_kernel(long n, const double* __restrict__ M, long ldm,
                            const double* __restrict__ lam, const double* __restrict__ v,
                            double* __restrict__ y, int sub_diag) {
  const long warps = (long)gridDim.x * (blockDim.x >> 5);
  const int lane = threadIdx.x & 31;
  for (long j = blockIdx.x * (long)(blockDim.x >> 5) + (threadIdx.x >> 5); j < n; j += warps) {
    const double* col = M + j * ldm;
    double acc = 0.0;
    for (long i = lane; i < n; i += 32) acc = fma(col[i], v[i], acc);
    acc = warp_sum(acc);
    if (lane == 0) y[j] = sub_diag ? acc - lam[j] * v[j] : acc;
  }
}

// v = y / ||y||; out = ||y|| (single block)
__global__ void normalize_kernel(long n, const double* __restrict__ y, double* __restrict__ v,
                                 double* out) {
  __shared__ double red[32];
  double s = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) s = fma(y[i], y[i], s);
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  double t = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
  const double nrm = sqrt(t);
  const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) v[i] = y[i] * inv;
  if (threadIdx.x == 0) *out = nrm;
}

__global__ void delta_kernel(double* scal, long n) {
  // the power iteration approaches the norm from below: scale by 1.5.  Floor:
  // S carries rounding noise of about sqrt(n) u ||A||; a pair whose gap is
  // below 1e8 times that noise would get a correction with a relative error
  // above 1e-8, so it is refined as part of a cluster instead
  const double est = 2.0 * (1.5 * scal[4] + scal[0] * 1.5 * scal[5]);
  const double noise = sqrt((double)n) * 1.1102230246251565e-16 * scal[0];
  scal[3] = fmax(est, 1e8 * noise);
}

// E (into R, tile by tile): with s = (s_ij + s_ji) / 2 (S symmetrised, so that
// E + E^T = R holds exactly and X^T X - I falls to second order),
// E_ij = (s + l_j r_ij) / (l_j - l_i) if |l_i - l_j| > delta, else r_ij / 2;
// the diagonal gets r_ii / 2.  32 x 32 tiles, S_ji through shared memory.
__global__ void correction_kernel(long n, const double* __restrict__ S, long lds,
                                  double* __restrict__ R, long ldr, const double* __restrict__ lam,
                                  const double* scal) {
  __shared__ double st[32][33];
  const double delta = scal[3];
  const long i0 = (long)blockIdx.x * 32, j0 = (long)blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const long row = j0 + threadIdx.x, col = i0 + r;  // S(j0 + tx, i0 + r)
    st[threadIdx.x][r] = (row < n && col < n) ? S[row + col * lds] : 0.0;
  }
  __syncthreads();
  const long i = i0 + threadIdx.x;
  if (i >= n) return;
  const double li = lam[i];
  for (int c = threadIdx.y; c < 32; c += blockDim.y) {
    const long j = j0 + c;
    if (j >= n) break;
    const double lj = lam[j];
    const double sij = 0.5 * (S[i + j * lds] + st[c][threadIdx.x]);  // st[c][tx] = S(j, i)
    const double r = R[i + j * ldr];
    const double d = lj - li;
    R[i + j * ldr] = (i != j && fabs(d) > delta) ? (sij + lj * r) / d : 0.5 * r;
  }
}

// The per-iteration steps after the products: eigenvalue estimates, norm
// estimates by power iteration, the cluster threshold and the correction E
// (into R).  S must be symmetric or is symmetrised; R holds -X^T X on entry.
int refine_middle(long n, const double* S, double* R, double* lam, double* v0, double* v1,
                  double* y0, double* y1, double* scal, cudaStream_t st) {
  const int threads = 256;
  const int gblocks = (int)std::min<long>(ceil_div_i(n, threads), 1024);
  const int wblocks = (int)std::min<long>(ceil_div_i(n, threads / 32), 4096);
  EVD_CUDA_TRY(cudaMemsetAsync(scal, 0, sizeof(double) * 32, st));
  lambda_kernel<<<gblocks, threads, 0, st>>>(n, S, n, R, n, lam, v0, v1, scal);
  EVD_LAUNCHED();
  for (int p = 0; p < kPowerSteps; ++p) {
    symv_kernel<<<wblocks, threads, 0, st>>>(n, S, n, lam, v0, y0, 1);
    EVD_LAUNCHED();
    normalize_kernel<<<1, 1024, 0, st>>>(n, y0, v0, scal + 4);
    EVD_LAUNCHED();
    symv_kernel<<<wblocks, threads, 0, st>>>(n, R, n, lam, v1, y1, 0);
    EVD_LAUNCHED();
    normalize_kernel<<<1, 1024, 0, st>>>(n, y1, v1, scal + 5);
    EVD_LAUNCHED();
  }
  delta_kernel<<<1, 1, 0, st>>>(scal, n);
  EVD_LAUNCHED();
  const unsigned tiles = (unsigned)((n + 31) / 32);
  correction_kernel<<<dim3(tiles, tiles), dim3(32, 8), 0, st>>>(n, S, n, R, n, lam, scal);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

// Workspace of the emulated-product refinement (bytes): the FP64 part of the
// DMMA version (3 n^2 + O(n) doubles) plus three quantised operands of
// `moduli` planes of n x ld bytes, the residue planes and the exponents
// (`with_f64` = false: the integer part only, from offset 0).
struct OzRefineLayout {
  size_t f64, qa, qx, qp, res, ea, ex, ep, end;
};

OzRefineLayout oz_refine_layout(long n, int moduli, bool with_f64 = true) {
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  OzRefineLayout L{};
  const size_t planes = (size_t)moduli * n * oz_ld(n);
  size_t o = 0;
  L.f64 = o; o = with_f64 ? al(o + 8 * refine_layout(n).end) : 0;
  L.qa = o; o = al(o + planes);
  L.qx = o; o = al(o + planes);
  L.qp = o; o = al(o + planes);
  L.res = o; o = al(o + (size_t)moduli * ((n + 15) / 16 * 16) * n);
  L.ea = o; o = al(o + 4 * n);
  L.ex = o; o = al(o + 4 * n);
  L.ep = o; o = al(o + 4 * n);
  L.end = o + 256;
  return L;
}

}  // namespace

long refine_ws_doubles(long n) { return (long)refine_layout(n).end; }

long refine_oz_ws_bytes(long n, int moduli) { return (long)oz_refine_layout(n, moduli).end; }
long refine_oz_int_bytes(long n, int moduli) {
  return (long)oz_refine_layout(n, moduli, false).end;
}

// RefSyEv with every product emulated on the integer tensor cores:
//   P = A X, R = -X^T X and S = X^T P with `moduli` moduli (14: FP64-level),
//   X <- X + X E with `moduli_update` moduli (E is small, so fewer bits of
//   it are needed for the same absolute accuracy).
// X^T X and X^T P are symmetric: only their lower tiles are multiplied and
// the CRT mirrors them.  A is quantised once for all iterations.
// f64: refine_ws_doubles(n) doubles; iwork: refine_oz_int_bytes(n, moduli)
// bytes (256-byte aligned)
int refine_syev_oz_split(long n, const double* A, long lda, double* w, double* X, long ldX,
                         int iters, int moduli, int moduli_update, double* f64, uint8_t* iwork,
                         cudaStream_t st) {
  if (n < 0 || iters < 0) return EVD_ERR_INVALID_ARG;
  if (n == 0 || iters == 0) return EVD_SUCCESS;
  if (!A || !w || !X || !f64 || !iwork || lda < n || ldX < n) return EVD_ERR_INVALID_ARG;
  if (n > 65535 || moduli < kOzMinMod || moduli > kOzMaxMod || moduli_update < kOzMinMod ||
      moduli_update > moduli)
    return EVD_ERR_INVALID_ARG;
  const OzRefineLayout L = oz_refine_layout(n, moduli, false);
  uint8_t* b8 = iwork;
  const RefineLayout F = refine_layout(n);
  double* base = reinterpret_cast<double*>(((uintptr_t)f64 + 255) & ~(uintptr_t)255);
  double *P = base + F.AX, *S = base + F.S, *R = base + F.R, *lam = base + F.lam;
  double *v0 = base + F.v0, *v1 = base + F.v1, *y0 = base + F.y0, *y1 = base + F.y1;
  double* scal = base + F.scal;
  int8_t* qa = reinterpret_cast<int8_t*>(b8 + L.qa);
  int8_t* qx = reinterpret_cast<int8_t*>(b8 + L.qx);
  int8_t* qp = reinterpret_cast<int8_t*>(b8 + L.qp);
  uint8_t* res = b8 + L.res;
  int* ea = reinterpret_cast<int*>(b8 + L.ea);
  int* ex = reinterpret_cast<int*>(b8 + L.ex);
  int* ep = reinterpret_cast<int*>(b8 + L.ep);
  // rows of A = columns of A (symmetric)
  EVD_TRY(oz_quantize(n, n, A, lda, qa, ea, moduli, st));
  for (int it = 0; it < iters; ++it) {
    EVD_TRY(oz_quantize(n, n, X, ldX, qx, ex, moduli, st));
    // P = A X
    EVD_TRY(oz_imma(n, n, n, qa, qx, res, moduli, false, st));
    EVD_TRY(oz_crt(n, n, n, res, ea, ex, moduli, 1.0, 0.0, nullptr, n, 0.0, P, n, false, st));
    // R = -X^T X (lower tiles, mirrored)
    EVD_TRY(oz_imma(n, n, n, qx, qx, res, moduli, true, st));
    EVD_TRY(oz_crt(n, n, n, res, ex, ex, moduli, -1.0, 0.0, nullptr, n, 0.0, R, n, true, st));
    // S = X^T P (lower tiles, mirrored)
    EVD_TRY(oz_quantize(n, n, P, n, qp, ep, moduli, st));
    EVD_TRY(oz_imma(n, n, n, qx, qp, res, moduli, true, st));
    EVD_TRY(oz_crt(n, n, n, res, ex, ep, moduli, 1.0, 0.0, nullptr, n, 0.0, S, n, true, st));
    EVD_TRY(refine_middle(n, S, R, lam, v0, v1, y0, y1, scal, st));
    // X <- X + X E: rows of X (through X^T in S, free now) and columns of E (in R)
    EVD_TRY(oz_transpose(n, n, X, ldX, S, n, st));
    EVD_TRY(oz_quantize(n, n, S, n, qp, ep, moduli_update, st));
    EVD_TRY(oz_quantize(n, n, R, n, qx, ex, moduli_update, st));
    EVD_TRY(oz_imma(n, n, n, qp, qx, res, moduli_update, false, st));
    EVD_TRY(oz_crt(n, n, n, res, ep, ex, moduli_update, 1.0, 1.0, X, ldX, 0.0, X, ldX, false,
                   st));
  }
  EVD_CUDA_TRY(cudaMemcpyAsync(w, lam, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  return EVD_SUCCESS;
}

int refine_syev(long n, const double* A, long lda, double* w, double* X, long ldX, int iters,
                double* work, long lwork, cudaStream_t st) {
  if (n < 0 || iters < 0) return EVD_ERR_INVALID_ARG;
  if (n == 0 || iters == 0) return EVD_SUCCESS;
  if (!A || !w || !X || !work || lda < n || ldX < n) return EVD_ERR_INVALID_ARG;
  if (n > 65535) return EVD_ERR_INVALID_ARG;  // keeps the tile grid and index products small
  const RefineLayout L = refine_layout(n);
  if (lwork < (long)L.end) return EVD_ERR_WORKSPACE;
  double* base = reinterpret_cast<double*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
  double *AX = base + L.AX, *S = base + L.S, *R = base + L.R, *lam = base + L.lam;
  double *v0 = base + L.v0, *v1 = base + L.v1, *y0 = base + L.y0, *y1 = base + L.y1;
  double* scal = base + L.scal;
  for (int it = 0; it < iters; ++it) {
    EVD_TRY(dgemm('n', 'n', n, n, n, 1.0, A, lda, X, ldX, 0.0, AX, n, st));
    EVD_TRY(dgemm('t', 'n', n, n, n, 1.0, X, ldX, AX, n, 0.0, S, n, st));
    EVD_TRY(dgemm('t', 'n', n, n, n, -1.0, X, ldX, X, ldX, 0.0, R, n, st));
    EVD_TRY(refine_middle(n, S, R, lam, v0, v1, y0, y1, scal, st));
    // X <- X + X E (E in R; through AX, which is free now)
    EVD_TRY(copy_matrix(n, n, X, ldX, AX, n, st));
    EVD_TRY(dgemm('n', 'n', n, n, n, 1.0, X, ldX, R, n, 1.0, AX, n, st));
    EVD_TRY(copy_matrix(n, n, AX, n, X, ldX, st));
  }
  EVD_CUDA_TRY(cudaMemcpyAsync(w, lam, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  return EVD_SUCCESS;
}

int refine_syev_oz(long n, const double* A, long lda, double* w, double* X, long ldX, int iters,
                   int moduli, int moduli_update, void* work, long lwork, cudaStream_t st) {
  if (n < 0 || iters < 0) return EVD_ERR_INVALID_ARG;
  if (n == 0 || iters == 0) return EVD_SUCCESS;
  if (n > 65535 || moduli < kOzMinMod || moduli > kOzMaxMod) return EVD_ERR_INVALID_ARG;
  if (!work) return EVD_ERR_INVALID_ARG;
  const OzRefineLayout L = oz_refine_layout(n, moduli);
  if (lwork < (long)L.end) return EVD_ERR_WORKSPACE;
  uint8_t* b8 = reinterpret_cast<uint8_t*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
  return refine_syev_oz_split(n, A, lda, w, X, ldX, iters, moduli, moduli_update,
                              reinterpret_cast<double*>(b8 + L.f64), b8 + L.qa, st);
}

}  // namespace evd

extern "C" long evd_refine_syev_work_size(long n) {
  if (n < 0 || n > 65535) return 0;
  return evd::refine_ws_doubles(n);
}

extern "C" int evd_refine_syev(long n, const double* A, long lda, double* w, double* X, long ldX,
                               int iters, double* work, long lwork, cudaStream_t stream) {
  return evd::refine_syev(n, A, lda, w, X, ldX, iters, work, lwork, stream);
}

extern "C" long evd_refine_syev_ozaki_work_size(long n, int moduli) {
  if (n < 0 || n > 65535 || moduli < evd::kOzMinMod || moduli > evd::kOzMaxMod) return 0;
  return evd::refine_oz_ws_bytes(n, moduli);
}

extern "C" int evd_refine_syev_ozaki(long n, const double* A, long lda, double* w, double* X,
                                     long ldX, int iters, int moduli, int moduli_update,
                                     void* work, long lwork_bytes, cudaStream_t stream) {
  try {
    EVD_TRY(evd::refine_syev_oz(n, A, lda, w, X, ldX, iters, moduli, moduli_update, work,
                                lwork_bytes, stream));
    return evd::oz_check_err(stream);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}
