// Accuracy metrics of an eigendecomposition (FP64 on the device).
//
// evd_check_orthogonality: ||A^T B - I||_F / M, the reference's
//   checkOrthogonality (util/tool/checkMetric.cu:5-24: Dgemm, IminusQ, Dnrm2),
//   returned instead of printed.
// evd_check_eig: residual ||A X - X diag(w)||_F / (n ||A||_F) and
//   orthogonality ||X^T X - I||_F / n.
// Norms are reduced in a fixed order (per-block partials, then one block), so
// the result is deterministic.
#include <mutex>

#include "common.cuh"
#include "gemm_f64.cuh"

namespace evd {

namespace {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 592;

// partial[b] = sum over this block's elements of (M[i,j] - shift*delta_ij - w_j*Y[i,j])^2
__global__ void sumsq_kernel(long m, long n, const double* __restrict__ M, long ldm, double shift,
                             const double* __restrict__ Y, long ldy, const double* __restrict__ w,
                             double* __restrict__ partial) {
  __shared__ double red[kRedThreads / 32];
  double s = 0.0;
  const long total = m * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    long i = idx % m, j = idx / m;
    double v = M[i + j * ldm];
    if (i == j) v -= shift;
    if (Y) v = fma(-w[j], Y[i + j * ldy], v);
    s = fma(v, v, s);
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = (threadIdx.x < kRedThreads / 32) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
  }
}

__global__ void final_sum_kernel(int nparts, const double* __restrict__ partial,
                                 double* __restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += partial[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = (threadIdx.x < (int)(blockDim.x / 32)) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) *out = t;
  }
}

// Reduction partials of the metrics (8 KB, module scope): the reference gives
// checkOrthogonality exactly an M x M work buffer, so the partial sums cannot
// live there.  Calls that overlap on the GPU share it.
__device__ double g_metric_partials[kRedBlocks + 16];

}  // namespace

// Device address of g_metric_partials on the current device (the runtime keeps
// one copy of the module per device), cached per device under a lock.
static int metric_scratch(double** p) {
  constexpr int kMaxDev = 64;
  static std::mutex mu;
  static double* addr[kMaxDev] = {};
  int d = -1;
  EVD_CUDA_TRY(cudaGetDevice(&d));
  if (d < 0 || d >= kMaxDev) return EVD_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(mu);
  if (addr[d] == nullptr) EVD_CUDA_TRY(cudaGetSymbolAddress((void**)&addr[d], g_metric_partials));
  *p = addr[d];
  return EVD_SUCCESS;
}

// sqrt(sum (M - shift I - Y diag(w))^2) into *dout (device); scratch >= kRedBlocks doubles
int frob_norm_dev(long m, long n, const double* M, long ldm, double shift, const double* Y,
                  long ldy, const double* w, double* scratch, double* dout, cudaStream_t st) {
  int blocks = (int)std::min<long>(kRedBlocks, std::max<long>(1, (m * n + 255) / 256));
  sumsq_kernel<<<blocks, kRedThreads, 0, st>>>(m, n, M, ldm, shift, Y, ldy, w, scratch);
  EVD_LAUNCHED();
  final_sum_kernel<<<1, 256, 0, st>>>(blocks, scratch, dout);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

}  // namespace evd

extern "C" int evd_check_orthogonality(long M, long N, const double* dA, long ldA,
                                       const double* dB, long ldB, double* work, double* result,
                                       cudaStream_t stream) {
  if (M <= 0 || N < 0 || ldA < N || ldB < N || !dA || !dB || !work || !result)
    return EVD_ERR_INVALID_ARG;
  // The reference computes A^T B with A, B of M columns and N rows
  // (cublasDgemm(T, N, M, M, N, ...)); work holds the M x M product.
  EVD_TRY(evd::dgemm('t', 'n', M, M, N, 1.0, dA, ldA, dB, ldB, 0.0, work, M, stream));
  double* scratch = nullptr;
  EVD_TRY(evd::metric_scratch(&scratch));
  EVD_TRY(evd::frob_norm_dev(M, M, work, M, 1.0, nullptr, 0, nullptr, scratch + 8, scratch,
                             stream));
  double h = 0.0;
  EVD_CUDA_TRY(cudaMemcpyAsync(&h, scratch, sizeof(double), cudaMemcpyDeviceToHost, stream));
  EVD_CUDA_TRY(cudaStreamSynchronize(stream));
  result[0] = sqrt(h) / (double)M;
  return EVD_SUCCESS;
}

extern "C" int evd_check_eig(long n, const double* A, long lda, const double* w, const double* X,
                             long ldX, double* work, double* result, cudaStream_t stream) {
  if (n <= 0 || lda < n || ldX < n || !A || !w || !X || !work || !result)
    return EVD_ERR_INVALID_ARG;
  double* AX = work;  // n x n
  double* scratch = nullptr;
  EVD_TRY(evd::metric_scratch(&scratch));
  double* sums = scratch;    // [0] resid^2 [1] ||A||^2 [2] orth^2
  double* part = scratch + 8;
  EVD_TRY(evd::dgemm('n', 'n', n, n, n, 1.0, A, lda, X, ldX, 0.0, AX, n, stream));
  EVD_TRY(evd::frob_norm_dev(n, n, AX, n, 0.0, X, ldX, w, part, sums + 0, stream));
  EVD_TRY(evd::frob_norm_dev(n, n, A, lda, 0.0, nullptr, 0, nullptr, part, sums + 1, stream));
  EVD_TRY(evd::dgemm('t', 'n', n, n, n, 1.0, X, ldX, X, ldX, 0.0, AX, n, stream));
  EVD_TRY(evd::frob_norm_dev(n, n, AX, n, 1.0, nullptr, 0, nullptr, part, sums + 2, stream));
  double h[3];
  EVD_CUDA_TRY(cudaMemcpyAsync(h, sums, 3 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  EVD_CUDA_TRY(cudaStreamSynchronize(stream));
  result[0] = sqrt(h[0]) / ((double)n * sqrt(h[1]));
  result[1] = sqrt(h[2]) / (double)n;
  return EVD_SUCCESS;
}
