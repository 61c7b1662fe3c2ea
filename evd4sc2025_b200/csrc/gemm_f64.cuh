// Internal interface of the FP64 DMMA GEMM (gemm_f64.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace evd {

enum GemmMode : int { kGemm = 0, kSyr2kLow = 1 };

struct GemmArgs {
  int m, n, k;
  double alpha, beta;
  const double* A;
  long lda, sA;
  const double* B;
  long ldb, sB;
  double* C;
  long ldc, sC;
  // second operand pair (SYR2K mode): used for k >= k1
  const double* A2;
  long lda2;
  const double* B2;
  long ldb2;
  int k1;
  // second A along M (transposed A only): rows m >= m1 of op(A) come from Am2
  const double* Am2;
  long ldam2;
  int m1;
  int mode;
  int splitk;
  double* ws;  // split-K partials: batch * splitk * m * n doubles
  int tiles_m, tiles_n;
  int vecA, vecB;
};

// Doubles of workspace needed for a split-K GEMM with `splits` partials.
inline size_t gemm_splitk_ws_doubles(long m, long n, int splits, long batch = 1) {
  return (splits > 1) ? (size_t)batch * splits * (size_t)m * n : 0;
}

// Split count the library would choose for an (m x n x k) product.
int choose_splitk(long m, long n, long k, long batch);

// C = alpha*op(A)*op(B) + beta*C.  splitk: 0 = automatic (bounded by ws),
// 1 = none.  ws/ws_doubles: caller scratch for split-K partial sums; when it is
// too small the split count is reduced until it fits (1 needs none).
int dgemm(char transa, char transb, long m, long n, long k, double alpha, const double* A,
          long lda, const double* B, long ldb, double beta, double* C, long ldc,
          cudaStream_t st, int splitk = 1, double* ws = nullptr, size_t ws_doubles = 0);

int dgemm_batched(char transa, char transb, long m, long n, long k, double alpha,
                  const double* A, long lda, long sA, const double* B, long ldb, long sB,
                  double beta, double* C, long ldc, long sC, long batch, cudaStream_t st);

// C = alpha*(A1 B1^T + A2 B2^T) + beta*C, K = k1 + k2 (one kernel, operand pair
// switched at k1).
int dgemm_nt_pair(long m, long n, long k1, long k2, double alpha, const double* A1, long lda1,
                  const double* B1, long ldb1, const double* A2, long lda2, const double* B2,
                  long ldb2, double beta, double* C, long ldc, cudaStream_t st, int splitk = 1,
                  double* ws = nullptr, size_t ws_doubles = 0);

// General two-operand form used by the ZY update:
//   op(A) = [A ; Am2] stacked along M (ta == 't' only, split at m1), and/or
//   op(A) = [A , A2] along K (ta == 'n' only, split at k1; B spans all of K,
//   or, when tb == 't', B is [B , B2] along K as well).
struct GemmPair {
  char ta, tb;
  long m, n, k;
  double alpha, beta;
  const double* A;
  long lda;
  const double* B;
  long ldb;
  double* C;
  long ldc;
  const double* A2 = nullptr;
  long lda2 = 0;
  long k1 = 0;
  const double* B2 = nullptr;
  long ldb2 = 0;
  const double* Am2 = nullptr;
  long ldam2 = 0;
  long m1 = 0;
};
int dgemm_pair(const GemmPair& g, cudaStream_t st, int splitk = 0, double* ws = nullptr,
               size_t ws_doubles = 0);

// C(lower) = alpha*(A B^T + B A^T) + beta*C(lower); upper = mirror of lower.
int syr2k_lower_mirror(long n, long k, double alpha, const double* A, long lda,
                       const double* B, long ldb, double beta, double* C, long ldc,
                       cudaStream_t st);

}  // namespace evd
