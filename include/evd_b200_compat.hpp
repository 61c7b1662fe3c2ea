// evd_b200_compat.hpp — drop-in C++ shims with the reference's exact
// signatures (hansheng1001/EVD4SC2025 api/inc/*.h), forwarding to the C ABI
// of evd_b200.h.  Existing call sites compile unchanged; the cuBLAS/cuSOLVER
// handles are accepted and ignored (this library uses neither), and the
// legacy default stream is used, as in the reference.  Errors are reported
// the reference's way (message + exit), see EVD_COMPAT_CHECK.
#pragma once

#include <cuda_fp16.h>

#include <cstdio>
#include <cstdlib>

#include "evd_b200.h"

// The reference passes cuBLAS/cuSOLVER handles; declare the same opaque types
// so that this header works with or without the vendor headers included.
struct cublasContext;
typedef struct cublasContext* cublasHandle_t;
struct cusolverDnContext;
typedef struct cusolverDnContext* cusolverDnHandle_t;

#ifndef EVD_COMPAT_CHECK
#define EVD_COMPAT_CHECK(call)                                                         \
  do {                                                                                 \
    int evd_rc_ = (call);                                                              \
    if (evd_rc_ != EVD_SUCCESS) {                                                      \
      std::fprintf(stderr, "evd_b200: %s failed: %s\n", #call, evd_status_string(evd_rc_)); \
      std::exit(1);                                                                    \
    }                                                                                  \
  } while (0)
#endif

// api/inc/zy_zy_sy2sb.h:5-24.  `work` must hold evd_sy2sb_work_size(M, b, nb)
// doubles (the reference driver allocates (M+nb)*(N+nb), which is larger);
// `info` is unused (the reference never reads it either).
template <typename T>
void my_ZY_ZY_SBR_Vector(cusolverDnHandle_t, cublasHandle_t, long M, long N, long b, long nb,
                         T* dOriA, long ldOriA, T* dA, long ldA, T* dW, long ldW, T* dY, long ldY,
                         T* dZ, long ldZ, T* dR, long ldR, T* work, int* info);

template <>
inline void my_ZY_ZY_SBR_Vector<double>(cusolverDnHandle_t, cublasHandle_t, long M, long N,
                                        long b, long nb, double* dOriA, long ldOriA, double* dA,
                                        long ldA, double* dW, long ldW, double* dY, long ldY,
                                        double* dZ, long ldZ, double* dR, long ldR, double* work,
                                        int* /*info*/) {
  if (M % nb != 0) {  // same message as the reference (api/zy_zy_sy2sb.cu:51-55)
    std::printf("M must be diviable by nb!\n");
    return;
  }
  EVD_COMPAT_CHECK(evd_sy2sb(M, N, b, nb, dOriA, ldOriA, dA, ldA, dW, ldW, dY, ldY, dZ, ldZ, dR,
                             ldR, work, (M + nb) * (N + nb), nullptr));
}

// api/inc/PanelQR.h:7-18 (double).  `work` as in the reference's driver.
template <typename T>
void panelQR(cusolverDnHandle_t, cublasHandle_t, long m, long n, T* A, long lda, T* W, long ldw,
             T* R, long ldr, T* work, int* info);

template <>
inline void panelQR<double>(cusolverDnHandle_t, cublasHandle_t, long m, long n, double* A,
                            long lda, double* W, long ldw, double* R, long ldr, double* work,
                            int* /*info*/) {
  EVD_COMPAT_CHECK(evd_panel_qr(m, n, A, lda, W, ldw, R, ldr, work,
                                evd_panel_qr_work_size(m, n), nullptr));
}

// panelQR<float> / panelQR<half> (api/panelQR.cu:262-701), n == 32.  `work`
// must hold evd_panel_qr_lp_work_size(m, n) bytes.
template <>
inline void panelQR<float>(cusolverDnHandle_t, cublasHandle_t, long m, long n, float* A,
                           long lda, float* W, long ldw, float* R, long ldr, float* work,
                           int* /*info*/) {
  EVD_COMPAT_CHECK(evd_panel_qr_s(m, n, A, lda, W, ldw, R, ldr, work,
                                  evd_panel_qr_lp_work_size(m, n), nullptr));
}

template <>
inline void panelQR<__half>(cusolverDnHandle_t, cublasHandle_t, long m, long n, __half* A,
                            long lda, __half* W, long ldw, __half* R, long ldr, __half* work,
                            int* /*info*/) {
  EVD_COMPAT_CHECK(evd_panel_qr_h(m, n, A, lda, W, ldw, R, ldr, work,
                                  evd_panel_qr_lp_work_size(m, n), nullptr));
}

// api/inc/TallShinnyQR.h:9-17 (M = 128, N = 32 is the only instantiation used).
template <typename T, long M, long N>
void hou_tsqr_panel(cublasHandle_t, long m, long n, T* A, long lda, T* R, long ldr, T* work) {
  static_assert(M == 128 && N == 32, "evd_b200 implements the 128 x 32 TSQR");
  if constexpr (sizeof(T) == 8) {
    EVD_COMPAT_CHECK(evd_tsqr(m, n, A, lda, R, ldr, work, evd_panel_qr_work_size(m, n), nullptr));
  } else if constexpr (sizeof(T) == 4) {
    EVD_COMPAT_CHECK(evd_tsqr_s(m, n, A, lda, R, ldr, work, evd_panel_qr_lp_work_size(m, n),
                                nullptr));
  } else {
    EVD_COMPAT_CHECK(evd_tsqr_h(m, n, A, lda, R, ldr, work, evd_panel_qr_lp_work_size(m, n),
                                nullptr));
  }
}

// api/inc/tc_ozimmu_syr2k.h:6-18: C(lower) = alpha (A B^T + B A^T) + beta C,
// upper triangle mirrored (the reference mirrors right after the call).
template <typename T>
void tc_ozimmu_syr2k(cublasHandle_t, long n, long k, T alpha, T* A, long lda, T* B, long ldb,
                     T beta, T* C, long ldc, long nb);

template <>
inline void tc_ozimmu_syr2k<double>(cublasHandle_t, long n, long k, double alpha, double* A,
                                    long lda, double* B, long ldb, double beta, double* C,
                                    long ldc, long nb) {
  EVD_COMPAT_CHECK(evd_syr2k_lower_mirror(n, k, alpha, A, lda, B, ldb, beta, C, ldc, nb, nullptr));
}

template <>
inline void tc_ozimmu_syr2k<float>(cublasHandle_t, long n, long k, float alpha, float* A,
                                   long lda, float* B, long ldb, float beta, float* C, long ldc,
                                   long nb) {
  EVD_COMPAT_CHECK(evd_syr2k_lower_s(n, k, alpha, A, lda, B, ldb, beta, C, ldc, nb, nullptr));
}

template <>
inline void tc_ozimmu_syr2k<__half>(cublasHandle_t, long n, long k, __half alpha, __half* A,
                                    long lda, __half* B, long ldb, __half beta, __half* C,
                                    long ldc, long nb) {
  EVD_COMPAT_CHECK(evd_syr2k_lower_h(n, k, __half2float(alpha), A, lda, B, ldb,
                                     __half2float(beta), C, ldc, nb, nullptr));
}

// api/inc/tc_syr2k.h:6-18: FP16 products, FP32 accumulation; hwork unused.
inline void tc_syr2k(cublasHandle_t, long n, long k, float alpha, float* A, long lda, float* B,
                     long ldb, float beta, float* C, long ldc, __half* hwork, long nb) {
  EVD_COMPAT_CHECK(evd_tc_syr2k(n, k, alpha, A, lda, B, ldb, beta, C, ldc, hwork, nb, nullptr));
}

// api/inc/BC_backTrans.h:3 — same name, same arguments, same return value.
inline int my_BC_back_trans_v8_10_noBandU(double* Q, long ldQ, double* U, long ldU, long n, int b,
                                          cudaStream_t stream = NULL) {
  return evd_bc_back(Q, ldQ, U, ldU, n, b, stream) == EVD_SUCCESS ? 0 : -1;
}

// api/inc/computerWYFromSlide.h:4
inline void computerWYFromSlide(cublasHandle_t, long M, long N, long slideWidth, double* dW,
                                long ldW, double* dY, long ldY, double* work) {
  EVD_COMPAT_CHECK(evd_wy_from_slide(M, N, slideWidth, dW, ldW, dY, ldY, work, nullptr));
}

// api/inc/computerQFromWY.h:4
inline void computerQFromWY(cublasHandle_t, long M, long N, double* dQ, long ldQ, double* dW,
                            long ldW, double* dY, long ldY) {
  EVD_COMPAT_CHECK(evd_q_from_wy(M, N, dQ, ldQ, dW, ldW, dY, ldY, nullptr));
}

// util/inc/checkMetric.h:3 — prints the metric like the reference.
inline void checkOrthogonality(cublasHandle_t, long M, long N, double* dA, long ldA, double* dB,
                               long ldB, double* work) {
  double r = 0.0;
  EVD_COMPAT_CHECK(evd_check_orthogonality(M, N, dA, ldA, dB, ldB, work, &r, nullptr));
  std::printf("The Orthogonality metrix is %g\n", r);
}
