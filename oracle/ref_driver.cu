// Input-injection driver for the reference's own GPU build (test oracle and
// GPU baseline; built by oracle/Makefile into oracle/_ref/, never shipped).
//
// Runs the reference pipeline of src/EVD/myEVD.cu:251-706 through the
// reference's own entry points on a given matrix:
//   my_ZY_ZY_SBR_Vector -> copyMatrixL2U -> band pack -> cooperative
//   chasing_kernel_one_timeV10<32> -> d, e to host -> host LAPACKE_dstedc
//   overlapped with my_SBRBack_BCBack on a second thread -> final Dgemm.
// Differences from the stock main: the input comes from a file (or the
// reference's own cuRAND generator), every buffer is zeroed first (the stock
// main reads uninitialised com[] and padding rows), and stage times are
// printed as one JSON line.  Optional outputs: eigenvalues and eigenvectors.
//
// usage: ref_driver n b nb input(.bin|-) out_prefix(|-) [reps] [outputs]
//   outputs "all" (default): w, X, d, e files; "w": eigenvalues only, plus the
//   result's residual ||AX - X diag(w)||_F / ||A||_F and orthogonality
//   ||X^T X - I||_F (cuBLAS, after the timed solves) as one JSON line.
#include <cooperative_groups.h>
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <mkl_lapacke.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "bugle_chasingV10.h"
#include "fileOpTool.h"
#include "kernelOther.h"
#include "zy_zy_sy2sb.h"

// defined in the reference's src/EVD/myEVD.cu (compiled with main renamed)
void my_SBRBack_BCBack(cublasHandle_t cublas_handle, double* dQ, long ldQ, double* dU, long ldU,
                       double* dW, long ldW, double* dY, long ldY, double* dwork, long n, long b,
                       cudaStream_t stream);

#define CK(x)                                                                          \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) {                                                           \
      fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      exit(2);                                                                         \
    }                                                                                  \
  } while (0)

__global__ void pack_band(int n, int b, const double* A, long lda, double* sub, int ldsub) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (i >= 2 * b || j >= n) return;
  sub[i + (long)j * ldsub] = (i <= b && j + i < n) ? A[(j + i) + (long)j * lda] : 0.0;
}
__global__ void unpack_tridiag(int n, const double* sub, int ldsub, double* d, double* e) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  d[j] = sub[(long)j * ldsub];
  if (j < n - 1) e[j] = sub[1 + (long)j * ldsub];
}

static float ev_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

int main(int argc, char** argv) {
  if (argc < 6) {
    printf("usage: %s n b nb input(.bin|-) out_prefix(|-) [reps]\n", argv[0]);
    return 0;
  }
  long n = atol(argv[1]), b = atol(argv[2]), nb = atol(argv[3]);
  std::string in = argv[4], outp = argv[5];
  int reps = argc > 6 ? atoi(argv[6]) : 1;
  const std::string outputs = argc > 7 ? argv[7] : "all";
  long m = n;
  cusolverDnHandle_t cusolver_handle;
  cublasHandle_t cublas_handle;
  cusolverDnCreate(&cusolver_handle);
  cublasCreate(&cublas_handle);

  double *dT, *dA, *dwork, *dR, *dW, *dY, *dZ, *dOriA, *dSub, *dU, *dQ, *mD, *mE;
  int *info, *com;
  CK(cudaMalloc(&dT, sizeof(double) * m * n));
  CK(cudaMalloc(&dA, sizeof(double) * m * n));
  CK(cudaMalloc(&dwork, sizeof(double) * (m + nb) * (n + nb)));
  CK(cudaMalloc(&dW, sizeof(double) * m * n));
  CK(cudaMalloc(&dY, sizeof(double) * m * n));
  CK(cudaMalloc(&dR, sizeof(double) * m * nb));
  CK(cudaMalloc(&dZ, sizeof(double) * m * nb));
  CK(cudaMalloc(&dOriA, sizeof(double) * m * n));
  CK(cudaMalloc(&dSub, sizeof(double) * 2 * b * n));
  CK(cudaMalloc(&dU, sizeof(double) * (m + nb) * n));
  CK(cudaMalloc(&dQ, sizeof(double) * (m + nb) * n));
  CK(cudaMalloc(&mD, sizeof(double) * n));
  CK(cudaMalloc(&mE, sizeof(double) * n));
  CK(cudaMalloc(&info, sizeof(int)));
  CK(cudaMalloc(&com, sizeof(int) * n));

  if (in == "-") {
    generateUniformMatrix(dT, m, n);  // the reference's own input: cuRAND seed 3000
    dim3 g((m + 31) / 32, (n + 31) / 32), bl(32, 32);
    launchKernel_CpyMatrixL2U(g, bl, n, dT, n);
  } else {
    std::vector<double> h(m * n);
    FILE* f = fopen(in.c_str(), "rb");
    if (!f || fread(h.data(), sizeof(double), m * n, f) != (size_t)(m * n)) {
      fprintf(stderr, "cannot read %s\n", in.c_str());
      return 3;
    }
    fclose(f);
    CK(cudaMemcpy(dT, h.data(), sizeof(double) * m * n, cudaMemcpyHostToDevice));
  }
  std::vector<double> hS(n), hE(n), Z((size_t)n * n);
  cudaEvent_t e0, e1, e2, e3, e4;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3);
  cudaEventCreate(&e4);
  int dev = 0, nbps = 0, sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbps, chasing_kernel_one_timeV10<32>, 1024, 0);
  int blockNum = nbps * sms;

  for (int rep = 0; rep < reps; ++rep) {
    // zero every buffer (the stock driver leaves com[], dU/dQ padding uninitialised)
    CK(cudaMemset(dwork, 0, sizeof(double) * (m + nb) * (n + nb)));
    CK(cudaMemset(dW, 0, sizeof(double) * m * n));
    CK(cudaMemset(dY, 0, sizeof(double) * m * n));
    CK(cudaMemset(dR, 0, sizeof(double) * m * nb));
    CK(cudaMemset(dZ, 0, sizeof(double) * m * nb));
    CK(cudaMemset(dU, 0, sizeof(double) * (m + nb) * n));
    CK(cudaMemset(dQ, 0, sizeof(double) * (m + nb) * n));
    CK(cudaMemset(com, 0, sizeof(int) * n));
    int zero = 0;
    CK(cudaMemcpyToSymbol(g_overFlag, &zero, sizeof(int)));
    CK(cudaMemcpy(dA, dT, sizeof(double) * m * n, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(dOriA, dT, sizeof(double) * m * n, cudaMemcpyDeviceToDevice));
    CK(cudaDeviceSynchronize());
    auto w0 = std::chrono::high_resolution_clock::now();
    cudaEventRecord(e0);
    my_ZY_ZY_SBR_Vector(cusolver_handle, cublas_handle, m, n, b, nb, dOriA, m, dA, m, dW, m, dY,
                        m, dZ, m, dR, m, dwork, info);
    {
      dim3 g((m + 31) / 32, (n + 31) / 32), bl(32, 32);
      launchKernel_CpyMatrixL2U(g, bl, m, dA, m);
    }
    cudaEventRecord(e1);
    {
      int ldSub = 2 * b;
      pack_band<<<dim3((2 * b + 63) / 64, n), 64>>>(n, b, dA, m, dSub, ldSub);
      long ldU = m + nb;
      int ni = (int)n, bi = (int)b;
      void* args[] = {&ni, &bi, &dSub, &ldSub, &dU, &ldU, &blockNum, &com};
      CK(cudaLaunchCooperativeKernel((void*)chasing_kernel_one_timeV10<32>, dim3(blockNum),
                                     dim3(32, 32), args));
      unpack_tridiag<<<(n + 255) / 256, 256>>>(n, dSub, ldSub, mD, mE);
    }
    cudaEventRecord(e2);
    CK(cudaMemcpy(hS.data(), mD, sizeof(double) * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hE.data(), mE, sizeof(double) * (n - 1), cudaMemcpyDeviceToHost));
    {
      dim3 g((m + 31) / 32, (n + 31) / 32), bl(32, 32);
      long ldQ = m + nb;
      launchKernel_ClearMatrix(g, bl, m, n, dQ, ldQ);
      dim3 gs((n + 31) / 32), bs(32);
      launchKernel_setMetrixTrValue(gs, bs, n, n, dQ, ldQ, 1.0);
    }
    CK(cudaDeviceSynchronize());
    auto b0 = std::chrono::high_resolution_clock::now();
    double dc_ms = 0.0, back_ms = 0.0;
    std::thread th([&] {
      auto t0 = std::chrono::high_resolution_clock::now();
      my_SBRBack_BCBack(cublas_handle, dQ, m + nb, dU, m + nb, dW, m, dY, m, dwork, n, b,
                        (cudaStream_t)0);
      cudaDeviceSynchronize();
      back_ms = std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();
    });
    {
      auto t0 = std::chrono::high_resolution_clock::now();
      lapack_int linfo = LAPACKE_dstedc(LAPACK_COL_MAJOR, 'I', (lapack_int)n, hS.data(), hE.data(),
                                        Z.data(), (lapack_int)n);
      dc_ms = std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();
      if (linfo != 0) fprintf(stderr, "dstedc info %d\n", (int)linfo);
    }
    th.join();
    auto b1 = std::chrono::high_resolution_clock::now();
    double overlap_ms = std::chrono::duration<double, std::milli>(b1 - b0).count();
    cudaEventRecord(e3);
    CK(cudaMemcpy(dwork, Z.data(), sizeof(double) * n * n, cudaMemcpyHostToDevice));
    double one = 1.0, zz = 0.0;
    cublasDgemm(cublas_handle, CUBLAS_OP_T, CUBLAS_OP_N, n, n, n, &one, dQ, m + nb, dwork, n, &zz,
                dY, m);
    cudaEventRecord(e4);
    CK(cudaDeviceSynchronize());
    auto w1 = std::chrono::high_resolution_clock::now();
    double total_ms = std::chrono::duration<double, std::milli>(w1 - w0).count();
    printf("{\"n\": %ld, \"b\": %ld, \"nb\": %ld, \"rep\": %d, \"sy2sb_ms\": %.3f, \"chase_ms\": %.3f, "
           "\"dstedc_host_ms\": %.3f, \"back_ms\": %.3f, \"dc_back_overlap_ms\": %.3f, "
           "\"final_gemm_ms\": %.3f, \"total_ms\": %.3f}\n",
           n, b, nb, rep, ev_ms(e0, e1), ev_ms(e1, e2), dc_ms, back_ms, overlap_ms, ev_ms(e3, e4),
           total_ms);
    fflush(stdout);
  }
  if (outp != "-" && outputs == "w") {
    FILE* f = fopen((outp + "_w.bin").c_str(), "wb");
    fwrite(hS.data(), sizeof(double), n, f);
    fclose(f);
    // accuracy of the last result (dT = A, dY = X, hS = w): R = A X - X diag(w)
    double one = 1.0, zz = 0.0, mone = -1.0, ra = 0.0, rr = 0.0, ro = 0.0;
    CK(cudaMemcpy(dU, hS.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    cublasDgemm(cublas_handle, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, dT, m, dY, m, &zz, dwork, n);
    cublasDdgmm(cublas_handle, CUBLAS_SIDE_RIGHT, n, n, dY, m, dU, 1, dQ, n);
    cublasDgeam(cublas_handle, CUBLAS_OP_N, CUBLAS_OP_N, n, n, &one, dwork, n, &mone, dQ, n, dwork, n);
    cublasDnrm2(cublas_handle, n * n, dwork, 1, &rr);
    cublasDnrm2(cublas_handle, m * n, dT, 1, &ra);
    // X^T X - I
    cublasDgemm(cublas_handle, CUBLAS_OP_T, CUBLAS_OP_N, n, n, n, &one, dY, m, dY, m, &zz, dwork, n);
    {
      dim3 gs((n + 31) / 32), bs(32);
      launchKernel_ClearMatrix(dim3((n + 31) / 32, (n + 31) / 32), dim3(32, 32), n, n, dQ, n);
      launchKernel_setMetrixTrValue(gs, bs, n, n, dQ, n, 1.0);
    }
    cublasDgeam(cublas_handle, CUBLAS_OP_N, CUBLAS_OP_N, n, n, &one, dwork, n, &mone, dQ, n, dwork, n);
    cublasDnrm2(cublas_handle, n * n, dwork, 1, &ro);
    CK(cudaDeviceSynchronize());
    printf("{\"accuracy\": {\"resid_fro_rel\": %.6e, \"orth_fro\": %.6e, \"resid\": %.6e, "
           "\"orth\": %.6e}}\n", rr / ra, ro, rr / ra / n, ro / n);
  } else if (outp != "-") {
    std::vector<double> X((size_t)n * n);
    CK(cudaMemcpy2D(X.data(), sizeof(double) * n, dY, sizeof(double) * m, sizeof(double) * n, n,
                    cudaMemcpyDeviceToHost));
    FILE* f = fopen((outp + "_w.bin").c_str(), "wb");
    fwrite(hS.data(), sizeof(double), n, f);
    fclose(f);
    f = fopen((outp + "_X.bin").c_str(), "wb");
    fwrite(X.data(), sizeof(double), (size_t)n * n, f);
    fclose(f);
    // the tridiagonal the reference's chase produced (for the chase/stedc oracle)
    CK(cudaMemcpy(hS.data(), mD, sizeof(double) * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hE.data(), mE, sizeof(double) * (n - 1), cudaMemcpyDeviceToHost));
    f = fopen((outp + "_d.bin").c_str(), "wb");
    fwrite(hS.data(), sizeof(double), n, f);
    fclose(f);
    f = fopen((outp + "_e.bin").c_str(), "wb");
    fwrite(hE.data(), sizeof(double), n - 1, f);
    fclose(f);
  }
  return 0;
}
