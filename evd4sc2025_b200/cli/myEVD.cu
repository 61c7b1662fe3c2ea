// myEVD <n> <b> <nb> [--dist uniform|gauss] [--seed S] [--reps R] [--no-check]
//       [--input A.bin] [--save-input A.bin] [--output eig.bin]
//       [--values] [--refine K]
//
// Command-line driver with the reference's surface (src/EVD/myEVD.cu:251-266:
// three positional arguments; a wrong count prints the usage and returns 0).
// Generates a symmetric test matrix on the device (default: U(0,1] lower
// triangle mirrored to the upper one, the reference's input shape; --dist gauss
// gives (G + G^T)/2), runs the B200 eigensolver through the C ABI, and prints
// the stage times, the FP64 rate of each stage with its own flop count, and
// the orthogonality / residual of the result.  --input reads A (n x n) from
// record 0 of a binary matrix file instead; --save-input writes the generated
// A; --output writes the eigenpairs (w, X) as a binary eigenpair file.
// --values times the eigenvalues-only solve instead; --refine K runs K
// Ogita-Aishima refinement iterations on the computed eigenpairs and prints
// their time and the metrics after them.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "evd_b200.h"

#define CK(x)                                                                             \
  do {                                                                                    \
    cudaError_t e_ = (x);                                                                 \
    if (e_ != cudaSuccess) {                                                              \
      fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return 1;                                                                           \
    }                                                                                     \
  } while (0)

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double u01(uint64_t h) {  // (0, 1]
  return ((double)(h >> 11) + 1.0) * (1.0 / 9007199254740992.0);
}

// symmetric matrix from a counter-based generator over the lower triangle
__global__ void gen_sym(long n, double* A, long lda, uint64_t seed, int gauss) {
  long j = blockIdx.y;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    long r = i >= j ? i : j, c = i >= j ? j : i;  // lower-triangle index
    uint64_t key = seed * 0x100000001B3ull + (uint64_t)r * (uint64_t)n + (uint64_t)c;
    double v;
    if (gauss) {
      double u1 = u01(mix64(2 * key)), u2 = u01(mix64(2 * key + 1));
      v = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
      if (r == c) v *= 1.4142135623730951;  // (G+G^T)/2 has var 1/2 off-diagonal, 1 on it
      else v *= 1.0;
      v *= 0.7071067811865476;
    } else {
      v = u01(mix64(key));
    }
    A[i + j * lda] = v;
  }
}

int main(int argc, char** argv) {
  if (argc < 4) {
    printf("Usage(b = nb in ZY): AppName <n> <b> <nb>\n");
    return 0;
  }
  long n = atol(argv[1]), b = atol(argv[2]), nb = atol(argv[3]);
  int gauss = 0, reps = 1, check = 1;
  uint64_t seed = 3000;
  const char *in_path = nullptr, *save_path = nullptr, *out_path = nullptr;
  int values_only = 0, refine = 0;
  for (int i = 4; i < argc; ++i) {
    if (!strcmp(argv[i], "--dist") && i + 1 < argc) gauss = !strcmp(argv[++i], "gauss");
    else if (!strcmp(argv[i], "--seed") && i + 1 < argc) seed = strtoull(argv[++i], 0, 10);
    else if (!strcmp(argv[i], "--reps") && i + 1 < argc) reps = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--no-check")) check = 0;
    else if (!strcmp(argv[i], "--input") && i + 1 < argc) in_path = argv[++i];
    else if (!strcmp(argv[i], "--save-input") && i + 1 < argc) save_path = argv[++i];
    else if (!strcmp(argv[i], "--output") && i + 1 < argc) out_path = argv[++i];
    else if (!strcmp(argv[i], "--values")) values_only = 1;
    else if (!strcmp(argv[i], "--refine") && i + 1 < argc) refine = atoi(argv[++i]);
  }
  printf("%s\nn=%ld, b=%ld, nb=%ld\n", evd_version(), n, b, nb);
  long wbytes = evd_syevd_work_size(n, b, nb);
  if (wbytes <= 0) {
    printf("unsupported sizes: need n >= 1, b == 32, nb = 32 * 2^k\n");
    return 1;
  }
  double *A, *w, *X;
  void* work;
  CK(cudaMalloc(&A, sizeof(double) * n * n));
  CK(cudaMalloc(&X, sizeof(double) * n * n));
  CK(cudaMalloc(&w, sizeof(double) * n));
  CK(cudaMalloc(&work, wbytes));
  if (in_path) {
    long r = 0, c = 0;
    int rc = evd_matrix_bin_shape(in_path, 0, &r, &c);
    if (rc == EVD_SUCCESS && (r != n || c != n)) rc = EVD_ERR_INVALID_ARG;
    if (rc == EVD_SUCCESS) rc = evd_read_matrix_bin(in_path, 0, n, n, A, n);
    if (rc != EVD_SUCCESS) {
      printf("cannot read a %ld x %ld matrix from %s: %s\n", n, n, in_path, evd_status_string(rc));
      return 1;
    }
    printf("A read from %s\n", in_path);
  } else {
    gen_sym<<<dim3((unsigned)((n + 255) / 256), (unsigned)n), 256>>>(n, A, n, seed, gauss);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    if (save_path) {
      int rc = evd_write_matrix_bin(save_path, 0, n, n, A, n);
      if (rc != EVD_SUCCESS) {
        printf("cannot write %s: %s\n", save_path, evd_status_string(rc));
        return 1;
      }
    }
  }
  double t[6];
  if (values_only) {
    for (int r = 0; r < reps; ++r) {
      int rc = evd_syevd_values(n, b, nb, A, n, w, work, wbytes, 1, 0);
      if (rc != EVD_SUCCESS) {
        printf("evd_syevd_values failed: %s\n", evd_status_string(rc));
        return 2;
      }
      evd_syevd_last_timings(t);
      printf("eigenvalues only %ldx%ld: sy2sb %.3f ms, chasing %.3f ms, multisection %.3f ms, "
             "total %.3f ms\n", n, n, t[0], t[1], t[2], t[5]);
    }
    cudaFree(A);
    cudaFree(X);
    cudaFree(w);
    cudaFree(work);
    return 0;
  }
  for (int r = 0; r < reps; ++r) {
    int rc = evd_syevd(n, b, nb, A, n, w, X, n, work, wbytes, 1, 0);
    if (rc != EVD_SUCCESS) {
      printf("evd_syevd failed: %s\n", evd_status_string(rc));
      return 2;
    }
    evd_syevd_last_timings(t);
    const double n3 = (double)n * n * n;
    printf("sy2sb %ldx%ld takes %.3f ms, tflops is %.3f\n", n, n, t[0], 4.0 / 3.0 * n3 / (t[0] * 1e9));
    printf("Bugle chasing %ldx%ld takes %.3f ms\n", n, n, t[1]);
    printf("sy2tr %ldx%ld takes %.3f ms, tflops is %.3f\n", n, n, t[0] + t[1],
           4.0 / 3.0 * n3 / ((t[0] + t[1]) * 1e9));
    printf("DC (device) %ldx%ld takes %.3f ms\n", n, n, t[2]);
    printf("BC back %ldx%ld takes %.3f ms, tflops is %.3f\n", n, n, t[3], 2.0 * n3 / (t[3] * 1e9));
    printf("SBR back %ldx%ld takes %.3f ms, tflops is %.3f\n", n, n, t[4], 2.0 * n3 / (t[4] * 1e9));
    printf("total EVD %ldx%ld takes %.3f ms, FP64-equivalent tflops is %.3f\n", n, n, t[5],
           16.0 / 3.0 * n3 / (t[5] * 1e9));
  }
  if (refine > 0) {
    long rn = evd_refine_syev_work_size(n);
    double* rw = nullptr;
    if (rn <= 0) {
      printf("refinement supports n <= 65535\n");
      return 1;
    }
    CK(cudaMalloc(&rw, sizeof(double) * rn));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, 0));
    int rc = evd_refine_syev(n, A, n, w, X, n, refine, rw, rn, 0);
    CK(cudaEventRecord(e1, 0));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (rc != EVD_SUCCESS) {
      printf("evd_refine_syev failed: %s\n", evd_status_string(rc));
      return 2;
    }
    printf("refinement %d iteration(s) %ldx%ld takes %.3f ms (%.3f TFLOP/s FP64)\n", refine, n, n,
           ms, 8.0 * refine * (double)n * n * n / (ms * 1e9));
    cudaFree(rw);
  }
  if (out_path) {
    int rc = evd_write_eigenpairs_bin(out_path, n, w, X, n);
    if (rc != EVD_SUCCESS) {
      printf("cannot write %s: %s\n", out_path, evd_status_string(rc));
      return 1;
    }
    printf("eigenpairs written to %s\n", out_path);
  }
  if (check) {
    double* cw;
    CK(cudaMalloc(&cw, sizeof(double) * (n * n + 1024)));
    double res[2];
    int rc = evd_check_eig(n, A, n, w, X, n, cw, res, 0);
    if (rc == EVD_SUCCESS) {
      printf("The Orthogonality metrix is %.3e\n", res[1]);
      printf("Residual ||AX - XW||_F / (n ||A||_F) is %.3e\n", res[0]);
    }
    cudaFree(cw);
  }
  cudaFree(A);
  cudaFree(X);
  cudaFree(w);
  cudaFree(work);
  return 0;
}
