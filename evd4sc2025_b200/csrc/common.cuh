// Shared device/host helpers for the B200 two-stage symmetric eigensolver.
//
// All matrices are FP64, column-major, with 64-bit leading dimensions, as in the
// reference (inc/myBase.h, api/inc/*.h).  Unlike the reference, which prints
// and exit()s on errors (inc/myBase.h:4-30), every entry point here returns an
// int status (EVD_* codes in include/evd_b200.h) and never terminates the host.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <stdio.h>

#include "../../include/evd_b200.h"

#define EVD_CUDA_TRY(call)                                                        \
  do {                                                                            \
    cudaError_t evd_err__ = (call);                                               \
    if (evd_err__ != cudaSuccess) {                                               \
      fprintf(stderr, "evd_b200: CUDA error %s at %s:%d: %s\n",                  \
              cudaGetErrorName(evd_err__), __FILE__, __LINE__,                    \
              cudaGetErrorString(evd_err__));                                     \
      return EVD_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

// Every kernel launch site ends with EVD_LAUNCHED(): counts the launch (see
// evd_launch_count) and surfaces launch errors.
#define EVD_LAUNCHED()                          \
  do {                                          \
    ::evd::note_launch();                       \
    EVD_CUDA_TRY(cudaGetLastError());           \
  } while (0)

#define EVD_TRY(call)                          \
  do {                                         \
    int evd_st__ = (call);                     \
    if (evd_st__ != EVD_SUCCESS) return evd_st__; \
  } while (0)

namespace evd {

constexpr int kWarp = 32;

// Device-side error word written by kernels that wait on other CTAs.  A wait
// that runs out of its iteration budget records where it gave up and returns,
// so no kernel can spin forever on a shared GPU.
enum DeviceError : int {
  kDevOk = 0,
  kDevTimeoutChase = 1,
  kDevTimeoutTree = 2,
  kDevBadShape = 3,
  kDevNoConvergence = 4,
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, m));
  return v;
}

// Acquire/release helpers for flag-based progress between CTAs (gpu scope).
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

inline int ceil_div_i(long a, long b) { return (int)((a + b - 1) / b); }

// SM count of the current device (cached per device; thread-safe).
int device_sm_count();
void note_launch();

// Raises `func`'s dynamic shared-memory limit to `bytes` once per (device,
// kernel); thread-safe, so host threads driving several devices or streams
// (the batched solver) may launch the same kernel concurrently.
int smem_attr_once(const void* func, int bytes);

// Reads a device error word written by a kernel (synchronises `st`) and maps
// it to an EVD_* status.
int read_device_error(const int* err_word, cudaStream_t st);

}  // namespace evd
