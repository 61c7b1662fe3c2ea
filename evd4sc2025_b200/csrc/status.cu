// Status strings and version of the C ABI.
#include "common.cuh"

extern "C" const char* evd_status_string(int status) {
  switch (status) {
    case EVD_SUCCESS: return "success";
    case EVD_ERR_INVALID_ARG: return "invalid argument";
    case EVD_ERR_CUDA: return "CUDA runtime error";
    case EVD_ERR_TIMEOUT: return "bounded device wait timed out";
    case EVD_ERR_NO_CONVERGENCE: return "iteration did not converge";
    case EVD_ERR_WORKSPACE: return "workspace too small";
    case EVD_ERR_IO: return "file I/O error";
    case EVD_ERR_HOST: return "host resource failure (threads or host memory)";
    default: return "unknown status";
  }
}

extern "C" const char* evd_version(void) { return "evd_b200 0.1 sm_100a"; }

// ---- launch accounting and the FP64 peak probe ----------------------------
#include <atomic>
#include <mutex>
#include <set>
#include <utility>

namespace evd {
static std::atomic<long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int device_sm_count() {
  constexpr int kMaxDev = 64;
  static std::atomic<int> sms[kMaxDev] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return 148;
  int v = sms[dev].load(std::memory_order_relaxed);
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    sms[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

int smem_attr_once(const void* func, int bytes) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  EVD_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({dev, func})) return EVD_SUCCESS;
  EVD_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.insert({dev, func});
  return EVD_SUCCESS;
}

namespace {
// Each warp keeps 8 independent 8x8x4 DMMA accumulators busy; 2 CTAs per SM.
__global__ void fp64_peak_kernel(double* out, int iters) {
  double c[8][2];
#pragma unroll
  for (int i = 0; i < 8; ++i) c[i][0] = c[i][1] = 0.0;
  const double a = threadIdx.x * 1e-3, b = 1.0 + threadIdx.x * 1e-4;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(c[i][0]), "+d"(c[i][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += c[i][0] + c[i][1];
  if (s == 1.2345678e300) out[threadIdx.x] = s;  // keeps the MMAs live
}
}  // namespace
}  // namespace evd

extern "C" long evd_launch_count(void) { return evd::g_launches.load(); }

extern "C" int evd_fp64_peak_probe(double* tflops, cudaStream_t stream) {
  if (!tflops) return EVD_ERR_INVALID_ARG;
  const int sms = evd::device_sm_count();
  const int blocks = 2 * sms, threads = 256, iters = 20000;
  cudaEvent_t e0, e1;
  EVD_CUDA_TRY(cudaEventCreate(&e0));
  EVD_CUDA_TRY(cudaEventCreate(&e1));
  evd::fp64_peak_kernel<<<blocks, threads, 0, stream>>>(nullptr, 100);  // warm-up
  EVD_LAUNCHED();
  EVD_CUDA_TRY(cudaEventRecord(e0, stream));
  evd::fp64_peak_kernel<<<blocks, threads, 0, stream>>>(nullptr, iters);
  EVD_LAUNCHED();
  EVD_CUDA_TRY(cudaEventRecord(e1, stream));
  EVD_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  EVD_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double flops = 2.0 * 8 * 8 * 4 * 8 * (threads / 32) * (double)blocks * iters;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return EVD_SUCCESS;
}
