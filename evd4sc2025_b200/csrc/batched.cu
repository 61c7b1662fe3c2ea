// Batched solves of many symmetric matrices of uneven orders.
//
// The reference solves one matrix per process (src/EVD/myEVD.cu:251-706).
// Here `nstreams` host threads each own a non-blocking CUDA stream and one
// slice of the caller's workspace (sized for the largest order of the batch);
// they take matrices largest first from a shared counter and run the full
// solver on their stream, so the latency-bound phases of one solve (panel
// factorisations, the chase, the divide and conquer's small merges) overlap
// the GEMM phases of others on the device.  The worker streams start after
// everything already enqueued on `stream` (an event), and `stream` waits for
// all of them at the end.  The block size of each solve is the largest
// 32 * 2^k (at most 1024) dividing 32 * ceil(n / 32) (at least 64): the same
// padded order the tuned table of the Python layer starts from.
#include <algorithm>
#include <atomic>
#include <numeric>
#include <thread>
#include <vector>

#include "common.cuh"

namespace evd {

int syevd(long n, long b, long nb, const double* A, long lda, double* w, double* X, long ldX,
          void* work, long lwork_bytes, int timed, cudaStream_t st);
size_t syevd_any_ws_bytes(long n, long b, long nb);

namespace {

long batch_nb(long n) {
  const long np = std::max<long>(64, (n + 31) / 32 * 32);
  long q = np / 32, nb = 32;
  while (nb * 2 <= 1024 && q % 2 == 0) {
    nb *= 2;
    q /= 2;
  }
  return nb;
}

size_t slice_bytes(long count, const long* n) {
  size_t mx = 0;
  for (long i = 0; i < count; ++i)
    mx = std::max(mx, syevd_any_ws_bytes(n[i], 32, batch_nb(n[i])));
  return (mx + 255) / 256 * 256;
}

}  // namespace
}  // namespace evd

extern "C" long evd_syevd_batched_work_size(long count, const long* n, int nstreams) {
  if (count < 0 || nstreams < 1 || nstreams > 64 || (count > 0 && !n)) return 0;
  for (long i = 0; i < count; ++i)
    if (n[i] < 1) return 0;
  if (count == 0) return 256;
  const int workers = (int)std::min<long>(nstreams, count);
  return (long)(evd::slice_bytes(count, n) * workers + 256);
}

static int syevd_batched_impl(long count, const long* n, const double* const* A,
                              const long* lda, double* const* w, double* const* X,
                              const long* ldX, int nstreams, void* work, long lwork_bytes,
                              cudaStream_t stream) {
  if (count < 0 || nstreams < 1 || nstreams > 64) return EVD_ERR_INVALID_ARG;
  if (count == 0) return EVD_SUCCESS;
  if (!n || !A || !lda || !w || !X || !ldX || !work) return EVD_ERR_INVALID_ARG;
  for (long i = 0; i < count; ++i)
    if (n[i] < 1 || !A[i] || !w[i] || !X[i] || lda[i] < n[i] || ldX[i] < n[i])
      return EVD_ERR_INVALID_ARG;
  const long need = evd_syevd_batched_work_size(count, n, nstreams);
  if (need <= 0) return EVD_ERR_INVALID_ARG;
  if (lwork_bytes < need) return EVD_ERR_WORKSPACE;
  const int workers = (int)std::min<long>(nstreams, count);
  const size_t slice = evd::slice_bytes(count, n);
  char* base = reinterpret_cast<char*>(((uintptr_t)work + 255) & ~(uintptr_t)255);

  std::vector<long> order(count);
  std::iota(order.begin(), order.end(), 0L);
  std::stable_sort(order.begin(), order.end(), [&](long a, long b) { return n[a] > n[b]; });

  int dev = 0;
  EVD_CUDA_TRY(cudaGetDevice(&dev));
  cudaEvent_t start;
  EVD_CUDA_TRY(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
  EVD_CUDA_TRY(cudaEventRecord(start, stream));
  std::vector<cudaStream_t> streams(workers, nullptr);
  std::vector<cudaEvent_t> ends(workers, nullptr);
  int rc = EVD_SUCCESS;
  for (int t = 0; t < workers && rc == EVD_SUCCESS; ++t) {
    if (cudaStreamCreateWithFlags(&streams[t], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ends[t], cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamWaitEvent(streams[t], start, 0) != cudaSuccess)
      rc = EVD_ERR_CUDA;
  }
  if (rc == EVD_SUCCESS) {
    std::atomic<long> next{0};
    std::atomic<int> first_error{EVD_SUCCESS};
    auto worker = [&](int t) {
      cudaSetDevice(dev);
      void* ws = base + (size_t)t * slice;
      for (;;) {
        if (first_error.load() != EVD_SUCCESS) break;
        const long k = next.fetch_add(1);
        if (k >= count) break;
        const long i = order[k];
        const int st = evd::syevd(n[i], 32, evd::batch_nb(n[i]), A[i], lda[i], w[i], X[i], ldX[i],
                                  ws, (long)slice, 0, streams[t]);
        if (st != EVD_SUCCESS) {
          int expect = EVD_SUCCESS;
          first_error.compare_exchange_strong(expect, st);
        }
      }
      cudaEventRecord(ends[t], streams[t]);
    };
    std::vector<std::thread> threads;
    try {
      threads.reserve(workers);
      for (int t = 0; t < workers; ++t) threads.emplace_back(worker, t);
    } catch (...) {  // a thread could not start: the started ones stop and are joined
      int expect = EVD_SUCCESS;
      first_error.compare_exchange_strong(expect, EVD_ERR_HOST);
    }
    for (auto& th : threads) th.join();
    rc = first_error.load();
    for (int t = 0; t < workers; ++t)
      if (cudaStreamWaitEvent(stream, ends[t], 0) != cudaSuccess && rc == EVD_SUCCESS)
        rc = EVD_ERR_CUDA;
  }
  for (int t = 0; t < workers; ++t) {
    if (streams[t]) cudaStreamSynchronize(streams[t]);
    if (ends[t]) cudaEventDestroy(ends[t]);
    if (streams[t]) cudaStreamDestroy(streams[t]);
  }
  cudaEventDestroy(start);
  return rc;
}

// The C ABI never lets a C++ exception (host allocation, thread creation)
// escape: it becomes EVD_ERR_HOST.
extern "C" int evd_syevd_batched(long count, const long* n, const double* const* A,
                                 const long* lda, double* const* w, double* const* X,
                                 const long* ldX, int nstreams, void* work, long lwork_bytes,
                                 cudaStream_t stream) {
  try {
    return syevd_batched_impl(count, n, A, lda, w, X, ldX, nstreams, work, lwork_bytes, stream);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}
