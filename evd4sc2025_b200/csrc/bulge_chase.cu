// Stage 2: band -> tridiagonal bulge chasing, persistent sm_100a kernel.
//
// Algorithm (same reflectors, same storage as chasing_kernel_one_timeV10,
// util/inc/bugle_chasingV10.h:21-392): sweep s (s = 0..n-3) annihilates column
// s below the subdiagonal.  Step k of sweep s works at opRow r = s+1+k*b:
//   u  = house(B1[:,0])                       (||u||^2 = 2, :137-200)
//   B1 = H B1,  S2 = H S2 H,  B1' = B1' H      (:207-336)
// where B1 is the block left of the diagonal block S2 (rows r..r+b-1) and B1'
// the bulge block below S2.  u is stored into U(r:r+b, s).
//
// B200 design (not the reference's): instead of one 1024-thread CTA per sweep
// with a grid.sync() after every step, each sweep is owned by ONE warp that
// keeps B1/S2/B1' in a private shared-memory window, and sweeps are pipelined
// through point-to-point progress flags (acquire/release at gpu scope).
// Workers take sweeps from an atomic ticket, so the sweep a warp waits on was
// taken earlier by a warp that is already running: no co-residency
// requirement, no cooperative launch.  The dependency rule is the reference's
// (step at opRow r may run once the previous sweep has published
// prog >= r + 2b, :81).  Every wait is bounded in time; on timeout the kernel
// records an error word and all workers drain, nothing spins forever.
#include "common.cuh"

namespace evd {

namespace {

constexpr int kChaseWarpsPerCta = 4;
constexpr unsigned long long kWaitTimeoutNs = 4000000000ull;  // 4 s

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Lane 0 waits until *flag >= target (or an error is raised elsewhere).
// Returns false when the sweep must be abandoned.
__device__ bool warp_wait_geq(const int* flag, int target, int* err, int code) {
  const int lane = threadIdx.x & 31;
  int ok = 1;
  if (lane == 0) {
    if (ld_acquire(flag) < target) {
      unsigned long long t0 = globaltimer_ns();
      unsigned spins = 0;
      while (ld_acquire(flag) < target) {
        __nanosleep(40);
        if ((++spins & 63u) == 0) {
          if (*(volatile int*)err != 0) {
            ok = 0;
            break;
          }
          if (globaltimer_ns() - t0 > kWaitTimeoutNs) {
            atomicCAS(err, 0, code);
            ok = 0;
            break;
          }
        }
      }
    }
  }
  ok = __shfl_sync(0xffffffffu, ok, 0);
  if (ok) (void)ld_acquire(flag);  // every lane acquires
  return ok != 0;
}

__device__ __forceinline__ void warp_publish(int* flag, int value) {
  __threadfence();
  __syncwarp();
  if ((threadIdx.x & 31) == 0) st_release(flag, value);
}

template <int BW>
__global__ void __launch_bounds__(32 * kChaseWarpsPerCta)
    chase_kernel(int n, double* __restrict__ sub, long ld, double* __restrict__ U, long ldU,
                 int* prog, int* ticket, int* err) {
  constexpr int LD = BW + 1;  // padded row stride of the per-warp tiles
  constexpr int kPerWarp = 3 * BW * LD + 2 * BW;
  extern __shared__ double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* base = sm + warp * kPerWarp;
  double* tB = base;                  // current B1 (row-major, rows = lanes)
  double* tN = base + BW * LD;        // bulge block B1'
  double* tS = base + 2 * BW * LD;    // diagonal block S2 (lower part)
  double* us = base + 3 * BW * LD;    // Householder vector
  double* vs = us + BW;               // symmetric-update vector

  for (;;) {
    int s = 0;
    if (lane == 0) s = atomicAdd(ticket, 1);
    s = __shfl_sync(0xffffffffu, s, 0);
    if (s >= n - 2) break;
    if (*(volatile int*)err != 0) break;

    long r = s + 1;
    int rb = min(BW, (int)(n - r));
    int cb = 1;
    if (s > 0 && !warp_wait_geq(prog + s - 1, (int)(r + 2 * BW), err, kDevTimeoutChase)) break;

    // B1 = column s, rows r .. r+rb-1
#pragma unroll
    for (int c = 0; c < BW; ++c) tB[lane * LD + c] = 0.0;
    if (lane < rb) tB[lane * LD] = __ldcg(sub + (1 + lane) + (long)s * ld);
    __syncwarp();

    bool alive = true;
    for (;;) {
      // Issue every load of this step (diagonal block S2, lower part, and the
      // bulge block B1' below it) first: one L2 round trip per step, overlapped
      // with the Householder vector and the B1 update below.
      const long r2 = r + rb;
      const int rb2 = min(BW, (int)(n - r2));
      double ls[BW], ln[BW];
#pragma unroll
      for (int c = 0; c < BW; ++c)
        ls[c] = (c <= lane && lane < rb && c < rb) ? __ldcg(sub + (lane - c) + (r + c) * ld) : 0.0;
#pragma unroll
      for (int c = 0; c < BW; ++c)
        ln[c] = (lane < rb2 && c < rb) ? __ldcg(sub + (rb + lane - c) + (r + c) * ld) : 0.0;

      // ---- Householder vector from B1[:,0] (reference convention) ----
      double x = (lane < rb) ? tB[lane * LD] : 0.0;
      double nrm2 = warp_sum(x * x);
      double u = 0.0;
      if (nrm2 > 0.0) {
        double scale = 1.0 / sqrt(nrm2);
        u = x * scale;
        double u0 = __shfl_sync(0xffffffffu, u, 0);
        double u0n = u0 + ((u0 >= 0.0) ? 1.0 : -1.0);
        if (lane == 0) u = u0n;
        u *= 1.0 / sqrt(fabs(u0n));
      }
      us[lane] = u;
      if (lane < rb) U[(r + lane) + (long)s * ldU] = u;
      __syncwarp();

      // ---- B1 <- H B1 (lane c owns column c) ----
      if (lane < cb) {
        double v = 0.0;
#pragma unroll
        for (int l = 0; l < BW; ++l) v = fma(us[l], tB[l * LD + lane], v);
#pragma unroll
        for (int l = 0; l < BW; ++l) tB[l * LD + lane] = fma(-v, us[l], tB[l * LD + lane]);
      }
      __syncwarp();
      // write back B1: element (r+l, r-cb+c) -> sub[(cb+l-c) + (r-cb+c)*ld]
      for (int c = 0; c < cb; ++c)
        if (lane < rb) __stcg(sub + (cb + lane - c) + (r - cb + c) * ld, tB[lane * LD + c]);

      // ---- S2 <- H S2 H  (symmetric rank-2 form, lower part stored) ----
#pragma unroll
      for (int c = 0; c < BW; ++c) tS[lane * LD + c] = ls[c];
#pragma unroll
      for (int c = 0; c < BW; ++c) tN[lane * LD + c] = ln[c];
      __syncwarp();
      double y = 0.0;
      if (lane < rb) {
#pragma unroll
        for (int c = 0; c < BW; ++c) {
          if (c < rb) {
            double sv = (c <= lane) ? tS[lane * LD + c] : tS[c * LD + lane];
            y = fma(sv, us[c], y);
          }
        }
      }
      double tt = warp_sum(u * y);
      double v = y - 0.5 * tt * u;
      vs[lane] = v;
      __syncwarp();
      if (lane < rb) {
#pragma unroll
        for (int c = 0; c < BW; ++c)
          if (c <= lane) tS[lane * LD + c] -= u * vs[c] + v * us[c];
      }
      __syncwarp();
      for (int c = 0; c < rb; ++c)
        if (lane >= c && lane < rb) __stcg(sub + (lane - c) + (r + c) * ld, tS[lane * LD + c]);

      // ---- bulge block B1' (rows r2.., cols r..r+rb-1) <- B1' H ----
      if (rb2 > 0) {
        double w = 0.0;
#pragma unroll
        for (int c = 0; c < BW; ++c) w = fma(tN[lane * LD + c], us[c], w);
#pragma unroll
        for (int c = 0; c < BW; ++c) tN[lane * LD + c] = fma(-w, us[c], tN[lane * LD + c]);
      }
      __syncwarp();
      if (rb2 <= 1) {
        if (rb2 == 1 && lane < rb) __stcg(sub + (rb - lane) + (r + lane) * ld, tN[lane]);
        warp_publish(prog + s, n + 3 * BW);
        break;
      }
      warp_publish(prog + s, (int)r2);

      cb = rb;
      rb = rb2;
      r = r2;
      double* tmp = tB;
      tB = tN;
      tN = tmp;
      if (s > 0 && !warp_wait_geq(prog + s - 1, (int)(r + 2 * BW), err, kDevTimeoutChase)) {
        alive = false;
        break;
      }
    }
    if (!alive) break;
    // restore tile roles for the next sweep
    tB = base;
    tN = base + BW * LD;
  }
}

__global__ void band_pack_kernel(int n, int b, const double* __restrict__ A, long ldA,
                                 double* __restrict__ sub, long ldSub) {
  long j = blockIdx.x * (long)blockDim.y + threadIdx.y;
  if (j >= n) return;
  for (int i = threadIdx.x; i < ldSub; i += blockDim.x) {
    double v = 0.0;
    if (i < 2 * b && i <= b && j + i < n) v = A[(j + i) + j * ldA];
    sub[i + j * ldSub] = v;
  }
}

__global__ void band_to_tridiag_kernel(int n, const double* __restrict__ sub, long ldSub,
                                       double* __restrict__ d, double* __restrict__ e) {
  long j = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (j >= n) return;
  d[j] = sub[j * ldSub];
  if (j < n - 1) e[j] = sub[1 + j * ldSub];
}

}  // namespace

int band_pack(long n, long b, const double* dA, long ldA, double* dSub, long ldSub,
              cudaStream_t st) {
  if (n < 0 || b <= 0 || ldA < n || ldSub < 2 * b) return EVD_ERR_INVALID_ARG;
  if (n == 0) return EVD_SUCCESS;
  dim3 blk(32, 8);
  band_pack_kernel<<<ceil_div_i(n, 8), blk, 0, st>>>((int)n, (int)b, dA, ldA, dSub, ldSub);
  EVD_CUDA_TRY(cudaGetLastError());
  return EVD_SUCCESS;
}

long chase_iwork_ints(long n) { return n + 64; }

// Launch the chase; does not synchronise.  iwork: chase_iwork_ints(n) ints.
// The error word is iwork[n + 32] (0 = ok).
int bulge_chase_async(long n, long b, double* dSub, long ldSub, double* dU, long ldU,
                      double* d, double* e, int* iwork, cudaStream_t st) {
  if (n < 0 || b != 32 || ldSub < 2 * b || (n > 0 && ldU < n)) return EVD_ERR_INVALID_ARG;
  if (n > (1L << 30)) return EVD_ERR_INVALID_ARG;
  if (n == 0) return EVD_SUCCESS;
  if (!dSub || !d || !iwork || (n > 2 && !dU) || (n > 1 && !e)) return EVD_ERR_INVALID_ARG;
  int* prog = iwork;
  int* ticket = iwork + n;
  int* err = iwork + n + 32;
  EVD_CUDA_TRY(cudaMemsetAsync(iwork, 0, sizeof(int) * chase_iwork_ints(n), st));
  if (n > 2) {
    constexpr int BW = 32;
    constexpr size_t smem = kChaseWarpsPerCta * (3 * BW * (BW + 1) + 2 * BW) * sizeof(double);
    static bool attr = false;
    if (!attr) {
      EVD_CUDA_TRY(cudaFuncSetAttribute(chase_kernel<BW>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      attr = true;
    }
    long sweeps = n - 2;
    long max_workers = 2L * device_sm_count() * kChaseWarpsPerCta;
    long workers = std::min(sweeps, max_workers);
    int ctas = ceil_div_i(workers, kChaseWarpsPerCta);
    chase_kernel<BW><<<ctas, 32 * kChaseWarpsPerCta, smem, st>>>((int)n, dSub, ldSub, dU, ldU,
                                                                 prog, ticket, err);
    EVD_CUDA_TRY(cudaGetLastError());
  }
  band_to_tridiag_kernel<<<ceil_div_i(n, 256), 256, 0, st>>>((int)n, dSub, ldSub, d, e);
  EVD_CUDA_TRY(cudaGetLastError());
  return EVD_SUCCESS;
}

int read_device_error(const int* err_word, cudaStream_t st) {
  int h = 0;
  EVD_CUDA_TRY(cudaMemcpyAsync(&h, err_word, sizeof(int), cudaMemcpyDeviceToHost, st));
  EVD_CUDA_TRY(cudaStreamSynchronize(st));
  if (h == kDevTimeoutChase || h == kDevTimeoutTree) return EVD_ERR_TIMEOUT;
  if (h == kDevNoConvergence) return EVD_ERR_NO_CONVERGENCE;
  if (h != 0) return EVD_ERR_INVALID_ARG;
  return EVD_SUCCESS;
}

}  // namespace evd

extern "C" int evd_band_pack(long n, long b, const double* dA, long ldA, double* dSub,
                             long ldSub, cudaStream_t stream) {
  return evd::band_pack(n, b, dA, ldA, dSub, ldSub, stream);
}

extern "C" long evd_bulge_chase_iwork_size(long n) {
  return (long)sizeof(int) * evd::chase_iwork_ints(n < 0 ? 0 : n);
}

extern "C" int evd_bulge_chase(long n, long b, double* dSub, long ldSub, double* dU, long ldU,
                               double* d, double* e, int* iwork, cudaStream_t stream) {
  int rc = evd::bulge_chase_async(n, b, dSub, ldSub, dU, ldU, d, e, iwork, stream);
  if (rc != EVD_SUCCESS || n <= 2) return rc;
  return evd::read_device_error(iwork + n + 32, stream);
}
