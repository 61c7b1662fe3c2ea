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
// B200 design (not the reference's, which runs one 1024-thread CTA per sweep
// and a grid.sync() after every step):
//  * each sweep is owned by one 128-thread CTA; sweeps are pipelined through
//    point-to-point progress flags (acquire/release, gpu scope) with the
//    reference's rule (a step at opRow r may run once the previous sweep has
//    published prog >= r + 2b, :81).  CTAs take sweeps from an atomic ticket,
//    so any sweep a CTA waits on belongs to a CTA that is already running.
//  * a step touches band columns [r, r+32) (S2 and B1') and [r-32, r) (B1).
//    In band storage (ld = 2b) those are contiguous 16 KB tiles: each step
//    copies one tile (columns [r, r+32), all 64 offsets) into shared memory
//    with 16-byte cp.async and stores the previous one, instead of gathering
//    blocks element by element.
//  * the copy is asynchronous and issued before the Householder vector and the
//    B1 update, which only need data already in shared memory, so its latency
//    overlaps that work; the previous tile is stored right after the B1 update.
//  * S2 <- H S2 H uses the symmetric rank-2 form (y = S u, v = y - (u^T y/2) u,
//    S -= u v^T + v u^T) and every block update runs on 128 threads (4 per
//    row/column; each dot product ends with a 4-lane sum on the DMMA pipe).
//  * every wait is bounded in time; on timeout the kernel records an error
//    word, all CTAs drain, and the host returns EVD_ERR_TIMEOUT.
#include <mutex>

#include "common.cuh"

namespace evd {

namespace {

constexpr int kBW = 32;                  // band width b
constexpr int kOff = 2 * kBW;            // band-storage rows per column (2b)
constexpr int kTileD = kBW * kOff;       // doubles per 32-column tile
constexpr int kChaseThreads = 128;
constexpr unsigned long long kWaitTimeoutNs = 4000000000ull;  // 4 s

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// All threads' prior writes -> visible at gpu scope, then thread 0 publishes.
__device__ __forceinline__ void cta_publish(int* flag, int value) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    st_release(flag, value);
  }
}

// Start the copy of band columns [c0, c0+ncol) (all 2b offsets) into smem;
// columns past ncol are zero-filled.  Completed by cp_async_commit_wait_all().
__device__ __forceinline__ void tile_load_async(double* t, const double* sub, long c0, int ncol) {
  const double2* src = reinterpret_cast<const double2*>(sub + c0 * kOff);
  double2* dst = reinterpret_cast<double2*>(t);
  const int n2 = ncol * kOff / 2;
  for (int i = threadIdx.x; i < kTileD / 2; i += kChaseThreads) {
    if (i < n2) cp_async16(dst + i, src + i);
    else dst[i] = make_double2(0.0, 0.0);
  }
}
__device__ __forceinline__ void tile_store(double* sub, const double* t, long c0, int ncol) {
  double2* dst = reinterpret_cast<double2*>(sub + c0 * kOff);
  const double2* src = reinterpret_cast<const double2*>(t);
  const int n2 = ncol * kOff / 2;
  for (int i = threadIdx.x; i < n2; i += kChaseThreads) __stcg(dst + i, src[i]);
}

// Reductions on the tensor pipe.  Inside a chase step the warp shuffles queue
// behind the shared-memory traffic of the tile copies (a 5-level shuffle sum
// took about 2400 cycles there, 190 alone); the DMMA unit is otherwise idle.
// mma.m8n8k4.f64 fragments: lane l holds A[l/4][l%4], B[l%4][l/4] and
// D[l/4][2(l%4)], D[l/4][2(l%4)+1].
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%4,%5};\n"
      : "=d"(d0), "=d"(d1)
      : "d"(a), "d"(b), "d"(0.0), "d"(0.0));
}

// Sum over each quad of lanes (4i .. 4i+3): A = values, B = ones.
__device__ __forceinline__ double quad_sum_tc(double v) {
  double d0, d1;
  dmma884(d0, d1, v, 1.0);
  return d0;
}

// Sum over the warp, returned to every lane: quad sums s_i (A = values,
// B = ones); then B2[0][j] = s_j gives D = s_j per column, so lane l holds
// s_{2(l%4)} and s_{2(l%4)+1}; their sum u_{l%4} as A3[i][k] = u_k against
// ones adds the four u_k.
__device__ __forceinline__ double warp_sum_tc(double v) {
  const int lane = threadIdx.x & 31;
  double d0, d1;
  dmma884(d0, d1, v, 1.0);
  dmma884(d0, d1, 1.0, (lane & 3) == 0 ? d0 : 0.0);
  const double u = d0 + d1;
  dmma884(d0, d1, u, 1.0);
  return d0;
}

struct ChaseSmem {
  double tile[2][kTileD];  // band columns [base, base+32), element (c, o) at c*64 + o
  double u[kBW];
  double v[kBW];
  double red[4];
  int ticket;
};

// Thread 0 waits until *flag >= target (or an error is raised elsewhere); the
// barrier itself (__syncthreads_and) gives every thread the verdict.
// false = abandon the sweep.
__device__ bool cta_wait_and(const int* flag, int target, int* err) {
  int ok = 1;
  if (threadIdx.x == 0 && ld_acquire(flag) < target) {
    unsigned long long t0 = globaltimer_ns();
    unsigned spins = 0;
    while (ld_acquire(flag) < target) {
      __nanosleep(32);
      if ((++spins & 31u) == 0) {
        if (*(volatile int*)err != 0) {
          ok = 0;
          break;
        }
        if (globaltimer_ns() - t0 > kWaitTimeoutNs) {
          atomicCAS(err, 0, kDevTimeoutChase);
          ok = 0;
          break;
        }
      }
    }
  }
  return __syncthreads_and(ok) != 0;
}

__global__ void __launch_bounds__(kChaseThreads)
    chase_kernel(int n, double* __restrict__ sub, double* __restrict__ U, long ldU, int* prog,
                 int* ticket, int* err, int s_begin, int s_end) {
  __shared__ __align__(16) ChaseSmem sm;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  // 4 threads per row / column: q = index (0..31), p = part (0..3, 8 entries each)
  const int q = tid >> 2, p = tid & 3;

  for (;;) {
    if (tid == 0) {
      int t = s_begin + atomicAdd(ticket, 1);
      if (*(volatile int*)err != 0) t = n;  // drain after an error elsewhere
      sm.ticket = t;
    }
    __syncthreads();
    const int s = sm.ticket;
    __syncthreads();
    if (s >= s_end) break;

    long r = s + 1;
    int rb = min(kBW, (int)(n - r));
    int cb = 1;  // columns of the previous tile (B1): 1 at the first step
    int cur = 0;
    if (s > 0 && !cta_wait_and(prog + s - 1, (int)(r + 2 * kBW), err)) break;
    // previous tile = column s (its offsets 1..rb hold B1 = A(r:r+rb, s))
    tile_load_async(sm.tile[1 - cur], sub, s, 1);
    cp_async_commit_wait_all();
    __syncthreads();

    bool alive = true;
    for (;;) {
      double* T = sm.tile[cur];       // columns [r, r+32): S2 and B1'
      double* P = sm.tile[1 - cur];   // columns [r-cb, r): B1 at offsets cb+i-j
      const long r2 = r + rb;
      const int rb2 = min(kBW, (int)(n - r2));
      // (1) start copying this step's tile; nothing below reads T until (4)
      tile_load_async(T, sub, r, min(kBW, (int)(n - r)));

      // (2) Householder vector from B1[:, 0] = P[0][cb + i]
      if (warp == 0) {
        const double x = (lane < rb) ? P[cb + lane] : 0.0;
        const double nrm2 = warp_sum_tc(x * x);
        double u = 0.0;
        if (nrm2 > 0.0) {
          u = x * rsqrt(nrm2);
          const double u0 = __shfl_sync(0xffffffffu, u, 0);
          const double u0n = u0 + ((u0 >= 0.0) ? 1.0 : -1.0);
          if (lane == 0) u = u0n;
          u *= rsqrt(fabs(u0n));
        }
        sm.u[lane] = u;
        if (U != nullptr && lane < rb) U[(r + lane) + (long)s * ldU] = u;
      }
      __syncthreads();

      // (3) B1 <- H B1 : column j = q, rows 8p..8p+7 (B1 is rb x cb)
      {
        const int j = q;
        double pv = 0.0;
        if (j < cb) {
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const int i = 8 * p + k;
            pv = fma(sm.u[i], P[j * kOff + cb + i - j], pv);
          }
        }
        pv = quad_sum_tc(pv);
        if (j < cb) {
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const int i = 8 * p + k;
            if (i < rb) P[j * kOff + cb + i - j] = fma(-pv, sm.u[i], P[j * kOff + cb + i - j]);
          }
        }
      }
      __syncthreads();
      // the previous tile (S2 of the last step + this B1) is now final: store
      // it and publish progress right away.  A successor may then read
      // columns < prog - 32 = r, i.e. exactly what has been stored; this
      // step's S2 and B1' (columns >= r) are not needed by it yet, so the
      // updates below stay off the inter-sweep critical path.
      tile_store(sub, P, r - cb, cb);
      // (4) this thread's copies of T are done; the barrier makes all visible
      cp_async_commit_wait_all();
      __syncthreads();
      if (rb2 > 1 && tid == 0) {
        __threadfence();
        st_release(prog + s, (int)r2);
      }

      // (5) S2 <- H S2 H  with S(i, j) = T[j][i-j] (i >= j)
      {
        const int i = q;
        double y = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int j = 8 * p + k;
          const double sv = (j <= i) ? T[j * kOff + (i - j)] : T[i * kOff + (j - i)];
          y = fma(sv, sm.u[j], y);
        }
        y = quad_sum_tc(y);
        // t = u^T y over the 32 rows: rows 8w..8w+7 live in warp w (p == 0 lanes)
        double uy = (p == 0) ? sm.u[i] * y : 0.0;
        uy = warp_sum_tc(uy);
        if (lane == 0) sm.red[warp] = uy;
        if (p == 0) sm.v[i] = y;  // y here; v_j = y_j - t u_j / 2 is formed below
        __syncthreads();
        const double t = (sm.red[0] + sm.red[1]) + (sm.red[2] + sm.red[3]);
        const double vi = y - 0.5 * t * sm.u[i];
        const double ui = sm.u[i];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int j = 8 * p + k;
          const double vj = sm.v[j] - 0.5 * t * sm.u[j];
          if (j <= i && i < rb) T[j * kOff + (i - j)] -= ui * vj + vi * sm.u[j];
        }
      }
      // (6) B1' <- B1' H : row i = q (rows r+rb+i), N(i, j) = T[j][rb + i - j].
      // S2 owns offsets <= rb-1-j of column j, B1' offsets >= rb-j: no overlap.
      if (rb2 > 0) {
        const int i = q;
        double w = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int j = 8 * p + k;
          if (j < rb) w = fma(T[j * kOff + rb + i - j], sm.u[j], w);
        }
        w = quad_sum_tc(w);
        if (i < rb2) {
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const int j = 8 * p + k;
            if (j < rb) T[j * kOff + rb + i - j] = fma(-w, sm.u[j], T[j * kOff + rb + i - j]);
          }
        }
      }
      if (rb2 <= 1) {
        __syncthreads();
        tile_store(sub, T, r, min(kBW, (int)(n - r)));
        cta_publish(prog + s, n + 3 * kBW);
        break;
      }
      cb = rb;
      rb = rb2;
      r = r2;
      cur = 1 - cur;
      // the next step's Householder warp reads B1 = this step's B1', written
      // by all four warps in (6): the wait below ends with a CTA barrier; sweep
      // 0 waits on nobody and takes the barrier alone
      if (s > 0) {
        if (!cta_wait_and(prog + s - 1, (int)(r + 2 * kBW), err)) {
          alive = false;
          break;
        }
      } else {
        __syncthreads();
      }
    }
    if (!alive) break;
    __syncthreads();
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
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

long chase_iwork_ints(long n) { return n + 64; }

// Sweeps [s0, s1) of the chase as one launch (part `part`, 0 <= part < 32, of
// a chase split into consecutive ranges; part 0 starts at s0 = 0 and clears
// the flags, tickets and error word).  Each part has its own ticket counter
// (iwork[n + part]); a part's first sweep waits on the previous sweep's
// progress flag, which the previous part's launch left at its final value.
// Splitting costs one pipeline drain per part boundary: the next part's
// first sweep starts when the previous sweep has reached the end of the band,
// not 2b rows after its start.
int chase_part_async(long n, long b, double* dSub, long ldSub, double* dU, long ldU, int* iwork,
                     long s0, long s1, int part, cudaStream_t st) {
  if (n < 0 || b != kBW || ldSub != 2 * b || (dU && n > 0 && ldU < n)) return EVD_ERR_INVALID_ARG;
  if (((uintptr_t)dSub & 15u) != 0) return EVD_ERR_INVALID_ARG;
  if (n > (1L << 30)) return EVD_ERR_INVALID_ARG;
  if (part < 0 || part >= 32 || s0 < 0 || s1 < s0 || (part == 0) != (s0 == 0))
    return EVD_ERR_INVALID_ARG;
  if (n == 0) return EVD_SUCCESS;
  if (!dSub || !iwork) return EVD_ERR_INVALID_ARG;
  int* prog = iwork;
  int* err = iwork + n + 32;
  if (part == 0) EVD_CUDA_TRY(cudaMemsetAsync(iwork, 0, sizeof(int) * chase_iwork_ints(n), st));
  s1 = std::min(s1, n - 2);
  if (s1 > s0) {
    // enough CTAs for the pipeline's concurrency (a sweep starts every 3 steps
    // and lasts about n/b steps), bounded by the GPU's resident capacity
    const long sweeps = s1 - s0;
    const long want = n / (3 * kBW) + 16;
    const int ctas = (int)std::min(std::min(sweeps, want), 6L * device_sm_count());
    chase_kernel<<<ctas, kChaseThreads, 0, st>>>((int)n, dSub, dU, ldU, prog, iwork + n + part,
                                                 err, (int)s0, (int)s1);
    EVD_LAUNCHED();
  }
  return EVD_SUCCESS;
}

// d and e from the chased band (after the last part).
int chase_tridiag(long n, const double* dSub, long ldSub, double* d, double* e, cudaStream_t st) {
  if (n <= 0) return EVD_SUCCESS;
  if (!dSub || !d || (n > 1 && !e)) return EVD_ERR_INVALID_ARG;
  band_to_tridiag_kernel<<<ceil_div_i(n, 256), 256, 0, st>>>((int)n, dSub, ldSub, d, e);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

// Launch the chase; does not synchronise.  iwork: chase_iwork_ints(n) ints.
// The error word is iwork[n + 32] (0 = ok).
// The tile copies need ldSub == 2b exactly (contiguous band columns) and a
// 16-byte aligned dSub.
int bulge_chase_async(long n, long b, double* dSub, long ldSub, double* dU, long ldU,
                      double* d, double* e, int* iwork, cudaStream_t st) {
  if (n < 0 || b != kBW || ldSub != 2 * b || (dU && n > 0 && ldU < n)) return EVD_ERR_INVALID_ARG;
  if (((uintptr_t)dSub & 15u) != 0) return EVD_ERR_INVALID_ARG;
  if (n > (1L << 30)) return EVD_ERR_INVALID_ARG;
  if (n == 0) return EVD_SUCCESS;
  if (!dSub || !d || !iwork || (n > 1 && !e)) return EVD_ERR_INVALID_ARG;  // dU may be NULL
  EVD_TRY(chase_part_async(n, b, dSub, ldSub, dU, ldU, iwork, 0, n - 2, 0, st));
  return chase_tridiag(n, dSub, ldSub, d, e, st);
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

// ---------------------------------------------------------------------------
// Allocation-free variant of the bulge chasing entry point.
//
// evd_bulge_chase needs a small integer scratch buffer (progress flags of the
// sweeps, the sweep ticket and an error word) and takes it from the caller.
// Some callers have no way to obtain device memory at the point where they
// run the chase: code that must not call cudaMalloc (it can synchronise the
// whole device, fail under memory pressure, or is simply unavailable to a
// plugin running inside a host framework that owns the allocator), and
// loops that are required to run with a fixed memory footprint.  For them the
// scratch lives in a file-scope device array instead, sized for bands of up
// to kNoAllocMaxN columns (256 KB that every GPU loading this library keeps
// until the process exits).
namespace evd {

constexpr long kNoAllocMaxN = 65536;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) int g_chase_noalloc_scratch[kNoAllocMaxN + 64];

// Device address of the scratch on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up with
// cudaGetSymbolAddress, once per device (with that device current), and cached.
static int chase_noalloc_scratch(int** out) {
  static std::mutex mu;
  static int* addr[kNoAllocMaxDevices] = {};
  int dev = 0;
  EVD_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return EVD_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(mu);
  if (addr[dev] == nullptr) {
    void* p = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&p, g_chase_noalloc_scratch);
    if (rc != cudaSuccess || p == nullptr) {
      fprintf(stderr, "evd_b200: cudaGetSymbolAddress for the chase scratch failed: %s\n",
              cudaGetErrorString(rc));
      return EVD_ERR_CUDA;
    }
    addr[dev] = static_cast<int*>(p);
  }
  *out = addr[dev];
  return EVD_SUCCESS;
}

}  // namespace evd

extern "C" int evd_bulge_chase_noalloc(long n, long b, double* dSub, long ldSub, double* dU,
                                       long ldU, double* d, double* e, cudaStream_t stream) {
  if (n > evd::kNoAllocMaxN) {
    fprintf(stderr,
            "evd_b200: evd_bulge_chase_noalloc supports n <= %ld (got n = %ld); use "
            "evd_bulge_chase with a caller-provided scratch buffer\n",
            evd::kNoAllocMaxN, n);
    return EVD_ERR_INVALID_ARG;
  }
  int* iw = nullptr;
  EVD_TRY(evd::chase_noalloc_scratch(&iw));
  // bulge_chase_async clears the flags, ticket and error word of the scratch
  // (cudaMemsetAsync) before every launch, so a call never sees stale state.
  int rc = evd::bulge_chase_async(n, b, dSub, ldSub, dU, ldU, d, e, iw, stream);
  if (rc != EVD_SUCCESS || n <= 2) return rc;
  return evd::read_device_error(iw + n + 32, stream);
}
