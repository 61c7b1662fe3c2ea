// Reduced-precision entry points of the reference's public API.
//
// The reference instantiates its panel QR and trailing SYR2K for float and
// half besides double (api/panelQR.cu:262-701, api/TCblas/tc_ozimmu_syr2k.cu:
// 343-629 and :683-720) and has a mixed update `tc_syr2k` (FP32 data, FP16
// tensor-core products, FP32 accumulation; api/TCblas/tc_syr2k.cu:144-330).
// The B200 versions:
//
// * tc_syr2k and the half SYR2K run one tcgen05 kernel: both operands are
//   packed once as FP16 rows with K contiguous (into the reference's `hwork`
//   when it fits, else a stream-ordered buffer), copied by TMA into 128-byte-
//   swizzled shared-memory tiles, multiplied 64 K at a time by
//   `tcgen05.mma.kind::f16` (M128 N256) into FP32 accumulators in tensor
//   memory by a persistent warp-specialised kernel, and the epilogue applies
//   alpha / beta on the lower triangle.  A B^T + B A^T is one product over
//   the concatenated K range: [A | B] * [B | A]^T.
// * the FP32 SYR2K is a SIMT FP32 kernel (exact FP32 multiply-add, the
//   arithmetic of CUBLAS_COMPUTE_32F that the reference asks cuBLAS for).
// * the FP32 / FP16 panel QR and TSQR convert the panel to FP64, run the
//   FP64 panel kernels (the panel is latency-bound: FP64 costs nothing there
//   and is more accurate) and round the results back.
#include <cuda_fp16.h>
#include <math.h>

#include <mutex>

#include "common.cuh"
#include "ozaki.cuh"
#include "panel_qr.cuh"

namespace evd {
namespace {

// ------------------------------------------------------------ conversions
__device__ __forceinline__ double to_d(float x) { return (double)x; }
__device__ __forceinline__ double to_d(__half x) { return (double)__half2float(x); }
__device__ __forceinline__ void from_d(double x, float* p) { *p = (float)x; }
__device__ __forceinline__ void from_d(double x, __half* p) { *p = __double2half(x); }

template <typename T>
__global__ void to_double_kernel(long m, long n, const T* __restrict__ src, long lds,
                                 double* __restrict__ dst, long ldd) {
  for (long j = blockIdx.y; j < n; j += gridDim.y)
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m; i += (long)gridDim.x * blockDim.x)
      dst[i + j * ldd] = to_d(src[i + j * lds]);
}

template <typename T>
__global__ void from_double_kernel(long m, long n, const double* __restrict__ src, long lds,
                                   T* __restrict__ dst, long ldd) {
  for (long j = blockIdx.y; j < n; j += gridDim.y)
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m; i += (long)gridDim.x * blockDim.x)
      from_d(src[i + j * lds], dst + i + j * ldd);
}

template <typename T>
int to_double(long m, long n, const T* src, long lds, double* dst, long ldd, cudaStream_t st) {
  if (m <= 0 || n <= 0) return EVD_SUCCESS;
  dim3 g((unsigned)std::min<long>(ceil_div_i(m, 256), 1024), (unsigned)std::min<long>(n, 65535));
  to_double_kernel<T><<<g, 256, 0, st>>>(m, n, src, lds, dst, ldd);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

template <typename T>
int from_double(long m, long n, const double* src, long lds, T* dst, long ldd, cudaStream_t st) {
  if (m <= 0 || n <= 0) return EVD_SUCCESS;
  dim3 g((unsigned)std::min<long>(ceil_div_i(m, 256), 1024), (unsigned)std::min<long>(n, 65535));
  from_double_kernel<T><<<g, 256, 0, st>>>(m, n, src, lds, dst, ldd);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

// --------------------------------------------------- panel QR in FP32/FP16
// Workspace in doubles: A, W (m x 32), R (32 x 32), then the FP64 panel's.
long lp_panel_ws_doubles(long m) { return 2 * m * 32 + 32 * 32 + 32 + panel_qr_ws_doubles(m); }

template <typename T>
int lp_panel(long m, long n, T* A, long lda, T* W, long ldw, T* R, long ldr, void* work,
             long lwork_bytes, bool form_wy, cudaStream_t st) {
  EVD_TRY(panel_qr_check(m, n, lda));
  if (!A || !R || !work || ldr < n || (form_wy && (!W || ldw < m))) return EVD_ERR_INVALID_ARG;
  if (lwork_bytes < (long)sizeof(double) * lp_panel_ws_doubles(m)) return EVD_ERR_WORKSPACE;
  double* base = reinterpret_cast<double*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
  // the alignment step may cost up to 255 bytes: the size query adds 32 doubles
  double* Ad = base;
  double* Wd = Ad + m * 32;
  double* Rd = Wd + m * 32;
  double* ws = Rd + 32 * 32;
  EVD_TRY(to_double(m, 32, A, lda, Ad, m, st));
  EVD_TRY(panel_counters_reset(m, ws, st));
  if (form_wy) {
    EVD_TRY(panel_qr_launch(m, Ad, m, ws, 1, Ad, m, Wd, m, Rd, 32, nullptr, 0, st));
    EVD_TRY(from_double(m, 32, Wd, m, W, ldw, st));
  } else {
    EVD_TRY(panel_qr_launch(m, Ad, m, ws, 0, nullptr, 0, nullptr, 0, Rd, 32, nullptr, 0, st));
  }
  EVD_TRY(from_double(m, 32, Ad, m, A, lda, st));
  EVD_TRY(from_double(32, 32, Rd, 32, R, ldr, st));
  return EVD_SUCCESS;
}

// ------------------------------------------------------- FP32 SIMT SYR2K
// C(lower) = alpha * [A | B] [B | A]^T + beta * C over lower-triangle tiles
// of 128 x 128; 256 threads, 8 x 8 outputs per thread, K chunks of 8 staged
// in shared memory (double-buffered).
constexpr int kSB = 128;  // tile edge
constexpr int kSK = 8;    // K chunk

__device__ __forceinline__ void tri_tile(long p, long& bi, long& bj) {
  // p -> (bi >= bj) with p = bi (bi + 1) / 2 + bj
  long i = (long)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
  while (i * (i + 1) / 2 > p) --i;
  while ((i + 1) * (i + 2) / 2 <= p) ++i;
  bi = i;
  bj = p - i * (i + 1) / 2;
}

// element kk (0 <= kk < 2k) of row r of the left ([A|B]) or right ([B|A]) operand
template <typename T>
__device__ __forceinline__ float cat_elem(const T* __restrict__ P, long ldp, const T* __restrict__ Q,
                                          long ldq, long n, long k, long r, long kk) {
  if (r >= n) return 0.0f;
  if (kk < k) return (float)P[r + kk * ldp];
  kk -= k;
  if (kk < k) return (float)Q[r + kk * ldq];
  return 0.0f;
}

__global__ void __launch_bounds__(256) ssyr2k_kernel(long n, long k, float alpha,
                                                     const float* __restrict__ A, long lda,
                                                     const float* __restrict__ B, long ldb,
                                                     float beta, float* __restrict__ C, long ldc) {
  __shared__ __align__(16) float Ls[2][kSK][kSB];
  __shared__ __align__(16) float Rs[2][kSK][kSB];
  long bi, bj;
  tri_tile(blockIdx.x, bi, bj);
  const long m0 = bi * kSB, n0 = bj * kSB;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;  // 16 x 16 threads, 8 x 8 each
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
  const long K2 = 2 * k;
  const long nk = (K2 + kSK - 1) / kSK;
  // staging: each thread loads 4 elements of each operand per chunk
  // (row = tid & 127, kk = (tid >> 7) * 4 + q)
  const int lr = tid & 127, lk = (tid >> 7) * 4;
  auto load = [&](long c, float* lv, float* rv) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long kk = c * kSK + lk + q;
      lv[q] = cat_elem(A, lda, B, ldb, n, k, m0 + lr, kk);
      rv[q] = cat_elem(B, ldb, A, lda, n, k, n0 + lr, kk);
    }
  };
  float lv[4], rv[4];
  load(0, lv, rv);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    Ls[0][lk + q][lr] = lv[q];
    Rs[0][lk + q][lr] = rv[q];
  }
  __syncthreads();
  for (long c = 0; c < nk; ++c) {
    const int buf = (int)(c & 1);
    if (c + 1 < nk) load(c + 1, lv, rv);
#pragma unroll
    for (int kk = 0; kk < kSK; ++kk) {
      float a[8], b[8];
      *reinterpret_cast<float4*>(a) = *reinterpret_cast<const float4*>(&Ls[buf][kk][ty * 4]);
      *reinterpret_cast<float4*>(a + 4) = *reinterpret_cast<const float4*>(&Ls[buf][kk][64 + ty * 4]);
      *reinterpret_cast<float4*>(b) = *reinterpret_cast<const float4*>(&Rs[buf][kk][tx * 4]);
      *reinterpret_cast<float4*>(b + 4) = *reinterpret_cast<const float4*>(&Rs[buf][kk][64 + tx * 4]);
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    if (c + 1 < nk) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        Ls[buf ^ 1][lk + q][lr] = lv[q];
        Rs[buf ^ 1][lk + q][lr] = rv[q];
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const long gi = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const long gj = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
      if (gi < n && gj <= gi) {
        float* c = C + gi + gj * ldc;
        *c = (beta == 0.0f) ? alpha * acc[i][j] : fmaf(alpha, acc[i][j], beta * *c);
      }
    }
  }
}

// ------------------------------------------------ tcgen05 FP16 SYR2K (TMEM)
// The operands are packed once into FP16 rows with K contiguous (below), then
// copied into shared memory by TMA and multiplied by tcgen05.mma into FP32
// accumulators in tensor memory.
constexpr int kTM = 128;  // rows of a tile of C (grid-size check)
constexpr unsigned long long kTWaitNs = 2000000000ull;  // 2 s per wait: far above any chunk

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `parity`; false after kTWaitNs (error recorded).
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  for (unsigned it = 0;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63u) == 63u && gtimer() - t0 > kTWaitNs) {
      atomicExch(err, kDevTimeoutTree);
      return false;
    }
  }
}


__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ float ld_elem(const float* p) { return __ldg(p); }
__device__ __forceinline__ float ld_elem(const __half* p) { return __half2float(p[0]); }

__device__ __forceinline__ float ld_c(const float* c) { return *c; }
__device__ __forceinline__ float ld_c(const __half* c) { return __half2float(*c); }
__device__ __forceinline__ void st_c(float* c, float v) { *c = v; }
__device__ __forceinline__ void st_c(__half* c, float v) { *c = __float2half_rn(v); }

__device__ __forceinline__ void store_c(float* c, float v, float alpha, float beta) {
  *c = (beta == 0.0f) ? alpha * v : fmaf(alpha, v, beta * *c);
}
__device__ __forceinline__ void store_c(__half* c, float v, float alpha, float beta) {
  *c = __float2half_rn((beta == 0.0f) ? alpha * v : fmaf(alpha, v, beta * __half2float(*c)));
}

// ---- FP16 operand copy + TMA-fed tensor-core SYR2K ----
// H (n rows x L = 2 kp halves, K contiguous per row, kp = k rounded up to
// 64): H[m][kk] = A(m, kk), H[m][kp + kk] = B(m, kk), zero in the padding.
// Rows of H are the K-major rows the tensor core reads.
template <typename TI>
__global__ void pack_h_kernel(long n, long k, long k8, const TI* __restrict__ A, long lda,
                              const TI* __restrict__ B, long ldb, __half* __restrict__ H) {
  __shared__ float tile[32][33];
  const long L = 2 * k8;
  const long m0 = (long)blockIdx.x * 32, c0 = (long)blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += 8) {  // read along m (coalesced)
    const long m = m0 + threadIdx.x, c = c0 + j;
    float v = 0.0f;
    if (m < n && c < L) {
      if (c < k8) {
        if (c < k) v = ld_elem(A + m + c * lda);
      } else if (c - k8 < k) {
        v = ld_elem(B + m + (c - k8) * ldb);
      }
    }
    tile[threadIdx.x][j] = v;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {  // write along kk (coalesced)
    const long m = m0 + i, c = c0 + threadIdx.x;
    if (m < n && c < L) H[m * L + c] = __float2half_rn(tile[i][threadIdx.x]);
  }
}

// The tensor-core kernel for packed operands: persistent and warp-
// specialised, one CTA per SM walking the lower 128 x 256 tiles of C
// (t = blockIdx.x, + gridDim.x, ...).  Warp 0 lane 0 issues TMA copies
// (cp.async.bulk.tensor, 128-byte swizzle, this GPU's own memory, no
// multicast) of 64-wide K chunks of [A | B] (128 rows) and [B | A] (256 rows)
// into a 4-stage ring; warp 1 lane 0 issues four tcgen05.mma.kind::f16
// M128 N256 K16 per chunk into one of two 256-column FP32 accumulators in
// tensor memory (tile i into buffer i & 1); warps 2-5 drain the other buffer
// (tcgen05.ld, alpha / beta, lower triangle only) while the next tile is
// multiplied.  Every wait is bounded; the MMA thread waits for its last MMAs
// before the tensor memory is freed.  The packed rows are K-major with the K
// range padded to a multiple of 64, so the [B | A] chunk of K offset
// 64 t + kp (mod 2 kp) is one box.
constexpr int kGM = 128, kGN = 256, kGK = 64;        // tile rows, columns, K per chunk
constexpr uint32_t kGTileA = kGM * kGK * 2;          // 16 KB
constexpr uint32_t kGTileB = kGN * kGK * 2;          // 32 KB
constexpr uint32_t kGStage = kGTileA + kGTileB;      // 48 KB
constexpr int kGStages = 4;
constexpr int kGThreads = 192;
constexpr int kGSmem = kGStages * (int)kGStage + 1024 + 256;
// kind::f16 instruction descriptor for M128 N256: D F32, A and B F16, K-major
constexpr uint32_t kGIdesc = (1u << 4) | ((uint32_t)(kGN >> 3) << 17) | ((uint32_t)(kGM >> 4) << 24);

__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  // start >> 4 | LBO 16 B (unused for swizzled K-major) | SBO 1024 B (8-row
  // groups) | version 1 | base offset 0 (tiles 1024-aligned) | SWIZZLE_128B
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load2(void* dst, const CUtensorMap* map, int x, int y,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void umma_f16_n256(uint32_t tmem, uint64_t da, uint64_t db,
                                              uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(da), "l"(db), "r"(kGIdesc), "r"(acc)
      : "memory");
}

// lower tile t (column block bn holds the 128-row tile rows 2 bn .. tm - 1)
__device__ __forceinline__ void g_tile(long t, int tm, int& bm, int& bn) {
  int c = 0;
  for (;; ++c) {
    const long cnt = tm - 2L * c;
    if (t < cnt) break;
    t -= cnt;
  }
  bn = c;
  bm = 2 * c + (int)t;
}

template <typename TC>
__global__ void __launch_bounds__(kGThreads, 1)
    tc_syr2k_tma_kernel(const __grid_constant__ CUtensorMap mapL,
                        const __grid_constant__ CUtensorMap mapR, long n, long kp, float alpha,
                        float beta, TC* __restrict__ C, long ldc, int tm, long ntiles, int* err) {
  extern __shared__ __align__(1024) uint8_t gsm[];
  uint8_t* stages = gsm + ((1024u - (smem_u32(gsm) & 1023u)) & 1023u);
  uint64_t* full = reinterpret_cast<uint64_t*>(stages + kGStages * kGStage);
  uint64_t* empty = full + kGStages;
  uint64_t* tfull = empty + kGStages;
  uint64_t* tempty = tfull + 2;
  uint64_t* done = tempty + 2;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long L = 2 * kp;
  const long nk = L / kGK;

  if (tid == 0) {
    for (int s = 0; s < kGStages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull + b, 1);
      mbar_init(tempty + b, 128);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapL)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapR)) : "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                     smem_u32(tslot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

  if (warp == 0) {
    if (lane == 0) {  // ---- TMA producer ----
      long gk = 0;
      bool ok = true;
      for (long t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        int bm, bn;
        g_tile(t, tm, bm, bn);
        for (long kb = 0; kb < nk; ++kb, ++gk) {
          const int s = (int)(gk % kGStages);
          if (gk >= kGStages &&
              !mbar_wait(empty + s, (uint32_t)((gk / kGStages - 1) & 1), err)) {
            ok = false;
            break;
          }
          uint8_t* sa = stages + s * kGStage;
          long kr = kb * kGK + kp;
          if (kr >= L) kr -= L;
          mbar_expect_tx(full + s, kGStage);
          tma_load2(sa, &mapL, (int)(kb * kGK), bm * kGM, full + s);
          tma_load2(sa + kGTileA, &mapR, (int)kr, bn * kGN, full + s);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer ----
      long gk = 0;
      int i = 0;
      bool ok = true;
      for (long t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++i) {
        const int b = i & 1;
        if (i >= 2 && !mbar_wait(tempty + b, (uint32_t)(((i >> 1) - 1) & 1), err)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc_tm = tmem + (uint32_t)(b * kGN);
        for (long kb = 0; kb < nk; ++kb, ++gk) {
          const int s = (int)(gk % kGStages);
          if (!mbar_wait(full + s, (uint32_t)((gk / kGStages) & 1), err)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sa = smem_u32(stages + s * kGStage);
          const uint32_t sb = sa + kGTileA;
#pragma unroll
          for (int ks = 0; ks < kGK / 16; ++ks)
            umma_f16_n256(acc_tm, smem_desc_sw128(sa + ks * 32), smem_desc_sw128(sb + ks * 32),
                          (kb > 0 || ks > 0) ? 1u : 0u);
          umma_commit(empty + s);
        }
        if (ok) umma_commit(tfull + b);
      }
      umma_commit(done);  // fires when every MMA issued above has completed
      mbar_wait(done, 0, err);
    }
  } else {  // ---- epilogue: warps 2-5, TMEM lanes 32 (warp % 4) .. + 31 ----
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    int i = 0;
    for (long t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
      const int b = i & 1;
      if (!mbar_wait(tfull + b, (uint32_t)((i >> 1) & 1), err)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      int bm, bn;
      g_tile(t, tm, bm, bn);
      const long gi = (long)bm * kGM + row;
      const long n0 = (long)bn * kGN;
#pragma unroll 1
      for (int c0 = 0; c0 < kGN; c0 += 32) {
        uint32_t v[32];
        const uint32_t addr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * kGN + c0);
#pragma unroll
        for (int h = 0; h < 2; ++h)
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
              "%10, %11, %12, %13, %14, %15}, [%16];"
              : "=r"(v[16 * h + 0]), "=r"(v[16 * h + 1]), "=r"(v[16 * h + 2]),
                "=r"(v[16 * h + 3]), "=r"(v[16 * h + 4]), "=r"(v[16 * h + 5]),
                "=r"(v[16 * h + 6]), "=r"(v[16 * h + 7]), "=r"(v[16 * h + 8]),
                "=r"(v[16 * h + 9]), "=r"(v[16 * h + 10]), "=r"(v[16 * h + 11]),
                "=r"(v[16 * h + 12]), "=r"(v[16 * h + 13]), "=r"(v[16 * h + 14]),
                "=r"(v[16 * h + 15])
              : "r"(addr + 16 * h));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (gi < n) {
          const long j0 = n0 + c0;
          // columns j0 .. min(j0 + 31, gi, n - 1) of row gi (jl + 1 of them);
          // the reads of C are issued together before any store (the compiler
          // cannot tell that the stores do not alias them, so it would
          // otherwise wait for each read in turn); every index is static, so
          // v and cv stay in registers
          const long jl = (gi < n - 1 ? gi : n - 1) - j0;
          TC* c = C + gi + j0 * ldc;
          float cv[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) cv[j] = (beta != 0.0f && j <= jl) ? ld_c(c + j * ldc) : 0.0f;
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (j <= jl) st_c(c + j * ldc, fmaf(beta, cv[j], alpha * __uint_as_float(v[j])));
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(tempty + b);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// A, B -> H (n rows x 2 kp halves, kp = k rounded up to 64), then the
// persistent kernel.
template <typename TI, typename TC>
int tc_syr2k_packed(long n, long k, float alpha, const TI* A, long lda, const TI* B, long ldb,
                    float beta, TC* C, long ldc, __half* H, int* err, cudaStream_t st) {
  const long kp = (k + 63) / 64 * 64;
  const long L = 2 * kp;
  dim3 pg((unsigned)((n + 31) / 32), (unsigned)((L + 31) / 32));
  pack_h_kernel<TI><<<pg, dim3(32, 8), 0, st>>>(n, k, kp, A, lda, B, ldb, H);
  EVD_LAUNCHED();
  CUtensorMap mapL, mapR;
  EVD_TRY(tma_map_rows16(&mapL, H, n, L, L, kGM));
  EVD_TRY(tma_map_rows16(&mapR, H, n, L, L, kGN));
  const int tm = (int)((n + kGM - 1) / kGM);
  long ntiles = 0;
  for (long c = 0; 2 * c < tm; ++c) ntiles += tm - 2 * c;
  const int grid = (int)std::min<long>(ntiles, device_sm_count());
  EVD_TRY(smem_attr_once((const void*)tc_syr2k_tma_kernel<TC>, kGSmem));
  tc_syr2k_tma_kernel<TC><<<grid, kGThreads, kGSmem, st>>>(mapL, mapR, n, kp, alpha, beta, C, ldc,
                                                           tm, ntiles, err);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

bool syr2k_args_ok(long n, long k, const void* A, long lda, const void* B, long ldb,
                   const void* C, long ldc) {
  if (n < 0 || k < 0 || ldc < std::max(1L, n)) return false;
  if (n > 0 && !C) return false;
  if (n > 0 && k > 0 && (!A || !B || lda < n || ldb < n)) return false;
  return (n + kTM - 1) / kTM < (1L << 15);  // tile pairs fit one grid dimension
}

// Scale C(lower) by beta (k == 0: no product).
template <typename TC>
__global__ void scale_lower_kernel(long n, float beta, TC* C, long ldc) {
  for (long j = blockIdx.y; j < n; j += gridDim.y)
    for (long i = j + blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
      store_c(C + i + j * ldc, 0.0f, 0.0f, beta);
}

template <typename TC>
int scale_lower(long n, float beta, TC* C, long ldc, cudaStream_t st) {
  if (n <= 0) return EVD_SUCCESS;
  dim3 g((unsigned)std::min<long>(ceil_div_i(n, 256), 1024), (unsigned)std::min<long>(n, 65535));
  scale_lower_kernel<TC><<<g, 256, 0, st>>>(n, beta, C, ldc);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

// error word for the bounded waits of the tensor-core kernel (one per device
// is enough: it only changes when a wait gives up)
int* tc_err_word() {
  static int* dev_word[64] = {nullptr};
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) return nullptr;
  if (!dev_word[d]) {
    int* p = nullptr;
    if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
    if (cudaMemset(p, 0, sizeof(int)) != cudaSuccess) return nullptr;
    dev_word[d] = p;
  }
  return dev_word[d];
}

int check_tc_err(int* err, cudaStream_t st) {
  int h = 0;
  EVD_CUDA_TRY(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  EVD_CUDA_TRY(cudaStreamSynchronize(st));
  if (h != 0) {
    cudaMemsetAsync(err, 0, sizeof(int), st);
    return EVD_ERR_TIMEOUT;
  }
  return EVD_SUCCESS;
}

// Library-private stream-ordered memory pool of the current device: it keeps
// its memory between calls (no release threshold), so a repeated call does
// not pay for a fresh allocation; the application's default pool is left as
// it is.
cudaMemPool_t lp_pool() {
  static cudaMemPool_t pools[64] = {nullptr};
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) return nullptr;
  if (!pools[d]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = d;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = UINT64_MAX;
    if (cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
      return nullptr;
    pools[d] = p;
  }
  return pools[d];
}

// Packs A, B into H (the caller's workspace, or a buffer of n x 2 k8 halves
// from the library's pool when H is null), runs the tensor-core kernel and
// reads the kernel's error word.
template <typename TI, typename TC>
int tc_syr2k_run(long n, long k, float alpha, const TI* A, long lda, const TI* B, long ldb,
                 float beta, TC* C, long ldc, __half* H, cudaStream_t st) {
  const long k8 = (k + 63) / 64 * 64;  // the packed K range (a multiple of 64)
  if ((2 * k8 + 31) / 32 >= 65536 || (n + 31) / 32 >= (1L << 31)) return EVD_ERR_INVALID_ARG;
  int* err = tc_err_word();
  if (!err) return EVD_ERR_CUDA;
  __half* own = nullptr;
  if (H == nullptr) {
    cudaMemPool_t pool = lp_pool();
    if (!pool) return EVD_ERR_CUDA;
    EVD_CUDA_TRY(
        cudaMallocFromPoolAsync((void**)&own, sizeof(__half) * (size_t)n * 2 * k8, pool, st));
    H = own;
  }
  const int rc = tc_syr2k_packed(n, k, alpha, A, lda, B, ldb, beta, C, ldc, H, err, st);
  if (own) EVD_CUDA_TRY(cudaFreeAsync(own, st));
  EVD_TRY(rc);
  return check_tc_err(err, st);
}

}  // namespace
}  // namespace evd

using evd::lp_panel;

// ---------------------------------------------------------------- C ABI
extern "C" long evd_panel_qr_lp_work_size(long m, long n) {
  if (evd::panel_qr_check(m, n, m) != EVD_SUCCESS) return 0;
  return (long)sizeof(double) * evd::lp_panel_ws_doubles(m);
}

extern "C" int evd_panel_qr_s(long m, long n, float* A, long lda, float* W, long ldw, float* R,
                              long ldr, void* work, long lwork_bytes, cudaStream_t stream) {
  return lp_panel(m, n, A, lda, W, ldw, R, ldr, work, lwork_bytes, true, stream);
}

extern "C" int evd_panel_qr_h(long m, long n, void* A, long lda, void* W, long ldw, void* R,
                              long ldr, void* work, long lwork_bytes, cudaStream_t stream) {
  return lp_panel(m, n, (__half*)A, lda, (__half*)W, ldw, (__half*)R, ldr, work, lwork_bytes,
                  true, stream);
}

extern "C" int evd_tsqr_s(long m, long n, float* A, long lda, float* R, long ldr, void* work,
                          long lwork_bytes, cudaStream_t stream) {
  return lp_panel(m, n, A, lda, (float*)nullptr, 0, R, ldr, work, lwork_bytes, false, stream);
}

extern "C" int evd_tsqr_h(long m, long n, void* A, long lda, void* R, long ldr, void* work,
                          long lwork_bytes, cudaStream_t stream) {
  return lp_panel(m, n, (__half*)A, lda, (__half*)nullptr, 0, (__half*)R, ldr, work, lwork_bytes,
                  false, stream);
}

extern "C" int evd_syr2k_lower_s(long n, long k, float alpha, const float* A, long lda,
                                 const float* B, long ldb, float beta, float* C, long ldc, long nb,
                                 cudaStream_t stream) {
  (void)nb;
  if (!evd::syr2k_args_ok(n, k, A, lda, B, ldb, C, ldc)) return EVD_ERR_INVALID_ARG;
  if (n == 0) return EVD_SUCCESS;
  if (k == 0 || alpha == 0.0f) return evd::scale_lower(n, beta, C, ldc, stream);
  const long T = (n + evd::kSB - 1) / evd::kSB;
  evd::ssyr2k_kernel<<<(unsigned)(T * (T + 1) / 2), 256, 0, stream>>>(n, k, alpha, A, lda, B, ldb,
                                                                     beta, C, ldc);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

extern "C" int evd_tc_syr2k(long n, long k, float alpha, const float* A, long lda, const float* B,
                            long ldb, float beta, float* C, long ldc, void* hwork, long nb,
                            cudaStream_t stream) {
  (void)nb;
  if (!evd::syr2k_args_ok(n, k, A, lda, B, ldb, C, ldc)) return EVD_ERR_INVALID_ARG;
  if (n == 0) return EVD_SUCCESS;
  if (k == 0 || alpha == 0.0f) return evd::scale_lower(n, beta, C, ldc, stream);
  // the reference's FP16 workspace (2 n k halves) holds the packed operands
  // when k % 64 == 0; otherwise (or without one) a stream-ordered buffer does
  const bool own = hwork == nullptr || k % 64 != 0 || ((uintptr_t)hwork & 15) != 0;
  return evd::tc_syr2k_run(n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                           own ? nullptr : (__half*)hwork, stream);
}

extern "C" int evd_syr2k_lower_h(long n, long k, float alpha, const void* A, long lda,
                                 const void* B, long ldb, float beta, void* C, long ldc, long nb,
                                 cudaStream_t stream) {
  (void)nb;
  if (!evd::syr2k_args_ok(n, k, A, lda, B, ldb, C, ldc)) return EVD_ERR_INVALID_ARG;
  if (n == 0) return EVD_SUCCESS;
  if (k == 0 || alpha == 0.0f) return evd::scale_lower(n, beta, (__half*)C, ldc, stream);
  return evd::tc_syr2k_run(n, k, alpha, (const __half*)A, lda, (const __half*)B, ldb, beta,
                           (__half*)C, ldc, nullptr, stream);
}
