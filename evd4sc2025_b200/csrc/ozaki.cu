// Emulated FP64 matrix products on the integer tensor cores (Ozaki scheme II:
// Ozaki, Uchino, Imamura, "Ozaki Scheme II: A GEMM-oriented emulation of
// floating-point matrix multiplication using an integer modular technique",
// 2025).  The reference has no counterpart: its products are cuBLAS DGEMMs
// (api/TCblas/tc_ozimmu_syr2k.cu:54-192 calls cublasDgemm), and this is the
// contraction that the mixed-precision solve and the eigenpair refinement run
// instead of FP64 DMMA.
//
// D = alpha * op(A) op(B) + beta * C + diag * I, with op(A) M x K, op(B) K x N:
//   1. every row i of op(A) is scaled by 2^e_i and rounded to an integer
//      vector a_i with ||a_i||_2 <= 2^P (likewise every column j of op(B) by
//      2^f_j to b_j), so |a_i . b_j| <= 2^2P < Mod / 2;
//   2. for each of N pairwise coprime moduli p_l <= 256 the residues
//      a mod p_l, b mod p_l (symmetric range, int8) are multiplied EXACTLY by
//      one tcgen05 kind::i8 GEMM with INT32 accumulation (|sum| <= K 2^14 <
//      2^31 for K < 2^17), and the epilogue stores (a . b) mod p_l as a byte;
//   3. the Chinese remainder theorem rebuilds a_i . b_j in (-Mod/2, Mod/2)
//      exactly (40-bit limbs held in doubles), which is converted to a double
//      and scaled back by 2^-(e_i + f_j).
// The only rounding is step 1: |D_ij - (op(A) op(B))_ij| <= ~ sqrt(K) 2^-P
// ||op(A)_i|| ||op(B)_j||.  14 moduli give P = 53 (FP64 inputs); fewer moduli
// trade accuracy for speed (P ~ 4 N - 2).
//
// The int8 GEMM (one persistent launch for all moduli): tiles of 128 x 256 as
// M128 N256 K32 tcgen05.mma into one of two 256-column INT32 accumulators in
// tensor memory; both operands K-major (rows of 128 bytes), brought in by TMA
// (cp.async.bulk.tensor, 128-byte swizzle, this GPU's own memory only, no
// multicast) through a 4-stage mbarrier ring.  One thread issues the copies,
// one thread the MMAs, and four warps drain the previous tile's accumulator
// (tcgen05.ld, Barrett reduction, byte stores) while the next tile is being
// multiplied.  Every wait is bounded (2 s) and reports EVD_ERR_TIMEOUT.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <math.h>

#include <mutex>

#include "common.cuh"
#include "ozaki.cuh"

namespace evd {
namespace {

// ------------------------------------------------------------------ moduli
// 256 and odd pairwise coprime numbers below it, largest first (their prime
// factors: 2; 3 5 17; 11 23; 251; 13 19; 241; 239; 233; 229; 227; 223; 7 31;
// 211; 199; 197; 193).
constexpr int kModTable[kOzMaxMod] = {256, 255, 253, 251, 247, 241, 239, 233,
                                      229, 227, 223, 217, 211, 199, 197, 193};

typedef unsigned __int128 u128;
constexpr u128 kLimbMask = ((u128)1 << 40) - 1;

// CRT constants are split into 40-bit limbs held exactly in doubles: a sum of
// up to 20 products (residue < 2^8) x (limb < 2^40) stays below 2^53.
constexpr int kOzLimbs = 4;  // Mod < 2^160 for 20 moduli
struct OzConsts {
  int nmod;
  int p[kOzMaxMod];
  unsigned magic[kOzMaxMod];   // floor(2^32 / p): Barrett quotient estimate
  int k16[kOzMaxMod], k32[kOzMaxMod], k48[kOzMaxMod];  // 2^16, 2^32, 2^48 mod p
  int nlimb;                   // 40-bit limbs needed for Mod (3 up to 15 moduli)
  double wl[kOzLimbs][kOzMaxMod];  // CRT weights (M / p) ((M / p)^-1 mod p), 40-bit limbs
  double ml[kOzLimbs];         // Mod, 40-bit limbs
  double Md;                   // Mod (rounded)
  double invM;                 // 1 / Mod
  int P;                       // bits of the integer operands (row norm <= 2^P)
};


// modular inverse of a mod p (p <= 256, gcd = 1), by search
int inv_mod(u128 a, int p) {
  const int r = (int)(a % (u128)p);
  for (int x = 1; x < p; ++x)
    if ((r * x) % p == 1) return x;
  return 0;
}

OzConsts make_consts(int nmod, long K) {
  OzConsts c{};
  c.nmod = nmod;
  u128 M = 1;
  for (int l = 0; l < nmod; ++l) M *= (u128)kModTable[l];
  for (int l = 0; l < nmod; ++l) {
    const int p = kModTable[l];
    c.p[l] = p;
    c.magic[l] = (unsigned)(((unsigned long long)1 << 32) / (unsigned long long)p);
    c.k16[l] = (int)((1ull << 16) % (unsigned long long)p);
    c.k32[l] = (int)((1ull << 32) % (unsigned long long)p);
    c.k48[l] = (int)((1ull << 48) % (unsigned long long)p);
    const u128 Mi = M / (u128)p;
    const u128 w = Mi * (u128)inv_mod(Mi, p);  // < M: (M/p) * (p - 1) < M < 2^126
    for (int i = 0; i < kOzLimbs; ++i) c.wl[i][l] = (double)((w >> (40 * i)) & kLimbMask);
  }
  for (int i = 0; i < kOzLimbs; ++i) c.ml[i] = (double)((M >> (40 * i)) & kLimbMask);
  c.nlimb = (M >> 120) == 0 ? 3 : 4;
  const long double Md =
      (long double)(unsigned long long)(M >> 64) * 18446744073709551616.0L +
      (long double)(unsigned long long)M;
  c.Md = (double)Md;
  c.invM = (double)(1.0L / Md);
  // largest P with (2^P + sqrt(K)/2)^2 < M/2 (the rounding of each element
  // adds at most 1/2, so a row's norm grows by at most sqrt(K)/2)
  const long double lim = sqrtl(Md / 2.0L) * (1.0L - 1e-12L) - sqrtl((long double)K) / 2.0L;
  int P = (int)floorl(log2l(lim));
  c.P = std::min(P, 53);
  return c;
}

// -------------------------------------------------------------- utilities
constexpr unsigned long long kOzWaitNs = 2000000000ull;

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
// bounded wait for phase `parity`; false (error recorded) after kOzWaitNs
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  for (unsigned it = 0;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63u) == 63u && gtimer() - t0 > kOzWaitNs) {
      atomicExch(err, kDevTimeoutTree);
      return false;
    }
  }
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// 3-D tiled TMA load (x = K byte offset, y = row, z = modulus plane) into this
// CTA's shared memory; completion counted on `bar`
__device__ __forceinline__ void tma_load3(void* dst, const CUtensorMap* map, int x, int y, int z,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  // start >> 4 | LBO 16 B (unused for swizzled K-major) | SBO 1024 B (8-row
  // groups) | version 1 | base offset 0 | SWIZZLE_128B
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

// kind::i8 instruction descriptor: D S32 (bits 4-5 = 2), A S8 (bits 7-9 = 1),
// B S8 (bits 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at 24-28
constexpr int kOzMmaM = 128, kOzMmaN = 256;
constexpr uint32_t kOzIdesc = (2u << 4) | (1u << 7) | (1u << 10) |
                              ((uint32_t)(kOzMmaN >> 3) << 17) | ((uint32_t)(kOzMmaM >> 4) << 24);

__device__ __forceinline__ void umma_i8(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(da), "l"(db), "r"(kOzIdesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// ----------------------------------------------------------- int8 GEMM
// Persistent, warp-specialised: one CTA per SM walks the tiles t = blockIdx.x,
// + gridDim.x, ... (modulus-major).  Warp 0 lane 0 issues the TMA copies of a
// 4-stage (lean: 2-stage) shared-memory ring, warp 1 lane 0 issues the MMAs
// into one of two 256-column INT32 accumulators in tensor memory (tile t into
// buffer t & 1), and warps 2-5 drain the other buffer (tcgen05.ld, Barrett
// reduction, byte stores) while the next tile is being multiplied.
constexpr int kPM = 128, kPN = 256, kPK = 128;   // tile rows, columns, K bytes per stage
constexpr uint32_t kPTileA = kPM * kPK;          // 16 KB
constexpr uint32_t kPTileB = kPN * kPK;          // 32 KB
constexpr uint32_t kPStage = kPTileA + kPTileB;  // 48 KB
constexpr int kPThreads = 192;
constexpr int kOzGroup = 8;                      // tile rows per rasterisation group (L2 reuse)
// 4 stages (193 KB) normally; 2 stages (97 KB) leave room for another
// kernel's CTA on the same SM (the bulge chase, 33 KB, runs beside the
// products that overlap it)
constexpr int oz_smem(int stages) { return stages * (int)kPStage + 1024 + 256; }

struct OzGemmArgs {
  long M, N, K;
  int tiles_m, tiles_n;
  int lower;           // only tiles that meet the lower triangle (row >= column)
  int nmod;
  long tiles_per_mod;
  uint8_t* R;          // residue planes: R[l * plane + m + n * ldr]
  long ldr, plane;
  int p[kOzMaxMod];
  unsigned magic[kOzMaxMod];
  int* err;
};

// tile index inside one modulus plane -> (tile row, tile column)
__device__ __forceinline__ void tile_coords(const OzGemmArgs& a, long t, int& bm, int& bn) {
  if (a.lower) {
    // column-block bn holds tile rows 2 bn .. tiles_m - 1 (rows of 128 meet
    // columns of 256 at or below the diagonal)
    int c = 0;
    for (;; ++c) {
      const long cnt = a.tiles_m - 2L * c;
      if (t < cnt) break;
      t -= cnt;
    }
    bn = c;
    bm = 2 * c + (int)t;
    return;
  }
  // groups of kOzGroup tile rows, column-major inside a group
  const long per = (long)kOzGroup * a.tiles_n;
  const long g = t / per, r = t % per;
  const long left = a.tiles_m - g * kOzGroup;
  const int rows = (int)(left < kOzGroup ? left : kOzGroup);
  bm = (int)(g * kOzGroup + r % rows);
  bn = (int)(r / rows);
}

__device__ __forceinline__ void mbar_arrive_cta(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

template <int STAGES>
__global__ void __launch_bounds__(kPThreads, 1)
    oz_imma_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                   const OzGemmArgs a) {
  extern __shared__ __align__(1024) uint8_t osm[];
  uint8_t* stages = osm + ((1024u - (smem_u32(osm) & 1023u)) & 1023u);
  uint64_t* full = reinterpret_cast<uint64_t*>(stages + STAGES * kPStage);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;
  uint64_t* tempty = tfull + 2;
  uint64_t* done = tempty + 2;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long nk = (a.K + kPK - 1) / kPK;
  const long total = a.tiles_per_mod * a.nmod;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull + b, 1);
      mbar_init(tempty + b, 128);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapB)) : "memory");
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
      for (long t = blockIdx.x; t < total && ok; t += gridDim.x) {
        const int l = (int)(t / a.tiles_per_mod);
        int bm, bn;
        tile_coords(a, t % a.tiles_per_mod, bm, bn);
        for (long kb = 0; kb < nk; ++kb, ++gk) {
          const int s = (int)(gk % STAGES);
          if (gk >= STAGES &&
              !mbar_wait(empty + s, (uint32_t)((gk / STAGES - 1) & 1), a.err)) {
            ok = false;
            break;
          }
          uint8_t* sa = stages + s * kPStage;
          mbar_expect_tx(full + s, kPStage);
          tma_load3(sa, &mapA, (int)(kb * kPK), bm * kPM, l, full + s);
          tma_load3(sa + kPTileA, &mapB, (int)(kb * kPK), bn * kPN, l, full + s);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer ----
      long gk = 0;
      int i = 0;
      bool ok = true;
      for (long t = blockIdx.x; t < total && ok; t += gridDim.x, ++i) {
        const int b = i & 1;
        if (i >= 2 && !mbar_wait(tempty + b, (uint32_t)(((i >> 1) - 1) & 1), a.err)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc_tm = tmem + (uint32_t)(b * kPN);
        for (long kb = 0; kb < nk; ++kb, ++gk) {
          const int s = (int)(gk % STAGES);
          if (!mbar_wait(full + s, (uint32_t)((gk / STAGES) & 1), a.err)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sa = smem_u32(stages + s * kPStage);
          const uint32_t sb = sa + kPTileA;
#pragma unroll
          for (int ks = 0; ks < kPK / 32; ++ks)
            umma_i8(acc_tm, smem_desc_sw128(sa + ks * 32), smem_desc_sw128(sb + ks * 32),
                    (kb > 0 || ks > 0) ? 1u : 0u);
          umma_commit(empty + s);
        }
        if (ok) umma_commit(tfull + b);
      }
      umma_commit(done);  // fires when every MMA issued above has completed
      mbar_wait(done, 0, a.err);
    }
  } else {  // ---- epilogue: warps 2-5, TMEM lanes 32 (warp % 4) .. + 31 ----
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    int i = 0;
    for (long t = blockIdx.x; t < total; t += gridDim.x, ++i) {
      const int b = i & 1;
      if (!mbar_wait(tfull + b, (uint32_t)((i >> 1) & 1), a.err)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int l = (int)(t / a.tiles_per_mod);
      int bm, bn;
      tile_coords(a, t % a.tiles_per_mod, bm, bn);
      const int p = a.p[l];
      const unsigned magic = a.magic[l];
      // |acc| <= K 2^14 <= 2^30 < p 2^23 (K <= 2^16, p >= 193): acc + off is in
      // [0, 2^32) and congruent to acc mod p
      const unsigned off = (unsigned)p << 23;
      uint8_t* R = a.R + (long)l * a.plane;
      const long gm = (long)bm * kPM + row;
      const long n0 = (long)bn * kPN;
      // 64 columns per wait: four x16 loads in flight, then the reductions
#pragma unroll 1
      for (int c0 = 0; c0 < kPN; c0 += 64) {
        uint32_t v[64];
        const uint32_t addr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * kPN + c0);
#pragma unroll
        for (int h = 0; h < 4; ++h)
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
        if (gm < a.M) {
          uint8_t* dst = R + gm + (n0 + c0) * a.ldr;
          const long left = a.N - (n0 + c0);
          const unsigned ldr = (unsigned)a.ldr;  // a plane is < 2^32 bytes
          if (left >= 64) {
            unsigned o = 0;
#pragma unroll
            for (int j = 0; j < 64; ++j, o += ldr) {
              const unsigned x = v[j] + off;
              unsigned r = x - __umulhi(x, magic) * (unsigned)p;  // in [0, 2p)
              r = (r >= (unsigned)p) ? r - (unsigned)p : r;
              dst[o] = (uint8_t)r;
            }
          } else {
            for (int j = 0; j < (int)left; ++j) {
              const unsigned x = v[j] + off;
              unsigned r = x - __umulhi(x, magic) * (unsigned)p;
              r = (r >= (unsigned)p) ? r - (unsigned)p : r;
              dst[(long)j * a.ldr] = (uint8_t)r;
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive_cta(tempty + b);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// ------------------------------------------------------------ quantisation
// Row r of the operand = column r of S (K contiguous): 2-norm, exponent
// e_r = P - ceil(log2 ||row||) (0 for a zero row), integers rint(S 2^e_r) and
// their residues mod every p_l (symmetric range) as int8 into
// Q[l * plane + r * ldq + k].  One block per row, 4 elements per thread.
__global__ void oz_quant_kernel(long rows, long K, const double* __restrict__ S, long lds,
                                int8_t* __restrict__ Q, long ldq, long plane, int* __restrict__ ex,
                                const OzConsts c) {
  __shared__ double red[32];
  __shared__ double sscale;
  for (long r = blockIdx.x; r < rows; r += gridDim.x) {
    const double* col = S + r * lds;
    double ss = 0.0;
    for (long k = threadIdx.x; k < K; k += blockDim.x) ss = fma(col[k], col[k], ss);
    ss = warp_sum(ss);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
      int e = 0;
      if (t > 0.0) {
        int E;
        frexp(sqrt(t), &E);  // ||row|| < 2^E
        e = c.P - E;
      }
      ex[r] = e;
      sscale = ldexp(1.0, e);
    }
    __syncthreads();
    const double scale = sscale;
    for (long k0 = 4 * (long)threadIdx.x; k0 < K; k0 += 4 * (long)blockDim.x) {
      // the integers |v| <= 2^53 as 16-bit limbs d3 2^48 + d2 2^32 + d1 2^16 +
      // d0 (d3 signed): v mod p = (d3 k48 + d2 k32 + d1 k16 + d0) mod p in
      // 32-bit integers, reduced by a Barrett step
      int d0[4], d1[4], d2[4], d3[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const long long t =
            (k0 + q < K) ? (long long)rint(col[k0 + q] * scale) : 0LL;
        d0[q] = (int)(t & 0xFFFF);
        d1[q] = (int)((t >> 16) & 0xFFFF);
        d2[q] = (int)((t >> 32) & 0xFFFF);
        d3[q] = (int)(t >> 48);
      }
      for (int li = 0; li < c.nmod; ++li) {
        const int p = c.p[li];
        const unsigned magic = c.magic[li];
        const int half = (p + 1) >> 1;
        const int off = p << 17;  // > 32 * 255 = max |d3 k48|: keeps the sum positive
        char4 o;
        int8_t* ob = reinterpret_cast<int8_t*>(&o);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const unsigned x =
              (unsigned)(d0[q] + off + d1[q] * c.k16[li] + d2[q] * c.k32[li] + d3[q] * c.k48[li]);
          int ri = (int)(x - __umulhi(x, magic) * (unsigned)p);  // in [0, 2p)
          if (ri >= p) ri -= p;
          if (ri >= half) ri -= p;
          ob[q] = (int8_t)ri;
        }
        int8_t* dst = Q + (long)li * plane + r * ldq + k0;
        if (k0 + 3 < K) {
          *reinterpret_cast<char4*>(dst) = o;
        } else {
          for (int q = 0; q < 4 && k0 + q < K; ++q) dst[q] = ob[q];
        }
      }
    }
    __syncthreads();  // red / sscale reused by the next row
  }
}

// B = A^T (FP64, column-major, m x n -> n x m), 32 x 32 tiles
__global__ void oz_transpose_kernel(long m, long n, const double* __restrict__ A, long lda,
                                    double* __restrict__ B, long ldb) {
  __shared__ double t[32][33];
  const long i0 = (long)blockIdx.x * 32, j0 = (long)blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const long i = i0 + threadIdx.x, j = j0 + r;
    t[r][threadIdx.x] = (i < m && j < n) ? A[i + j * lda] : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const long j = j0 + threadIdx.x, i = i0 + r;  // B(j, i) = A(i, j)
    if (i < m && j < n) B[j + i * ldb] = t[threadIdx.x][r];
  }
}

// --------------------------------------------------------------- CRT
// Limb arithmetic of the reconstruction: a value is x3 2^120 + x2 2^80 +
// x1 2^40 + x0 with every limb an integer held exactly in a double.
// canonical: x0, x1, x2 in [0, 2^40), the sign in x3
__device__ __forceinline__ void limbs_canon(double (&x)[kOzLimbs]) {
#pragma unroll
  for (int i = 0; i < kOzLimbs - 1; ++i) {
    const double c = floor(x[i] * 0x1p-40);
    x[i] = fma(-c, 0x1p40, x[i]);
    x[i + 1] += c;
  }
}
__device__ __forceinline__ double limbs_value(const double (&x)[kOzLimbs]) {
  return fma(x[3], 0x1p120, fma(x[2], 0x1p80, fma(x[1], 0x1p40, x[0])));
}

// The integer in (-Mod/2, Mod/2) with given residues, as a double: from the
// limb sums S = sum_l r_l w_l (exact), X = S - q Mod with q from a rounded
// quotient, then the representative nearest zero (the product's bound keeps
// the true value within Mod/4, far from the decision points), then the
// magnitude's limbs summed from the top limb down (each step one rounding).
// X = sum_l r_l w_l (limb sums, exact) -> the representative in
// (-Mod/2, Mod/2) as a double
__device__ __forceinline__ double crt_finish(double (&x)[kOzLimbs], const OzConsts& c) {
  const double q = floor(limbs_value(x) * c.invM);
#pragma unroll
  for (int i = 0; i < kOzLimbs; ++i) x[i] = fma(-q, c.ml[i], x[i]);
  limbs_canon(x);
  // X = v + k Mod with k in {-1, 0, 1, 2} and |v| < Mod/4: k = rint(X / Mod)
  const double k = rint(limbs_value(x) * c.invM);
  if (k != 0.0) {
#pragma unroll
    for (int i = 0; i < kOzLimbs; ++i) x[i] = fma(-k, c.ml[i], x[i]);
    limbs_canon(x);
  }
  const bool neg = x[3] < 0.0;
  if (neg) {
#pragma unroll
    for (int i = 0; i < kOzLimbs; ++i) x[i] = -x[i];
    limbs_canon(x);
  }
  const double mag = fma(x[3], 0x1p120, fma(x[2], 0x1p80, fma(x[1], 0x1p40, x[0])));
  return neg ? -mag : mag;
}

// D(m, n) = alpha 2^-(ea_m + eb_n) crt(m, n) + beta C(m, n) + diag [m == n].
// lower: only m >= n is rebuilt and D(n, m) receives the same value (a
// symmetric product).  Tiles of 128 rows x 32 columns, 256 threads: thread
// (g = t % 32, c = t / 32) rebuilds rows 4g..4g+3 of columns c, c+8, c+16,
// c+24 (one 4-byte load per modulus and column); the mirrored writes go
// through shared memory so that both stores are coalesced.
constexpr int kCrtRows = 128, kCrtCols = 32;
template <int NL>
__global__ void __launch_bounds__(256)
    oz_crt_kernel(long M, long N, const uint8_t* __restrict__ R, long ldr, long plane,
                  const int* __restrict__ ea, const int* __restrict__ eb, double alpha,
                  double beta, const double* C, long ldc, double diag, double* D, long ldd,
                  int lower, const OzConsts c) {
  __shared__ double t[kCrtCols][kCrtRows + 1];
  const long i0 = (long)blockIdx.x * kCrtRows, j0 = (long)blockIdx.y * kCrtCols;
  if (lower && j0 >= i0 + kCrtRows) return;  // the tile lies above the diagonal
  const int g = threadIdx.x & 31, cc = threadIdx.x >> 5;
  const long ib = i0 + 4 * g;
  const bool full4 = ib + 3 < M && (ldr & 3) == 0;
#pragma unroll 1
  for (int q = 0; q < 4; ++q) {
    const int cl = cc + 8 * q;
    const long j = j0 + cl;
    double out[4] = {0.0, 0.0, 0.0, 0.0};
    if (j < N && (!lower || ib + 3 >= j)) {
      // residues of the 4 rows, modulus by modulus
      double x[4][kOzLimbs];
#pragma unroll
      for (int e = 0; e < 4; ++e)
#pragma unroll
        for (int i = 0; i < kOzLimbs; ++i) x[e][i] = 0.0;
      const uint8_t* base = R + ib + j * ldr;
      // all residue words first (loads in flight together), then the sums
      uint32_t w4[kOzMaxMod];
#pragma unroll
      for (int li = 0; li < kOzMaxMod; ++li) {
        w4[li] = 0;
        if (li < c.nmod) {
          if (full4) {
            w4[li] = __ldg(reinterpret_cast<const uint32_t*>(base + li * plane));
          } else {
            for (int e = 0; e < 4; ++e)
              if (ib + e < M) w4[li] |= (uint32_t)base[li * plane + e] << (8 * e);
          }
        }
      }
#pragma unroll
      for (int li = 0; li < kOzMaxMod; ++li) {
        if (li < c.nmod) {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            // byte -> double without a conversion instruction: 2^52 + r as bits
            const double r = __hiloint2double(0x43300000, (int)((w4[li] >> (8 * e)) & 0xFFu)) -
                             4503599627370496.0;
#pragma unroll
            for (int i = 0; i < NL; ++i) x[e][i] = fma(r, c.wl[i][li], x[e][i]);
          }
        }
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const long i = ib + e;
        if (i < M && (!lower || i >= j)) {
          const double v = crt_finish(x[e], c);
          double o = alpha * ldexp(v, -(ea[i] + eb[j]));
          if (beta != 0.0) o = fma(beta, C[i + j * ldc], o);
          if (i == j) o += diag;
          D[i + j * ldd] = o;
          out[e] = o;
        }
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) t[cl][4 * g + e] = out[e];
  }
  if (!lower) return;
  __syncthreads();
  // mirror: D(j, i) = D(i, j) for i > j; a warp writes 32 consecutive j of one i
  for (int r = threadIdx.x >> 5; r < kCrtRows; r += 8) {
    const long i = i0 + r, j = j0 + (threadIdx.x & 31);
    if (i < M && j < N && i > j) D[j + i * ldd] = t[threadIdx.x & 31][r];
  }
}

// D = beta C + diag I (the product vanishes); lower: both triangles from C's lower
__global__ void oz_axpby_kernel(long M, long N, double beta, const double* C, long ldc, double diag,
                                double* D, long ldd, int lower) {
  const long i = (long)blockIdx.x * 32 + threadIdx.x;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const long j = (long)blockIdx.y * 32 + r;
    if (i >= M || j >= N) continue;
    const long si = (lower && i < j) ? j : i, sj = (lower && i < j) ? i : j;
    double v = beta != 0.0 ? beta * C[si + sj * ldc] : 0.0;
    if (i == j) v += diag;
    D[i + j * ldd] = v;
  }
}

// ------------------------------------------------------------ host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// planes of int8 rows (K bytes used of ld), `rows` rows per plane, nmod planes
int make_plane_map(CUtensorMap* map, const int8_t* base, long rows, long K, long ld, long plane,
                   int nmod, int box_rows) {
  auto enc = encode_fn();
  if (!enc) return EVD_ERR_CUDA;
  cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)nmod};
  cuuint64_t strides[2] = {(cuuint64_t)ld, (cuuint64_t)plane};
  cuuint32_t box[3] = {(cuuint32_t)kPK, (cuuint32_t)box_rows, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void*)base, dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? EVD_SUCCESS : EVD_ERR_CUDA;
}

}  // namespace

int tma_map_rows16(CUtensorMap* map, const void* base, long rows, long elems, long ld,
                   int box_rows) {
  auto enc = encode_fn();
  if (!enc) return EVD_ERR_CUDA;
  cuuint64_t dims[2] = {(cuuint64_t)elems, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base), dims,
                   strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? EVD_SUCCESS : EVD_ERR_CUDA;
}

namespace {

int* oz_err_word() {
  static int* words[64] = {nullptr};
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) return nullptr;
  if (!words[d]) {
    int* p = nullptr;
    if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
    if (cudaMemset(p, 0, sizeof(int)) != cudaSuccess) return nullptr;
    words[d] = p;
  }
  return words[d];
}

long al256(long x) { return (x + 255) / 256 * 256; }

}  // namespace

long oz_ld(long K) { return (K + 127) / 128 * 128; }

OzLayout oz_layout(long M, long N, long K, int nmod, bool need_transpose) {
  OzLayout L{};
  const long ldq = oz_ld(K);
  const long ldr = (M + 15) / 16 * 16;
  long o = 0;
  L.qa = o; o = al256(o + (long)nmod * M * ldq);
  L.qb = o; o = al256(o + (long)nmod * N * ldq);
  L.res = o; o = al256(o + (long)nmod * ldr * N);
  L.ea = o; o = al256(o + 4 * M);
  L.eb = o; o = al256(o + 4 * N);
  L.tr = o; o = al256(o + (need_transpose ? 8 * std::max(M, N) * K : 0));
  L.bytes = o + 256;
  return L;
}

int oz_quantize(long rows, long K, const double* S, long lds, int8_t* Q, int* ex, int nmod,
                cudaStream_t st) {
  if (rows <= 0 || K <= 0) return EVD_SUCCESS;
  const OzConsts c = make_consts(nmod, K);
  const long ldq = oz_ld(K);
  const long plane = rows * ldq;
  const int blocks = (int)std::min<long>(rows, 8L * device_sm_count());
  oz_quant_kernel<<<blocks, 256, 0, st>>>(rows, K, S, lds, Q, ldq, plane, ex, c);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

int oz_transpose(long m, long n, const double* A, long lda, double* B, long ldb,
                 cudaStream_t st) {
  if (m <= 0 || n <= 0) return EVD_SUCCESS;
  oz_transpose_kernel<<<dim3(ceil_div_i(m, 32), ceil_div_i(n, 32)), dim3(32, 8), 0, st>>>(
      m, n, A, lda, B, ldb);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

int oz_imma(long M, long N, long K, const int8_t* QA, const int8_t* QB, uint8_t* Rz, int nmod,
            bool lower, cudaStream_t st, bool lean) {
  if (M <= 0 || N <= 0) return EVD_SUCCESS;
  if (K <= 0 || K > kOzMaxK) return EVD_ERR_INVALID_ARG;  // INT32 accumulation bound
  const long ldq = oz_ld(K);
  CUtensorMap ma, mb;
  EVD_TRY(make_plane_map(&ma, QA, M, K, ldq, M * ldq, nmod, kPM));
  EVD_TRY(make_plane_map(&mb, QB, N, K, ldq, N * ldq, nmod, kPN));
  const OzConsts c = make_consts(nmod, K);
  OzGemmArgs a{};
  a.M = M; a.N = N; a.K = K;
  a.tiles_m = ceil_div_i(M, kPM);
  a.tiles_n = ceil_div_i(N, kPN);
  a.lower = lower ? 1 : 0;
  a.nmod = nmod;
  a.R = Rz;
  a.ldr = (M + 15) / 16 * 16;
  a.plane = a.ldr * N;
  for (int l = 0; l < nmod; ++l) {
    a.p[l] = c.p[l];
    a.magic[l] = c.magic[l];
  }
  a.err = oz_err_word();
  if (!a.err) return EVD_ERR_CUDA;
  long tiles = 0;
  if (lower) {
    for (long bn = 0; 2 * bn < a.tiles_m; ++bn) tiles += a.tiles_m - 2 * bn;
  } else {
    tiles = (long)a.tiles_m * a.tiles_n;
  }
  a.tiles_per_mod = tiles;
  const long total = tiles * nmod;
  const int grid = (int)std::min<long>(total, device_sm_count());
  if (lean) {
    EVD_TRY(smem_attr_once((const void*)oz_imma_kernel<2>, oz_smem(2)));
    oz_imma_kernel<2><<<grid, kPThreads, oz_smem(2), st>>>(ma, mb, a);
  } else {
    EVD_TRY(smem_attr_once((const void*)oz_imma_kernel<4>, oz_smem(4)));
    oz_imma_kernel<4><<<grid, kPThreads, oz_smem(4), st>>>(ma, mb, a);
  }
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

int oz_crt(long M, long N, long K, const uint8_t* Rz, const int* ea, const int* eb, int nmod,
           double alpha, double beta, const double* C, long ldc, double diag, double* D, long ldd,
           bool lower, cudaStream_t st) {
  if (M <= 0 || N <= 0) return EVD_SUCCESS;
  const OzConsts c = make_consts(nmod, K);
  const long ldr = (M + 15) / 16 * 16;
  const dim3 grid(ceil_div_i(M, kCrtRows), ceil_div_i(N, kCrtCols));
  if (c.nlimb == 3)
    oz_crt_kernel<3><<<grid, 256, 0, st>>>(M, N, Rz, ldr, ldr * N, ea, eb, alpha, beta, C, ldc,
                                           diag, D, ldd, lower ? 1 : 0, c);
  else
    oz_crt_kernel<4><<<grid, 256, 0, st>>>(M, N, Rz, ldr, ldr * N, ea, eb, alpha, beta, C, ldc,
                                           diag, D, ldd, lower ? 1 : 0, c);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

int oz_check_err(cudaStream_t st) {
  int* err = oz_err_word();
  if (!err) return EVD_ERR_CUDA;
  return read_device_error(err, st);
}

int oz_gemm(char ta, char tb, long M, long N, long K, double alpha, const double* A, long lda,
            const double* B, long ldb, double beta, const double* C, long ldc, double diag,
            double* D, long ldd, int nmod, bool lower, void* work, long lwork, cudaStream_t st,
            bool lean) {
  ta = (char)(ta | 0x20);
  tb = (char)(tb | 0x20);
  if ((ta != 'n' && ta != 't') || (tb != 'n' && tb != 't')) return EVD_ERR_INVALID_ARG;
  if (M < 0 || N < 0 || K < 0 || nmod < kOzMinMod || nmod > kOzMaxMod) return EVD_ERR_INVALID_ARG;
  if (lower && M != N) return EVD_ERR_INVALID_ARG;
  if (M == 0 || N == 0) return EVD_SUCCESS;
  if (!D || ldd < M || (beta != 0.0 && (!C || ldc < M))) return EVD_ERR_INVALID_ARG;
  if (K == 0 || alpha == 0.0) {  // D = beta C + diag I
    oz_axpby_kernel<<<dim3(ceil_div_i(M, 32), ceil_div_i(N, 32)), dim3(32, 8), 0, st>>>(
        M, N, beta, C, ldc, diag, D, ldd, lower ? 1 : 0);
    EVD_LAUNCHED();
    return EVD_SUCCESS;
  }
  if (!A || !B || K > kOzMaxK) return EVD_ERR_INVALID_ARG;
  if (lda < (ta == 't' ? K : M) || ldb < (tb == 't' ? N : K)) return EVD_ERR_INVALID_ARG;
  const bool need_tr = (ta == 'n') || (tb == 't');
  const OzLayout L = oz_layout(M, N, K, nmod, need_tr);
  if (!work || lwork < L.bytes) return EVD_ERR_WORKSPACE;
  uint8_t* base = reinterpret_cast<uint8_t*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
  int8_t* qa = reinterpret_cast<int8_t*>(base + L.qa);
  int8_t* qb = reinterpret_cast<int8_t*>(base + L.qb);
  uint8_t* rz = base + L.res;
  int* ea = reinterpret_cast<int*>(base + L.ea);
  int* eb = reinterpret_cast<int*>(base + L.eb);
  double* tr = reinterpret_cast<double*>(base + L.tr);
  // rows of op(A) with K contiguous: columns of A when ta == 't', else of A^T
  if (ta == 't') {
    EVD_TRY(oz_quantize(M, K, A, lda, qa, ea, nmod, st));
  } else {
    EVD_TRY(oz_transpose(M, K, A, lda, tr, K, st));
    EVD_TRY(oz_quantize(M, K, tr, K, qa, ea, nmod, st));
  }
  // columns of op(B) with K contiguous: columns of B when tb == 'n'
  if (tb == 'n') {
    EVD_TRY(oz_quantize(N, K, B, ldb, qb, eb, nmod, st));
  } else {
    EVD_TRY(oz_transpose(N, K, B, ldb, tr, K, st));
    EVD_TRY(oz_quantize(N, K, tr, K, qb, eb, nmod, st));
  }
  EVD_TRY(oz_imma(M, N, K, qa, qb, rz, nmod, lower, st, lean));
  EVD_TRY(oz_crt(M, N, K, rz, ea, eb, nmod, alpha, beta, C, ldc, diag, D, ldd, lower, st));
  return EVD_SUCCESS;
}

// C(lower, mirrored) = alpha (Y Z^T + Z Y^T) + beta C as ONE emulated product
// [Y | Z] [Z | Y]^T (K = 2k): the rows of both operands are rows of Y and Z,
// brought K-contiguous by transposes into the workspace.
long oz_syr2k_ws_bytes(long n, long k, int nmod) {
  const long K = 2 * k;
  const long ldq = oz_ld(K);
  long o = 0;
  o = al256(o + 8 * K * n);                           // [Y | Z]^T
  o = al256(o + 8 * K * n);                           // [Z | Y]^T
  o = al256(o + (long)nmod * n * ldq);                // qa
  o = al256(o + (long)nmod * n * ldq);                // qb
  o = al256(o + (long)nmod * ((n + 15) / 16 * 16) * n);  // residues
  o = al256(o + 4 * n);
  o = al256(o + 4 * n);
  return o + 256;
}

int oz_syr2k_lower(long n, long k, double alpha, const double* Y, long ldy, const double* Z,
                   long ldz, double beta, double* C, long ldc, int nmod, void* work, long lwork,
                   cudaStream_t st) {
  if (n <= 0) return EVD_SUCCESS;
  if (k <= 0 || 2 * k > kOzMaxK || nmod < kOzMinMod || nmod > kOzMaxMod)
    return EVD_ERR_INVALID_ARG;
  if (lwork < oz_syr2k_ws_bytes(n, k, nmod)) return EVD_ERR_WORKSPACE;
  const long K = 2 * k;
  const long ldq = oz_ld(K);
  uint8_t* b = reinterpret_cast<uint8_t*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
  long o = 0;
  double* t1 = reinterpret_cast<double*>(b + o); o = al256(o + 8 * K * n);
  double* t2 = reinterpret_cast<double*>(b + o); o = al256(o + 8 * K * n);
  int8_t* qa = reinterpret_cast<int8_t*>(b + o); o = al256(o + (long)nmod * n * ldq);
  int8_t* qb = reinterpret_cast<int8_t*>(b + o); o = al256(o + (long)nmod * n * ldq);
  uint8_t* rz = b + o; o = al256(o + (long)nmod * ((n + 15) / 16 * 16) * n);
  int* ea = reinterpret_cast<int*>(b + o); o = al256(o + 4 * n);
  int* eb = reinterpret_cast<int*>(b + o);
  EVD_TRY(oz_transpose(n, k, Y, ldy, t1, K, st));
  EVD_TRY(oz_transpose(n, k, Z, ldz, t1 + k, K, st));
  EVD_TRY(oz_transpose(n, k, Z, ldz, t2, K, st));
  EVD_TRY(oz_transpose(n, k, Y, ldy, t2 + k, K, st));
  EVD_TRY(oz_quantize(n, K, t1, K, qa, ea, nmod, st));
  EVD_TRY(oz_quantize(n, K, t2, K, qb, eb, nmod, st));
  EVD_TRY(oz_imma(n, n, K, qa, qb, rz, nmod, true, st));
  EVD_TRY(oz_crt(n, n, K, rz, ea, eb, nmod, alpha, beta, C, ldc, 0.0, C, ldc, true, st));
  return EVD_SUCCESS;
}

int oz_bits(int nmod, long K) {
  if (nmod < kOzMinMod || nmod > kOzMaxMod || K <= 0) return 0;
  return make_consts(nmod, K).P;
}

}  // namespace evd

extern "C" long evd_dgemm_ozaki_work_size(char transa, char transb, long m, long n, long k,
                                          int moduli) {
  if (m < 0 || n < 0 || k < 0 || moduli < evd::kOzMinMod || moduli > evd::kOzMaxMod) return 0;
  const char ta = (char)(transa | 0x20), tb = (char)(transb | 0x20);
  return evd::oz_layout(m, n, k, moduli, ta == 'n' || tb == 't').bytes;
}

extern "C" int evd_dgemm_ozaki(char transa, char transb, long m, long n, long k, double alpha,
                               const double* A, long lda, const double* B, long ldb, double beta,
                               double* C, long ldc, int moduli, void* work, long lwork,
                               cudaStream_t stream) {
  try {
    EVD_TRY(evd::oz_gemm(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 0.0, C,
                         ldc, moduli, false, work, lwork, stream));
    return evd::oz_check_err(stream);
  } catch (...) {
    return EVD_ERR_HOST;
  }
}

extern "C" int evd_ozaki_bits(int moduli, long k) { return evd::oz_bits(moduli, k); }
