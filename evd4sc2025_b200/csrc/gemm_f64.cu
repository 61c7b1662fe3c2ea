// FP64 GEMM / SYR2K on the B200 FP64 tensor path (DMMA, mma.sync m8n8k4 f64).
//
// sm_100a has no FP64 kind for tcgen05.mma, so the FP64-accurate contractions
// of the eigensolver (the reference's CUBLAS_COMPUTE_64F GemmEx/Dgemm/Dsyr2k
// calls, e.g. api/zy_zy_sy2sb.cu:134-394, api/TCblas/tc_ozimmu_syr2k.cu:209-341,
// src/EVD/myEVD.cu:151-232) run on DMMA: 8x8x4 FP64 MMAs issued by every warp,
// operands staged in shared memory by a multi-stage cp.async pipeline.
//
// Layouts: column-major A (m x k, or k x m when transposed), B (k x n, or
// n x k when transposed), C (m x n).  Shared-memory tiles keep the global
// contiguous dimension contiguous and are padded by 4 doubles per row so that
// the m8n8k4 fragment loads (row = lane/4, k = lane%4) are bank-conflict free.
//
// Modes:
//   kGemm      C = alpha*op(A)*op(B) + beta*C (strided batched over grid.y)
//   kSyr2kLow  lower-triangular tiles only, K split in two operand pairs
//              (A,B) for k < k1 and (A2,B2) beyond; the epilogue writes the
//              lower triangle and mirrors it into the upper triangle.
//   split-K    grid.y = splits: each split writes raw partial sums into a
//              workspace; dgemm_splitk_reduce_kernel sums them in a fixed
//              order (deterministic) and applies alpha/beta.
#include <algorithm>
#include <math.h>

#include "common.cuh"
#include "gemm_f64.cuh"

namespace evd {

namespace {

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// m16n8k4: A rows g and g+8 (column t), B row t (column g); D holds
// (g, 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1).
__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b));
}

// m16n8k8: A (g, t), (g+8, t), (g, t+4), (g+8, t+4); B (t, g), (t+4, g).
__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], const double (&a)[8],
                                            const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
// m16n8k16: A (g + 8(q&1), t + 4(q>>1)) for q = 0..7; B (t + 4q, g) for q = 0..3.
__device__ __forceinline__ void dmma_16x8x16(double (&d)[4], const double (&a)[8],
                                             const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

constexpr int kPad = 4;

template <bool TA, int BM, int BK>
struct ATile {
  // TA == false: A is m x k, m contiguous -> smem [k][BM+pad]
  // TA == true : A is k x m, k contiguous -> smem [m][BK+pad]
  static constexpr int kSize = TA ? BM * (BK + kPad) : BK * (BM + kPad);
  __device__ static __forceinline__ int at(int mi, int ki) {
    return TA ? mi * (BK + kPad) + ki : ki * (BM + kPad) + mi;
  }
};

template <bool TB, int BN, int BK>
struct BTile {
  // TB == false: B is k x n, k contiguous -> smem [n][BK+pad]
  // TB == true : B is n x k, n contiguous -> smem [k][BN+pad]
  static constexpr int kSize = TB ? BK * (BN + kPad) : BN * (BK + kPad);
  __device__ static __forceinline__ int at(int ki, int ni) {
    return TB ? ki * (BN + kPad) + ni : ni * (BK + kPad) + ki;
  }
};

// Copy one (rows x cols) tile whose global contiguous dimension has extent
// `cont` (tile length CL along it) and strided dimension extent SL.
// `g(ci, si)` -> global pointer, `lim_c`/`lim_s` valid extents from the tile
// origin, `s_off(ci, si)` -> smem offset.  vec16 copies two doubles per op.
template <int CL, int SL, int NT, typename GPtr, typename SOff>
__device__ __forceinline__ void load_tile(double* smem, GPtr g, SOff s_off, int lim_c,
                                          int lim_s, bool vec16, const double* safe) {
  if (vec16) {
    constexpr int kChunks = (CL / 2) * SL;
#pragma unroll
    for (int c = threadIdx.x; c < kChunks; c += NT) {
      int si = c / (CL / 2);
      int ci = (c % (CL / 2)) * 2;
      int rem = lim_c - ci;
      int bytes = (si < lim_s && rem > 0) ? (rem >= 2 ? 16 : 8) : 0;
      const double* src = bytes ? g(ci, si) : safe;
      cp_async16(smem + s_off(ci, si), src, bytes);
    }
  } else {
    constexpr int kChunks = CL * SL;
#pragma unroll
    for (int c = threadIdx.x; c < kChunks; c += NT) {
      int si = c / CL;
      int ci = c % CL;
      int bytes = (si < lim_s && ci < lim_c) ? 8 : 0;
      const double* src = bytes ? g(ci, si) : safe;
      cp_async8(smem + s_off(ci, si), src, bytes);
    }
  }
}

template <bool TA, bool TB, int BM, int BN, int BK, int WM, int WN, int STAGES, int MMA>
__global__ void __launch_bounds__((BM / WM) * (BN / WN) * 32)
    dgemm_kernel(const GemmArgs p) {
  constexpr int NWM = BM / WM, NWN = BN / WN;
  constexpr int NT = NWM * NWN * 32;
  // MMA: 0 = m8n8k4, 1 = m16n8k4, 2 = m16n8k8, 3 = m16n8k16
  constexpr int MR = (MMA >= 1) ? 16 : 8;  // rows per MMA tile
  constexpr int NC = (MMA >= 1) ? 4 : 2;   // accumulators per lane per MMA tile
  constexpr int KS = (MMA == 3) ? 16 : ((MMA == 2) ? 8 : 4);  // k per MMA
  constexpr int NA = (MMA == 3) ? 8 : ((MMA == 2) ? 4 : ((MMA == 1) ? 2 : 1));
  constexpr int NB = KS / 4;
  constexpr int MI = WM / MR, NJ = WN / 8;
  using AT = ATile<TA, BM, BK>;
  using BT = BTile<TB, BN, BK>;

  extern __shared__ __align__(16) double smem[];
  double* As = smem;
  double* Bs = smem + STAGES * AT::kSize;

  // ---- tile coordinates ----
  int tm, tn, z = blockIdx.y;
  if (p.mode == kSyr2kLow) {
    // lower-triangular tile enumeration, column-major: column tj holds T - tj tiles
    int T = p.tiles_m;
    long bid = blockIdx.x;
    // tj = largest j with j*T - j*(j-1)/2 <= bid
    double Td = T + 0.5;
    int tj = (int)(Td - sqrt(Td * Td - 2.0 * (double)bid));
    if (tj < 0) tj = 0;
    if (tj > T - 1) tj = T - 1;
    while (tj > 0 && (long)tj * T - (long)tj * (tj - 1) / 2 > bid) --tj;
    while ((long)(tj + 1) * T - (long)(tj + 1) * tj / 2 <= bid) ++tj;
    long start = (long)tj * T - (long)tj * (tj - 1) / 2;
    tn = tj;
    tm = tj + (int)(bid - start);
  } else {
    tm = blockIdx.x % p.tiles_m;
    tn = blockIdx.x / p.tiles_m;
  }
  const int m0 = tm * BM, n0 = tn * BN;

  int batch = z, split = 0;
  if (p.splitk > 1) {
    batch = z / p.splitk;
    split = z % p.splitk;
  }
  const double* Ab = p.A + (long)batch * p.sA;
  const double* Bb = p.B + (long)batch * p.sB;

  // K range of this split (multiple of BK except the last)
  const int ktot = p.k;
  int kbeg = 0, kend = ktot;
  if (p.splitk > 1) {
    int ktiles = (ktot + BK - 1) / BK;
    int per = (ktiles + p.splitk - 1) / p.splitk;
    kbeg = min(ktot, split * per * BK);
    kend = min(ktot, (split + 1) * per * BK);
  }
  const int KT = (kend - kbeg + BK - 1) / BK;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm0 = (warp % NWM) * WM, wn0 = (warp / NWM) * WN;
  const int g = lane >> 2, t = lane & 3;

  double acc[MI][NJ][NC];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int h = 0; h < NC; ++h) acc[i][j][h] = 0.0;

  auto issue = [&](int kt, int stage) {
    const int k0 = kbeg + kt * BK;
    const int klim = min(BK, kend - k0);
    double* as = As + stage * AT::kSize;
    double* bs = Bs + stage * BT::kSize;
    // operand-pair selection for the two-pair (SYR2K) mode: one K value per
    // strided index, so a chunk never straddles k1.
    const int mlim = p.m - m0, nlim = p.n - n0;
    if (!TA) {
      load_tile<BM, BK, NT>(
          as,
          [&](int ci, int si) {
            int kg = k0 + si;
            if (kg < p.k1) return Ab + (long)(m0 + ci) + (long)kg * p.lda;
            return p.A2 + (long)(m0 + ci) + (long)(kg - p.k1) * p.lda2;
          },
          [&](int ci, int si) { return AT::at(ci, si); }, mlim, klim, p.vecA, p.A);
    } else {
      load_tile<BK, BM, NT>(
          as,
          [&](int ci, int si) {
            int mg = m0 + si;
            if (mg < p.m1) return Ab + (long)(k0 + ci) + (long)mg * p.lda;
            return p.Am2 + (long)(k0 + ci) + (long)(mg - p.m1) * p.ldam2;
          },
          [&](int ci, int si) { return AT::at(si, ci); }, klim, mlim, p.vecA, p.A);
    }
    if (!TB) {
      load_tile<BK, BN, NT>(
          bs, [&](int ci, int si) { return Bb + (long)(k0 + ci) + (long)(n0 + si) * p.ldb; },
          [&](int ci, int si) { return BT::at(ci, si); }, klim, nlim, p.vecB, p.B);
    } else {
      load_tile<BN, BK, NT>(
          bs,
          [&](int ci, int si) {
            int kg = k0 + si;
            if (kg < p.k1) return Bb + (long)(n0 + ci) + (long)kg * p.ldb;
            return p.B2 + (long)(n0 + ci) + (long)(kg - p.k1) * p.ldb2;
          },
          [&](int ci, int si) { return BT::at(si, ci); }, nlim, klim, p.vecB, p.B);
    }
  };

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < KT) issue(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < KT; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      int nk = kt + STAGES - 1;
      if (nk < KT) issue(nk, nk % STAGES);
      cp_async_commit();
    }
    const double* as = As + (kt % STAGES) * AT::kSize;
    const double* bs = Bs + (kt % STAGES) * BT::kSize;
#pragma unroll
    for (int kk = 0; kk < BK; kk += KS) {
      double a[MI][8], b[NJ][4];
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int q = 0; q < NA; ++q)
          a[i][q] = as[AT::at(wm0 + i * MR + g + 8 * (q & 1), kk + t + 4 * (q >> 1))];
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int q = 0; q < NB; ++q) b[j][q] = bs[BT::at(kk + t + 4 * q, wn0 + j * 8 + g)];
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          double(&dd)[4] = *reinterpret_cast<double(*)[4]>(&acc[i][j][0]);
          if (MMA == 3) dmma_16x8x16(dd, a[i], b[j]);
          else if (MMA == 2) dmma_16x8x8(dd, a[i], b[j]);
          else if (MMA == 1) dmma_16x8x4(dd, a[i][0], a[i][1], b[j][0]);
          else dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i][0], b[j][0]);
        }
    }
  }
  cp_async_wait<0>();

  // ---- epilogue ----
  if (p.splitk > 1) {
    double* W = p.ws + ((long)batch * p.splitk + split) * (long)p.m * p.n;
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int h = 0; h < NC; ++h) {
          int r = m0 + wm0 + i * MR + g + 8 * (h >> 1), c = n0 + wn0 + j * 8 + 2 * t + (h & 1);
          if (r < p.m && c < p.n) W[r + (long)c * p.m] = acc[i][j][h];
        }
    return;
  }
  double* Cb = p.C + (long)batch * p.sC;
  const bool mirror = (p.mode == kSyr2kLow);
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int h = 0; h < NC; ++h) {
        int r = m0 + wm0 + i * MR + g + 8 * (h >> 1), c = n0 + wn0 + j * 8 + 2 * t + (h & 1);
        if (r >= p.m || c >= p.n) continue;
        if (mirror && r < c) continue;
        double* dst = Cb + r + (long)c * p.ldc;
        double v = p.alpha * acc[i][j][h];
        if (p.beta != 0.0) v = fma(p.beta, *dst, v);
        *dst = v;
        if (mirror && r != c) Cb[c + (long)r * p.ldc] = v;
      }
}

// ---------------------------------------------------------------------------
// Lean variant of dgemm_kernel for the common cases (no M-split operand pair,
// 16-byte aligned operands, K-split pair only at a multiple of BK): every
// thread's share of a tile copy is fixed at kernel start (one contiguous
// offset, one strided line plus a fixed stride per pass), so a k-tile costs
// one pointer computation per operand and a predicate per chunk instead of a
// full address computation per chunk.  Plain products use grouped
// rasterisation (kRaster tile rows at a time) so that the CTAs resident at
// once share their A and B panels in L2.
constexpr int kRaster = 8;

// Per-thread copy of a (CL contiguous x SL strided) tile into smem laid out
// [strided][CL + kPad], in 16-byte chunks.
template <int CL, int SL, int NT>
struct TileCopy {
  static constexpr int CH = CL / 2;  // chunks per strided line
  static_assert(NT % CH == 0, "threads must cover whole lines");
  static constexpr int SS = NT / CH;  // lines per pass
  static_assert(SL % SS == 0, "passes must cover the tile");
  static constexpr int R = SL / SS;   // passes
  static_assert(R <= 32, "predicate mask");
  int ci, si0;
  __device__ __forceinline__ void init() {
    ci = (threadIdx.x % CH) * 2;
    si0 = threadIdx.x / CH;
  }
  // bytes valid from contiguous index c (relative) given `rem` valid elements
  __device__ __forceinline__ static int cbytes(int rem) { return rem >= 2 ? 16 : (rem == 1 ? 8 : 0); }
  // strided lines si0 + r*SS < lim
  __device__ __forceinline__ unsigned smask(int lim) const {
    unsigned mk = 0;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (si0 + r * SS < lim) mk |= 1u << r;
    return mk;
  }
  __device__ __forceinline__ void issue(double* smem, const double* g, long step, int cb,
                                        unsigned mk, const double* safe) const {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int bytes = ((mk >> r) & 1u) ? cb : 0;
      cp_async16(smem + (si0 + r * SS) * (CL + kPad) + ci, bytes ? g + (long)r * step : safe,
                 bytes);
    }
  }
  // Same with one precomputed pointer per strided line (the line's element
  // ci of the tile is rows[r][koff]).
  __device__ __forceinline__ void issue_rows(double* smem, const double* const (&rows)[R],
                                             long koff, int cb, unsigned mk,
                                             const double* safe) const {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int bytes = ((mk >> r) & 1u) ? cb : 0;
      cp_async16(smem + (si0 + r * SS) * (CL + kPad) + ci, bytes ? rows[r] + koff : safe,
                 bytes);
    }
  }
};

template <bool TA, bool TB, int BM, int BN, int BK, int WM, int WN, int STAGES, int MMA>
__global__ void __launch_bounds__((BM / WM) * (BN / WN) * 32)
    dgemm_fast_kernel(const GemmArgs p) {
  constexpr int NWM = BM / WM, NWN = BN / WN;
  constexpr int NT = NWM * NWN * 32;
  constexpr int MR = (MMA >= 1) ? 16 : 8;
  constexpr int NC = (MMA >= 1) ? 4 : 2;
  constexpr int KS = (MMA == 3) ? 16 : ((MMA == 2) ? 8 : 4);
  constexpr int NA = (MMA == 3) ? 8 : ((MMA == 2) ? 4 : ((MMA == 1) ? 2 : 1));
  constexpr int NB = KS / 4;
  constexpr int MI = WM / MR, NJ = WN / 8;
  using AT = ATile<TA, BM, BK>;
  using BT = BTile<TB, BN, BK>;
  using ACopy = TileCopy<TA ? BK : BM, TA ? BM : BK, NT>;
  using BCopy = TileCopy<TB ? BN : BK, TB ? BK : BN, NT>;

  extern __shared__ __align__(16) double smem[];
  double* As = smem;
  double* Bs = smem + STAGES * AT::kSize;

  int tm, tn, z = blockIdx.y;
  if (p.mode == kSyr2kLow) {
    int T = p.tiles_m;
    long bid = blockIdx.x;
    double Td = T + 0.5;
    int tj = (int)(Td - sqrt(Td * Td - 2.0 * (double)bid));
    if (tj < 0) tj = 0;
    if (tj > T - 1) tj = T - 1;
    while (tj > 0 && (long)tj * T - (long)tj * (tj - 1) / 2 > bid) --tj;
    while ((long)(tj + 1) * T - (long)(tj + 1) * tj / 2 <= bid) ++tj;
    long start = (long)tj * T - (long)tj * (tj - 1) / 2;
    tn = tj;
    tm = tj + (int)(bid - start);
  } else {
    // grouped rasterisation: kRaster tile rows, column by column
    const int id = blockIdx.x;
    const int span = kRaster * p.tiles_n;
    const int grp = id / span, first = grp * kRaster;
    const int gm = min(kRaster, p.tiles_m - first);
    const int in = id - grp * span;
    tm = first + in % gm;
    tn = in / gm;
  }
  const int m0 = tm * BM, n0 = tn * BN;

  int batch = z, split = 0;
  if (p.splitk > 1) {
    batch = z / p.splitk;
    split = z % p.splitk;
  }
  const double* Ab = p.A + (long)batch * p.sA;
  const double* Bb = p.B + (long)batch * p.sB;

  const int ktot = p.k;
  int kbeg = 0, kend = ktot;
  if (p.splitk > 1) {
    int ktiles = (ktot + BK - 1) / BK;
    int per = (ktiles + p.splitk - 1) / p.splitk;
    kbeg = min(ktot, split * per * BK);
    kend = min(ktot, (split + 1) * per * BK);
  }
  const int KT = (kend - kbeg + BK - 1) / BK;

  ACopy ac;
  BCopy bc;
  ac.init();
  bc.init();
  // fixed predicates along M / N
  int a_cb = 16, b_cb = 16;
  unsigned a_mk = ~0u, b_mk = ~0u;
  if (!TA) a_cb = ACopy::cbytes(p.m - m0 - ac.ci);
  else a_mk = ac.smask(p.m - m0);
  // transposed A: rows m >= m1 of op(A) come from Am2 (the stacked operand of
  // the ZY update); one pointer per copied line, fixed for the whole kernel
  const double* arow[ACopy::R];
  if (TA) {
#pragma unroll
    for (int r = 0; r < ACopy::R; ++r) {
      const int mg = m0 + ac.si0 + r * ACopy::SS;
      arow[r] = (mg < p.m1 || p.Am2 == nullptr) ? Ab + ac.ci + (long)mg * p.lda
                                                : p.Am2 + ac.ci + (long)(mg - p.m1) * p.ldam2;
    }
  }
  if (TB) b_cb = BCopy::cbytes(p.n - n0 - bc.ci);
  else b_mk = bc.smask(p.n - n0);

  auto issue = [&](int kt, int stage) {
    const int k0 = kbeg + kt * BK;
    const int klim = kend - k0;  // valid K in this tile (may exceed BK)
    double* as = As + stage * AT::kSize;
    double* bs = Bs + stage * BT::kSize;
    if (!TA) {
      const bool second = k0 >= p.k1;
      const double* base = second ? p.A2 : Ab;
      const long ld = second ? p.lda2 : p.lda;
      const int kk = second ? k0 - p.k1 : k0;
      const double* g = base + (long)(m0 + ac.ci) + (long)(kk + ac.si0) * ld;
      const unsigned mk = (klim >= BK) ? ~0u : ac.smask(klim);
      ac.issue(as, g, (long)ACopy::SS * ld, a_cb, mk, p.A);
    } else {
      const int cb = (klim >= BK) ? 16 : ACopy::cbytes(klim - ac.ci);
      ac.issue_rows(as, arow, k0, cb, a_mk, p.A);
    }
    if (!TB) {
      const double* g = Bb + (long)(k0 + bc.ci) + (long)(n0 + bc.si0) * p.ldb;
      const int cb = (klim >= BK) ? 16 : BCopy::cbytes(klim - bc.ci);
      bc.issue(bs, g, (long)BCopy::SS * p.ldb, cb, b_mk, p.B);
    } else {
      const bool second = k0 >= p.k1;
      const double* base = second ? p.B2 : Bb;
      const long ld = second ? p.ldb2 : p.ldb;
      const int kk = second ? k0 - p.k1 : k0;
      const double* g = base + (long)(n0 + bc.ci) + (long)(kk + bc.si0) * ld;
      const unsigned mk = (klim >= BK) ? ~0u : bc.smask(klim);
      bc.issue(bs, g, (long)BCopy::SS * ld, b_cb, mk, p.B);
    }
  };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm0 = (warp % NWM) * WM, wn0 = (warp / NWM) * WN;
  const int g = lane >> 2, t = lane & 3;

  double acc[MI][NJ][NC];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int h = 0; h < NC; ++h) acc[i][j][h] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < KT) issue(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < KT; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      int nk = kt + STAGES - 1;
      if (nk < KT) issue(nk, nk % STAGES);
      cp_async_commit();
    }
    const double* as = As + (kt % STAGES) * AT::kSize;
    const double* bs = Bs + (kt % STAGES) * BT::kSize;
#pragma unroll
    for (int kk = 0; kk < BK; kk += KS) {
      double a[MI][8], b[NJ][4];
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int q = 0; q < NA; ++q)
          a[i][q] = as[AT::at(wm0 + i * MR + g + 8 * (q & 1), kk + t + 4 * (q >> 1))];
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int q = 0; q < NB; ++q) b[j][q] = bs[BT::at(kk + t + 4 * q, wn0 + j * 8 + g)];
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          double(&dd)[4] = *reinterpret_cast<double(*)[4]>(&acc[i][j][0]);
          if (MMA == 3) dmma_16x8x16(dd, a[i], b[j]);
          else if (MMA == 2) dmma_16x8x8(dd, a[i], b[j]);
          else if (MMA == 1) dmma_16x8x4(dd, a[i][0], a[i][1], b[j][0]);
          else dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i][0], b[j][0]);
        }
    }
  }
  cp_async_wait<0>();

  if (p.splitk > 1) {
    double* W = p.ws + ((long)batch * p.splitk + split) * (long)p.m * p.n;
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int h = 0; h < NC; ++h) {
          int r = m0 + wm0 + i * MR + g + 8 * (h >> 1), c = n0 + wn0 + j * 8 + 2 * t + (h & 1);
          if (r < p.m && c < p.n) W[r + (long)c * p.m] = acc[i][j][h];
        }
    return;
  }
  double* Cb = p.C + (long)batch * p.sC;
  const bool mirror = (p.mode == kSyr2kLow);
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int h = 0; h < NC; ++h) {
        int r = m0 + wm0 + i * MR + g + 8 * (h >> 1), c = n0 + wn0 + j * 8 + 2 * t + (h & 1);
        if (r >= p.m || c >= p.n) continue;
        if (mirror && r < c) continue;
        double* dst = Cb + r + (long)c * p.ldc;
        double v = p.alpha * acc[i][j][h];
        if (p.beta != 0.0) v = fma(p.beta, *dst, v);
        *dst = v;
        if (mirror && r != c) Cb[c + (long)r * p.ldc] = v;
      }
}

__global__ void dgemm_splitk_reduce_kernel(int m, int n, int splits, long batch_count,
                                           const double* ws, double alpha, double beta,
                                           double* C, long ldc, long sC) {
  long total = (long)m * n;
  for (long b = 0; b < batch_count; ++b) {
    const double* W = ws + b * splits * total;
    double* Cb = C + b * sC;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
      double s = 0.0;
      for (int q = 0; q < splits; ++q) s += W[q * total + idx];
      long r = idx % m, c = idx / m;
      double* dst = Cb + r + c * ldc;
      double v = alpha * s;
      if (beta != 0.0) v = fma(beta, *dst, v);
      *dst = v;
    }
  }
}

template <bool TA, bool TB, int BM, int BN, int BK, int WM, int WN, int STAGES, int MMA = 0,
          bool FAST = false>
int launch_cfg(GemmArgs p, int grid_x, int grid_y, cudaStream_t st) {
  constexpr int NT = (BM / WM) * (BN / WN) * 32;
  constexpr size_t smem =
      STAGES * (ATile<TA, BM, BK>::kSize + BTile<TB, BN, BK>::kSize) * sizeof(double);
  auto kern = FAST ? dgemm_fast_kernel<TA, TB, BM, BN, BK, WM, WN, STAGES, MMA>
                   : dgemm_kernel<TA, TB, BM, BN, BK, WM, WN, STAGES, MMA>;
  EVD_TRY(smem_attr_once((const void*)kern, (int)smem));
  kern<<<dim3(grid_x, grid_y), NT, smem, st>>>(p);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

static inline bool aligned16(const void* ptr, long ld) {
  return (((uintptr_t)ptr & 15u) == 0) && ((ld & 1) == 0);
}

template <bool TA, bool TB>
int dispatch_shape(GemmArgs p, long batch, cudaStream_t st) {
  // Tile shapes chosen by measurement on B200 (DGEMM 8192^3: 64x64 tiles with
  // four 32x32 warps and m16n8k16 DMMA reach 30 TFLOP/s, 128x128 tiles 27;
  // the skinny n = 32 ZY products run best as 64x32 tiles with split-K).
  // The lean kernel serves every call whose operands are 16-byte aligned and
  // whose K-split operand pair (if any) switches at a multiple of BK = 16;
  // the general kernel covers the rest (odd alignments).
  const bool fast = p.vecA && p.vecB && (TA || p.Am2 == nullptr || p.m1 >= p.m) &&
                    (p.k1 >= p.k || p.k1 % 16 == 0);
  if (p.n <= 32 && p.mode == kGemm) {
    constexpr int BM = 64, BN = 32;
    p.tiles_m = ceil_div_i(p.m, BM);
    p.tiles_n = ceil_div_i(p.n, BN);
    int grid_x = p.tiles_m * p.tiles_n;
    int grid_y = (int)batch * max(1, p.splitk);
    return fast ? launch_cfg<TA, TB, BM, BN, 16, 16, 32, 4, 3, true>(p, grid_x, grid_y, st)
                : launch_cfg<TA, TB, BM, BN, 16, 16, 32, 4, 3>(p, grid_x, grid_y, st);
  }
  constexpr int BM = 64, BN = 64;
  p.tiles_m = ceil_div_i(p.m, BM);
  p.tiles_n = ceil_div_i(p.n, BN);
  int grid_x = (p.mode == kSyr2kLow) ? p.tiles_m * (p.tiles_m + 1) / 2
                                     : p.tiles_m * p.tiles_n;
  int grid_y = (int)batch * max(1, p.splitk);
  // the lean kernel with two stages: 36 KB of shared memory per CTA lets six
  // CTAs (24 warps) share an SM, which hides the DMMA latency better than
  // deeper prefetch (B200: 32.8 / 33.5 TFLOP/s NN / TN 8192^3-class against
  // 32.6 / 32.3 with four stages)
  return fast ? launch_cfg<TA, TB, BM, BN, 16, 32, 32, 2, 3, true>(p, grid_x, grid_y, st)
              : launch_cfg<TA, TB, BM, BN, 16, 32, 32, 4, 3>(p, grid_x, grid_y, st);
}

}  // namespace

static bool aligned16_all(const double* ptr, long ld, long stride) {
  return aligned16(ptr, ld) && ((stride & 1) == 0);
}

static int gemm_run(GemmArgs p, bool ta, bool tb, long batch, cudaStream_t st,
                    double* ws, size_t ws_doubles) {
  if (p.m <= 0 || p.n <= 0 || batch <= 0) return EVD_SUCCESS;
  p.vecA = aligned16_all(p.A, p.lda, p.sA) && (p.A2 == nullptr || aligned16(p.A2, p.lda2)) &&
           (p.Am2 == nullptr || aligned16(p.Am2, p.ldam2));
  if (p.Am2 == nullptr || p.m1 <= 0) p.m1 = p.m;
  p.vecB = aligned16_all(p.B, p.ldb, p.sB) && (p.B2 == nullptr || aligned16(p.B2, p.ldb2));
  if (p.k1 <= 0 || p.A2 == nullptr) p.k1 = p.k;
  if (p.k <= 0) p.splitk = 1;
  // shrink the split count until the partial sums fit in the caller's scratch
  while (p.splitk > 1 && gemm_splitk_ws_doubles(p.m, p.n, p.splitk, batch) > ws_doubles)
    p.splitk >>= 1;
  if (p.splitk > 1) p.ws = ws;
  if ((long)batch * (p.splitk > 1 ? p.splitk : 1) > 65535) return EVD_ERR_INVALID_ARG;
  int st_code;
  if (!ta && !tb) st_code = dispatch_shape<false, false>(p, batch, st);
  else if (!ta && tb) st_code = dispatch_shape<false, true>(p, batch, st);
  else if (ta && !tb) st_code = dispatch_shape<true, false>(p, batch, st);
  else st_code = dispatch_shape<true, true>(p, batch, st);
  if (st_code != EVD_SUCCESS) return st_code;
  if (p.splitk > 1) {
    long total = (long)p.m * p.n;
    int blocks = (int)std::min<long>((total + 255) / 256, 4L * device_sm_count());
    dgemm_splitk_reduce_kernel<<<blocks, 256, 0, st>>>(p.m, p.n, p.splitk, batch, p.ws,
                                                       p.alpha, p.beta, p.C, p.ldc, p.sC);
    EVD_LAUNCHED();
  }
  return EVD_SUCCESS;
}

int choose_splitk(long m, long n, long k, long batch) {
  // Enough CTAs for about four per SM when the output is small and K long
  // (eight for the n <= 32 panel products, measured best on B200).
  const long bm = 64, bn = (n <= 32) ? 32 : 64;
  long tiles = ((m + bm - 1) / bm) * ((n + bn - 1) / bn) * batch;
  long want = ((n <= 32) ? 8L : 4L) * device_sm_count();
  if (tiles >= want || k < 512) return 1;
  long s = (want + tiles - 1) / tiles;
  long kmax = k / 256;  // keep >= 256 of K per split
  if (s > kmax) s = kmax;
  if (s > 32) s = 32;
  return (int)std::max<long>(1, s);
}

static inline bool is_trans(char c) { return c == 't' || c == 'T' || c == 'c' || c == 'C'; }

int dgemm(char transa, char transb, long m, long n, long k, double alpha, const double* A,
          long lda, const double* B, long ldb, double beta, double* C, long ldc,
          cudaStream_t st, int splitk, double* ws, size_t ws_doubles) {
  bool ta = is_trans(transa), tb = is_trans(transb);
  if (m < 0 || n < 0 || k < 0) return EVD_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return EVD_SUCCESS;
  if (C == nullptr || ldc < m) return EVD_ERR_INVALID_ARG;
  if (k > 0) {
    if (A == nullptr || B == nullptr) return EVD_ERR_INVALID_ARG;
    if (lda < (ta ? k : m) || ldb < (tb ? n : k)) return EVD_ERR_INVALID_ARG;
  }
  if (m > INT32_MAX || n > INT32_MAX || k > INT32_MAX) return EVD_ERR_INVALID_ARG;
  GemmArgs p{};
  p.m = (int)m;
  p.n = (int)n;
  p.k = (int)k;
  p.alpha = alpha;
  p.beta = beta;
  p.A = A ? A : C;
  p.lda = lda;
  p.B = B ? B : C;
  p.ldb = ldb;
  p.C = C;
  p.ldc = ldc;
  p.mode = kGemm;
  p.splitk = (splitk > 0) ? splitk : choose_splitk(m, n, k, 1);
  return gemm_run(p, ta, tb, 1, st, ws, ws_doubles);
}

int dgemm_batched(char transa, char transb, long m, long n, long k, double alpha,
                  const double* A, long lda, long sA, const double* B, long ldb, long sB,
                  double beta, double* C, long ldc, long sC, long batch, cudaStream_t st) {
  bool ta = is_trans(transa), tb = is_trans(transb);
  if (m < 0 || n < 0 || k < 0 || batch < 0) return EVD_ERR_INVALID_ARG;
  if (m == 0 || n == 0 || batch == 0) return EVD_SUCCESS;
  if (C == nullptr || ldc < m) return EVD_ERR_INVALID_ARG;
  if (k > 0 && (lda < (ta ? k : m) || ldb < (tb ? n : k))) return EVD_ERR_INVALID_ARG;
  if (batch > 65535 || m > INT32_MAX || n > INT32_MAX || k > INT32_MAX)
    return EVD_ERR_INVALID_ARG;
  GemmArgs p{};
  p.m = (int)m;
  p.n = (int)n;
  p.k = (int)k;
  p.alpha = alpha;
  p.beta = beta;
  p.A = A ? A : C;
  p.lda = lda;
  p.sA = sA;
  p.B = B ? B : C;
  p.ldb = ldb;
  p.sB = sB;
  p.C = C;
  p.ldc = ldc;
  p.sC = sC;
  p.mode = kGemm;
  p.splitk = 1;
  return gemm_run(p, ta, tb, batch, st, nullptr, 0);
}

int dgemm_nt_pair(long m, long n, long k1, long k2, double alpha, const double* A1, long lda1,
                  const double* B1, long ldb1, const double* A2, long lda2, const double* B2,
                  long ldb2, double beta, double* C, long ldc, cudaStream_t st, int splitk,
                  double* ws, size_t ws_doubles) {
  if (m < 0 || n < 0 || k1 < 0 || k2 < 0) return EVD_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return EVD_SUCCESS;
  if (C == nullptr || ldc < m) return EVD_ERR_INVALID_ARG;
  if (k1 == 0) return dgemm('n', 't', m, n, k2, alpha, A2, lda2, B2, ldb2, beta, C, ldc, st,
                            splitk, ws, ws_doubles);
  if (k2 == 0) return dgemm('n', 't', m, n, k1, alpha, A1, lda1, B1, ldb1, beta, C, ldc, st,
                            splitk, ws, ws_doubles);
  if (lda1 < m || lda2 < m || ldb1 < n || ldb2 < n) return EVD_ERR_INVALID_ARG;
  if (m > INT32_MAX || n > INT32_MAX || k1 + k2 > INT32_MAX) return EVD_ERR_INVALID_ARG;
  GemmArgs p{};
  p.m = (int)m;
  p.n = (int)n;
  p.k = (int)(k1 + k2);
  p.k1 = (int)k1;
  p.alpha = alpha;
  p.beta = beta;
  p.A = A1;
  p.lda = lda1;
  p.B = B1;
  p.ldb = ldb1;
  p.A2 = A2;
  p.lda2 = lda2;
  p.B2 = B2;
  p.ldb2 = ldb2;
  p.C = C;
  p.ldc = ldc;
  p.mode = kGemm;
  p.splitk = (splitk > 0) ? splitk : choose_splitk(m, n, k1 + k2, 1);
  return gemm_run(p, false, true, 1, st, ws, ws_doubles);
}

int dgemm_pair(const GemmPair& g, cudaStream_t st, int splitk, double* ws, size_t ws_doubles) {
  const bool ta = is_trans(g.ta), tb = is_trans(g.tb);
  if (g.m < 0 || g.n < 0 || g.k < 0) return EVD_ERR_INVALID_ARG;
  if (g.m == 0 || g.n == 0) return EVD_SUCCESS;
  if (!g.C || g.ldc < g.m) return EVD_ERR_INVALID_ARG;
  if (g.Am2 && (!ta || g.m1 <= 0 || g.m1 > g.m)) return EVD_ERR_INVALID_ARG;
  if (g.A2 && (ta || g.k1 <= 0 || g.k1 > g.k)) return EVD_ERR_INVALID_ARG;
  if (g.B2 && (!tb || !g.A2)) return EVD_ERR_INVALID_ARG;
  if (g.m > INT32_MAX || g.n > INT32_MAX || g.k > INT32_MAX) return EVD_ERR_INVALID_ARG;
  GemmArgs p{};
  p.m = (int)g.m;
  p.n = (int)g.n;
  p.k = (int)g.k;
  p.alpha = g.alpha;
  p.beta = g.beta;
  p.A = g.A ? g.A : g.C;
  p.lda = g.lda;
  p.B = g.B ? g.B : g.C;
  p.ldb = g.ldb;
  p.C = g.C;
  p.ldc = g.ldc;
  p.A2 = g.A2;
  p.lda2 = g.lda2;
  p.k1 = g.A2 ? (int)g.k1 : 0;
  p.B2 = g.B2 ? g.B2 : (g.A2 ? p.B : nullptr);
  p.ldb2 = g.B2 ? g.ldb2 : g.ldb;
  if (g.A2 && !g.B2 && tb) return EVD_ERR_INVALID_ARG;
  p.Am2 = g.Am2;
  p.ldam2 = g.ldam2;
  p.m1 = g.Am2 ? (int)g.m1 : 0;
  p.mode = kGemm;
  p.splitk = (splitk > 0) ? splitk : choose_splitk(g.m, g.n, g.k, 1);
  return gemm_run(p, ta, tb, 1, st, ws, ws_doubles);
}

int syr2k_lower_mirror(long n, long k, double alpha, const double* A, long lda,
                       const double* B, long ldb, double beta, double* C, long ldc,
                       cudaStream_t st) {
  if (n < 0 || k < 0) return EVD_ERR_INVALID_ARG;
  if (n == 0) return EVD_SUCCESS;
  if (C == nullptr || ldc < n || (k > 0 && (lda < n || ldb < n))) return EVD_ERR_INVALID_ARG;
  if (n > INT32_MAX || 2 * k > INT32_MAX) return EVD_ERR_INVALID_ARG;
  GemmArgs p{};
  p.m = (int)n;
  p.n = (int)n;
  p.k = (int)(2 * k);
  p.k1 = (int)k;
  p.alpha = alpha;
  p.beta = beta;
  p.A = A ? A : C;
  p.lda = lda;
  p.B = B ? B : C;
  p.ldb = ldb;
  p.A2 = B ? B : C;
  p.lda2 = ldb;
  p.B2 = A ? A : C;
  p.ldb2 = lda;
  p.C = C;
  p.ldc = ldc;
  p.mode = kSyr2kLow;
  p.splitk = 1;
  if (k == 0) {
    p.k = 0;
    p.A2 = nullptr;
    p.B2 = nullptr;
  }
  return gemm_run(p, false, true, 1, st, nullptr, 0);
}

}  // namespace evd

extern "C" int evd_dgemm(char transa, char transb, long m, long n, long k, double alpha,
                         const double* A, long lda, const double* B, long ldb, double beta,
                         double* C, long ldc, cudaStream_t stream) {
  // No caller scratch on this entry point, so no split-K.
  return evd::dgemm(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream, 1);
}

extern "C" int evd_dgemm_strided_batched(char transa, char transb, long m, long n, long k,
                                         double alpha, const double* A, long lda, long strideA,
                                         const double* B, long ldb, long strideB, double beta,
                                         double* C, long ldc, long strideC, long batch,
                                         cudaStream_t stream) {
  return evd::dgemm_batched(transa, transb, m, n, k, alpha, A, lda, strideA, B, ldb, strideB,
                            beta, C, ldc, strideC, batch, stream);
}

extern "C" int evd_syr2k_lower_mirror(long n, long k, double alpha, const double* A, long lda,
                                      const double* B, long ldb, double beta, double* C,
                                      long ldc, long nb, cudaStream_t stream) {
  (void)nb;
  return evd::syr2k_lower_mirror(n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
}
