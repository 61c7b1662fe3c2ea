// Panel factorisation for stage 1: tall-skinny QR (m x 32) and the compact
// Householder form Q = I - W Y^T.
//
// Reference: panelQR<double> (api/panelQR.cu:54-108) = hou_tsqr_panel<128,32>
// (api/inc/TallShinnyQR.h:9-133, leaf kernel util/inc/kernelQR.h:215-414),
// then IminusQ, cusolverDnDgetrf without pivoting, getLower and a Dtrsm.
//
// Same numerics, B200 structure:
//  * The TSQR tree has the reference's shape (128-row tiles, R factors
//    stacked 32 rows per child, fan-in 4; api/inc/TallShinnyQR.h:9-133).  The
//    shape is kept on purpose: the signs of R (hence of Y, W and the band)
//    follow from the Householder sign rule applied node by node, so another
//    tree gives R up to row signs, not the reference's R.  It runs as ONE
//    up-sweep kernel: each CTA factors its tile in registers, publishes its R,
//    and the last child to arrive at a parent (atomic counter) goes on to
//    factor the parent.  Nobody waits, so there is no grid barrier and no
//    spin.  The reference launches one kernel plus batched GEMMs per level.
//  * One finishing kernel forms each tile's rows of the explicit thin Q
//    (leaf Q times the 32x32 path product down the tree, right to left as
//    the reference's recursion), and in the same pass rebuilds the Householder
//    form: the unpivoted LU of (I - Q)[0:32] (recomputed redundantly by each
//    CTA from tile 0's data, so no inter-CTA dependency), Y = (I-Q) U^{-1}
//    (rows >= 32) or L1 (rows < 32), W = (I-Q) L1^{-T}.  This replaces the
//    getrf + getLower + trsm + copy kernels.
//  * In the sy2sb pipeline the finishing kernel writes Y and W straight into
//    dY/dW and the band (R over zeros) into dA (the reference's copyMatrix +
//    getU, api/zy_zy_sy2sb.cu:122-125).
#include "common.cuh"
#include "panel_qr.cuh"

namespace evd {

namespace {

constexpr int kTile = 128;        // rows per TSQR tile (reference: M = 128)
constexpr int kNB = 32;           // panel width (reference: N = 32)
constexpr int kFan = kTile / kNB; // children per tree node (their R factors fill one tile)
constexpr int kThreads = 256;     // 8 warps x 4 columns
constexpr int kRPL = kTile / 32;  // rows per lane in a tile QR
constexpr int kSub = 128;         // rows per CTA of the finishing kernel
constexpr int kMaxLevels = 16;

struct TsqrPlan {
  int m;
  int nlev;                 // number of levels; level nlev-1 is the root (1 tile)
  int T[kMaxLevels];        // tiles at each level
  int rows[kMaxLevels];     // rows of the matrix factored at each level
  long soff[kMaxLevels];    // offset (doubles) of stack S_L in ws (L >= 1)
  int coff[kMaxLevels];     // offset of the arrival counters of level L (L >= 1)
  long qtop_off;            // 32x32 copy of tile 0's leaf Q rows 0..31
  long cnt_off;             // int counters start (in doubles, aligned)
  int ncnt;
  long total;               // doubles
};

TsqrPlan make_plan(long m) {
  TsqrPlan p{};
  p.m = (int)m;
  int L = 0;
  p.rows[0] = (int)m;
  p.T[0] = ceil_div_i(m, kTile);
  int coff = 0;
  while (p.T[L] > 1 && L + 1 < kMaxLevels) {
    p.rows[L + 1] = kNB * p.T[L];
    p.T[L + 1] = ceil_div_i(p.rows[L + 1], kTile);
    p.coff[L + 1] = coff;
    coff += p.T[L + 1];
    ++L;
  }
  p.nlev = L + 1;
  p.ncnt = coff;
  // Arrival counters come first, at a fixed offset: a workspace sized (and
  // zeroed) for the largest panel then serves every smaller panel, whose
  // counters are a prefix of the same region (the kernels reset each counter
  // after use).
  p.cnt_off = 0;
  long off = (coff + 1) / 2 + 2;  // ints packed two per double
  off = (off + 1) / 2 * 2;        // keep the stacks 16-byte aligned
  for (int l = 1; l < p.nlev; ++l) {
    p.soff[l] = off;
    off += (long)p.rows[l] * kNB;
  }
  p.qtop_off = off;
  off += kNB * kNB;
  p.total = off;
  return p;
}

// Full warp sums of four per-lane partials (one per column of the warp):
// reduce-scatter (lanes keep two columns, then one) and a broadcast back, 20
// 32-bit shuffles instead of 40 for four butterflies.
__device__ __forceinline__ void warp_sum4(double (&p)[4], int lane) {
  const bool b4 = lane & 16, b3 = lane & 8;
  const double s0 = b4 ? p[0] : p[2], s1 = b4 ? p[1] : p[3];
  const double r0 = __shfl_xor_sync(0xffffffffu, s0, 16);
  const double r1 = __shfl_xor_sync(0xffffffffu, s1, 16);
  const double k0 = (b4 ? p[2] : p[0]) + r0;  // column 2*b4
  const double k1 = (b4 ? p[3] : p[1]) + r1;  // column 2*b4 + 1
  const double r = __shfl_xor_sync(0xffffffffu, b3 ? k0 : k1, 8);
  double k = (b3 ? k1 : k0) + r;  // column 2*b4 + b3
  k += __shfl_xor_sync(0xffffffffu, k, 4);
  k += __shfl_xor_sync(0xffffffffu, k, 2);
  k += __shfl_xor_sync(0xffffffffu, k, 1);
#pragma unroll
  for (int c = 0; c < 4; ++c) p[c] = __shfl_sync(0xffffffffu, k, (c >> 1) * 16 + (c & 1) * 8);
}

// Householder QR of one tile (mm <= 128 rows, 32 columns) held in registers:
// warp w owns columns w, w + 8, w + 16, w + 24 (a[c] holds column 8c + w),
// lane l owns rows l + 32 i (i < 4).  Writes R (32 x 32, upper; diag =
// -sign(x0) ||x||) to Rdst and leaves the reflectors in the tile (column j,
// rows >= j; rows above hold R) for tile_form_q.  Same steps as
// my_hou_kernel<128,32> (util/inc/kernelQR.h:215-414): u = x/||x||,
// u0 += sign(u0), u scaled to ||u||^2 = 2.
// Look-ahead: once reflector j is in shared memory, the owner of column j+1
// (another warp) applies it to that column alone, builds reflector j+1 and
// publishes it (bar.arrive on a named barrier), and only then applies j to its
// other columns; every other warp waits on that barrier (bar.sync) and applies
// j to its columns.  The dependency chain per column is then one single-column
// update and one reflector, not a reflector plus a four-column update and a
// CTA barrier.  Barrier of column j: 1 + (j & 3) (0 is __syncthreads); at most
// two are in flight, because a warp must wait on column j before it can
// publish j + 1.
struct TileSmem {
  double V[kNB * kTile];  // reflector j at V[j * kTile ..]
  double RR[kNB];
};
constexpr size_t kTileSmem = sizeof(TileSmem);

__device__ __forceinline__ int qr_bar(int j) { return 1 + (j & 3); }
__device__ __forceinline__ void qr_bar_arrive(int id) {
  asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "n"(kThreads) : "memory");
}
__device__ __forceinline__ void qr_bar_wait(int id) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "n"(kThreads) : "memory");
}

// Reflector of column j from a[c] (c = j / 8, this warp owns j): writes
// V[j], RR[j] and the reflector into a[c] (rows >= j).
__device__ __forceinline__ void tile_reflector(double (&a)[4][kRPL], int j, int mm, int lane,
                                               TileSmem& sm) {
  const int oc = j >> 3;
  double x[kRPL], ss = 0.0;
#pragma unroll
  for (int i = 0; i < kRPL; ++i) {
    const int row = lane + 32 * i;
    double v = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (c == oc) v = a[c][i];
    x[i] = (row >= j && row < mm) ? v : 0.0;
    ss = fma(x[i], x[i], ss);
  }
  const double nrm2 = warp_sum(ss);
  const double x0 = __shfl_sync(0xffffffffu, x[0], j);  // row j: lane j, i = 0
  // A zero column (nothing to annihilate) gets u = sqrt(2) e_j rather than
  // u = 0: H = I - u u^T then only flips row j, R_jj = 0, every reflector
  // keeps ||u||^2 = 2, and I - Q stays nonsingular for the Householder
  // reconstruction (u = 0 would give a zero pivot there).
  const bool live = nrm2 > 0.0;
  const double rn = live ? rsqrt(nrm2) : 0.0;  // 1 / ||x||
  const double u0 = x0 * rn;
  const double u0n = live ? u0 + ((u0 >= 0.0) ? 1.0 : -1.0) : 1.4142135623730951;
  const double s2 = live ? rsqrt(fabs(u0n)) : 1.0;
  if (lane == 0) sm.RR[j] = live ? ((u0 >= 0.0) ? -(nrm2 * rn) : nrm2 * rn) : 0.0;
#pragma unroll
  for (int i = 0; i < kRPL; ++i) {
    const int row = lane + 32 * i;
    const double u = ((row == j) ? u0n : x[i] * rn) * s2;
    sm.V[j * kTile + row] = u;
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (c == oc && row >= j) a[c][i] = u;
  }
}

__device__ void tile_factor(double* src, long ld, int mm, double* Rdst, long ldR, TileSmem& sm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double a[4][kRPL];
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int i = 0; i < kRPL; ++i) {
      const int row = lane + 32 * i;
      a[c][i] = (row < mm) ? __ldcg(src + row + (long)(8 * c + warp) * ld) : 0.0;
    }

  if (warp == 0) {
    tile_reflector(a, 0, mm, lane, sm);
    qr_bar_arrive(qr_bar(0));
  }
  for (int j = 0; j < kNB; ++j) {
    if (warp != (j & 7)) qr_bar_wait(qr_bar(j));  // reflector j is in V[j]
    double uv[kRPL];
#pragma unroll
    for (int i = 0; i < kRPL; ++i) uv[i] = sm.V[j * kTile + lane + 32 * i];
    const int j1 = j + 1;
    const bool own1 = j1 < kNB && warp == (j1 & 7);
    if (own1) {
      // column j + 1 first, then its reflector, published at once
      const int c1 = j1 >> 3;
      double p0 = 0.0, p1 = 0.0;
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (c == c1) {
#pragma unroll
          for (int i = 0; i < kRPL; i += 2) {
            p0 = fma(uv[i], a[c][i], p0);
            p1 = fma(uv[i + 1], a[c][i + 1], p1);
          }
        }
      const double dot = warp_sum(p0 + p1);
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (c == c1) {
#pragma unroll
          for (int i = 0; i < kRPL; ++i) a[c][i] = fma(-dot, uv[i], a[c][i]);
        }
      tile_reflector(a, j1, mm, lane, sm);
      qr_bar_arrive(qr_bar(j1));
    }
    if (8 * 3 + warp <= j) continue;  // all columns of this warp factored (warp-uniform)
    // the warp's other columns right of j (column j + 1 is done above); the
    // four dot products are reduced together
    double pc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double p0 = 0.0, p1 = 0.0;
#pragma unroll
      for (int i = 0; i < kRPL; i += 2) {
        p0 = fma(uv[i], a[c][i], p0);
        p1 = fma(uv[i + 1], a[c][i + 1], p1);
      }
      pc[c] = p0 + p1;
    }
    warp_sum4(pc, lane);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int h = 8 * c + warp;
      const double dot = (h > j && h != j1) ? pc[c] : 0.0;
#pragma unroll
      for (int i = 0; i < kRPL; ++i) a[c][i] = fma(-dot, uv[i], a[c][i]);
    }
  }
  __syncthreads();  // RR complete

  // R: row k = lane (i = 0), column h = 8c + w; reflectors back into the tile
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int h = 8 * c + warp;
    const double r = (lane < h) ? a[c][0] : ((lane == h) ? sm.RR[h] : 0.0);
    Rdst[lane + (long)h * ldR] = r;
#pragma unroll
    for (int i = 0; i < kRPL; ++i) {
      const int row = lane + 32 * i;
      if (row < mm) src[row + (long)h * ld] = a[c][i];
    }
  }
}

// Explicit thin Q = H_0 ... H_31 I[:, :32] of a factored tile, from the
// reflectors left in it, accumulated backwards and written over them.  Before
// H_j is applied, columns c < j are still e_c, which H_j leaves unchanged, so
// warps whose columns are all left of j skip the step.
__device__ void tile_form_q(double* src, long ld, int mm, TileSmem& sm, double* qtop_copy) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int e = threadIdx.x; e < kNB * kTile; e += kThreads) {
    const int j = e / kTile, row = e % kTile;
    sm.V[e] = (row >= j && row < mm) ? __ldcg(src + row + (long)j * ld) : 0.0;
  }
  __syncthreads();
  double q[4][kRPL];
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int i = 0; i < kRPL; ++i) q[c][i] = (lane + 32 * i == 4 * warp + c) ? 1.0 : 0.0;
  for (int j = kNB - 1; j >= 0; --j) {
    if (4 * warp + 3 < j) continue;  // warp-uniform
    double uv[kRPL];
#pragma unroll
    for (int i = 0; i < kRPL; ++i) uv[i] = sm.V[j * kTile + lane + 32 * i];
    double pc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double p0 = 0.0, p1 = 0.0;
#pragma unroll
      for (int i = 0; i < kRPL; i += 2) {
        p0 = fma(uv[i], q[c][i], p0);
        p1 = fma(uv[i + 1], q[c][i + 1], p1);
      }
      pc[c] = p0 + p1;
    }
    warp_sum4(pc, lane);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double dot = (4 * warp + c >= j) ? pc[c] : 0.0;
#pragma unroll
      for (int i = 0; i < kRPL; ++i) q[c][i] = fma(-dot, uv[i], q[c][i]);
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int i = 0; i < kRPL; ++i) {
      const int row = lane + 32 * i;
      if (row < mm) {
        src[row + (long)(4 * warp + c) * ld] = q[c][i];
        if (qtop_copy && row < kNB) qtop_copy[row + (4 * warp + c) * kNB] = q[c][i];
      }
    }
}

__global__ void __launch_bounds__(kThreads, 1) tsqr_up_kernel(const TsqrPlan plan, double* A,
                                                              long lda, double* ws, double* Rout,
                                                              long ldr) {
  extern __shared__ __align__(16) double up_smem[];
  TileSmem& sm = *reinterpret_cast<TileSmem*>(up_smem);
  __shared__ int is_last;
  int* cnt = reinterpret_cast<int*>(ws + plan.cnt_off);
  int level = 0, idx = blockIdx.x;
  for (;;) {
    double* src;
    long ld;
    if (level == 0) {
      src = A + (long)idx * kTile;
      ld = lda;
    } else {
      src = ws + plan.soff[level] + (long)idx * kTile;
      ld = plan.rows[level];
    }
    int mm = min(kTile, plan.rows[level] - idx * kTile);
    const bool root = (plan.T[level] == 1);
    double* Rdst;
    long ldR;
    if (root) {
      Rdst = Rout;
      ldR = ldr;
    } else {
      Rdst = ws + plan.soff[level + 1] + (long)idx * kNB;
      ldR = plan.rows[level + 1];
    }
    tile_factor(src, ld, mm, Rdst, ldR, sm);
    if (root) break;
    const int parent = idx / kFan;
    const int nch = min(kFan, plan.T[level] - kFan * parent);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      int* c = cnt + plan.coff[level + 1] + parent;
      int old = atomicAdd(c, 1);
      is_last = (old == nch - 1);
      if (is_last) *c = 0;  // self-reset for the next panel
    }
    __syncthreads();
    if (!is_last) break;
    __threadfence();
    ++level;
    idx = parent;
  }
}

// Explicit Q of every tree node, all levels at once (the up-sweep left the
// reflectors in each node's tile): one CTA per node.
__global__ void __launch_bounds__(kThreads, 1) tsqr_q_kernel(const TsqrPlan plan, double* A,
                                                             long lda, double* ws) {
  extern __shared__ __align__(16) double q_smem[];
  TileSmem& sm = *reinterpret_cast<TileSmem*>(q_smem);
  int idx = blockIdx.x, level = 0;
  while (level < plan.nlev && idx >= plan.T[level]) {
    idx -= plan.T[level];
    ++level;
  }
  if (level >= plan.nlev) return;
  double* src;
  long ld;
  if (level == 0) {
    src = A + (long)idx * kTile;
    ld = lda;
  } else {
    src = ws + plan.soff[level] + (long)idx * kTile;
    ld = plan.rows[level];
  }
  const int mm = min(kTile, plan.rows[level] - idx * kTile);
  tile_form_q(src, ld, mm, sm, (level == 0 && idx == 0) ? ws + plan.qtop_off : nullptr);
}

struct FinishSmem {
  double M[kNB * (kNB + 1)];
  double T[kNB * (kNB + 1)];
  double B[kNB * (kNB + 1)];
  double LU[kNB * (kNB + 1)];
};

// C = Bm * M (32x32x32) into Out (all padded stride 33), 256 threads.
__device__ void mul32(const double* Bm, const double* M, double* Out) {
  for (int e = threadIdx.x; e < kNB * kNB; e += kThreads) {
    int r = e & 31, c = e >> 5;
    double s = 0.0;
#pragma unroll 8
    for (int k = 0; k < kNB; ++k) s = fma(Bm[r * 33 + k], M[k * 33 + c], s);
    Out[r * 33 + c] = s;
  }
}

// Path product for leaf tile t: M = B_1 (B_2 (... B_top)) with
// B_L = S_L[32*idx_{L-1} : +32, :].  Result in sm.M.
__device__ void path_product(const TsqrPlan& plan, const double* ws, int t, FinishSmem& sm) {
  int idxs[kMaxLevels];
  idxs[0] = t;
  for (int L = 1; L < plan.nlev; ++L) idxs[L] = idxs[L - 1] / kFan;
  for (int e = threadIdx.x; e < kNB * kNB; e += kThreads) {
    int r = e & 31, c = e >> 5;
    sm.M[r * 33 + c] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int L = plan.nlev - 1; L >= 1; --L) {
    const double* S = ws + plan.soff[L];
    long ld = plan.rows[L];
    long r0 = (long)kNB * idxs[L - 1];
    for (int e = threadIdx.x; e < kNB * kNB; e += kThreads) {
      int r = e & 31, c = e >> 5;
      sm.B[r * 33 + c] = __ldcg(S + r0 + r + (long)c * ld);
    }
    __syncthreads();
    mul32(sm.B, sm.M, sm.T);
    __syncthreads();
    for (int e = threadIdx.x; e < kNB * kNB; e += kThreads) {
      int r = e & 31, c = e >> 5;
      sm.M[r * 33 + c] = sm.T[r * 33 + c];
    }
    __syncthreads();
  }
}

// mode 0: write the explicit thin Q into A (evd_tsqr).
// mode 1: write Y (into Yout), W (into Wout), and optionally the band panel
//         (R over zeros) into Aband (sy2sb).
__global__ void __launch_bounds__(kThreads, 1)
    tsqr_finish_kernel(const TsqrPlan plan, const double* ws, double* A, long lda, int mode,
                       double* Yout, long ldy, double* Wout, long ldw, const double* Rin,
                       long ldr, double* Aband, long ldband) {
  extern __shared__ double dsm[];
  __shared__ FinishSmem sm;
  double* Qs = dsm;                   // 128 x 33 : rows of Q (then Y)
  double* Ws = dsm + kSub * 33;       // 128 x 33 : W rows
  const int t = blockIdx.x;
  const int r0 = t * kSub;
  const int mm = min(kSub, plan.m - r0);
  const int leaf = r0 / kTile;       // TSQR leaf tile holding these rows

  // tile rows of Q = Qleaf_t * M_t; the leaf Q tile is staged in shared
  // memory (coalesced) before the product
  for (int e = threadIdx.x; e < kSub * kNB; e += kThreads) {
    int r = e & (kSub - 1), c = e >> 7;
    Ws[r * 33 + c] = (r < mm) ? __ldcg(A + (long)(r0 + r) + (long)c * lda) : 0.0;
  }
  path_product(plan, ws, leaf, sm);  // ends with __syncthreads
  for (int e = threadIdx.x; e < kSub * kNB; e += kThreads) {
    int r = e & (kSub - 1), c = e >> 7;
    double s = 0.0;
#pragma unroll 8
    for (int k = 0; k < kNB; ++k) s = fma(Ws[r * 33 + k], sm.M[k * 33 + c], s);
    Qs[r * 33 + c] = s;
  }
  __syncthreads();

  if (mode == 0) {
    for (int e = threadIdx.x; e < kSub * kNB; e += kThreads) {
      int r = e & (kSub - 1), c = e >> 7;
      if (r < mm) A[(long)(r0 + r) + (long)c * lda] = Qs[r * 33 + c];
    }
    return;
  }

  // LU of (I - Qtop), Qtop = Qleaf_0[0:32] * M_0 (recomputed by every CTA)
  if (leaf != 0) path_product(plan, ws, 0, sm);
  {
    const double* q0 = ws + plan.qtop_off;
    if (t == 0) {
      for (int e = threadIdx.x; e < kNB * kNB; e += kThreads) {
        int r = e & 31, c = e >> 5;
        sm.LU[r * 33 + c] = ((r == c) ? 1.0 : 0.0) - Qs[r * 33 + c];
      }
    } else {
      for (int e = threadIdx.x; e < kNB * kNB; e += kThreads) {
        int r = e & 31, c = e >> 5;
        double s = 0.0;
#pragma unroll 8
        for (int k = 0; k < kNB; ++k) s = fma(__ldcg(q0 + r + k * kNB), sm.M[k * 33 + c], s);
        sm.LU[r * 33 + c] = ((r == c) ? 1.0 : 0.0) - s;
      }
    }
  }
  __syncthreads();
  // unpivoted LU in place (one warp, lane = row, the row in registers; row k
  // is broadcast by shuffles)
  if (threadIdx.x < 32) {
    const int r = threadIdx.x;
    double lu[kNB];
#pragma unroll
    for (int c = 0; c < kNB; ++c) lu[c] = sm.LU[r * 33 + c];
#pragma unroll
    for (int k = 0; k < kNB; ++k) {
      const double piv = __shfl_sync(0xffffffffu, lu[k], k);
      const double l = lu[k] / piv;
      if (r > k) lu[k] = l;
#pragma unroll
      for (int c = k + 1; c < kNB; ++c) {
        const double ukc = __shfl_sync(0xffffffffu, lu[c], k);
        if (r > k) lu[c] = fma(-l, ukc, lu[c]);
      }
    }
#pragma unroll
    for (int c = 0; c < kNB; ++c) sm.LU[r * 33 + c] = lu[c];
  }
  __syncthreads();

  // per row: iq = e_gr - q ;  even thread -> Y row, odd thread -> W row
  const int row = threadIdx.x >> 1;
  const bool doW = threadIdx.x & 1;
  double x[kNB];
  if (row < mm) {
    const int gr = r0 + row;
#pragma unroll
    for (int h = 0; h < kNB; ++h) x[h] = ((gr == h) ? 1.0 : 0.0) - Qs[row * 33 + h];
    if (!doW) {
      if (gr < kNB) {
#pragma unroll
        for (int h = 0; h < kNB; ++h) x[h] = (h < gr) ? sm.LU[gr * 33 + h] : ((h == gr) ? 1.0 : 0.0);
      } else {
        // y U = iq  (U upper, non-unit)
#pragma unroll
        for (int h = 0; h < kNB; ++h) {
          double s = x[h];
#pragma unroll
          for (int k = 0; k < h; ++k) s = fma(-x[k], sm.LU[k * 33 + h], s);
          x[h] = s / sm.LU[h * 33 + h];
        }
      }
    } else {
      // w L1^T = iq  (L1 unit lower): w_j = iq_j - sum_{k<j} L1[j,k] w_k
#pragma unroll
      for (int h = 0; h < kNB; ++h) {
        double s = x[h];
#pragma unroll
        for (int k = 0; k < h; ++k) s = fma(-sm.LU[h * 33 + k], x[k], s);
        x[h] = s;
      }
    }
  }
  __syncthreads();
  if (row < mm) {
    double* dst = doW ? Ws : Qs;
#pragma unroll
    for (int h = 0; h < kNB; ++h) dst[row * 33 + h] = x[h];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kSub * kNB; e += kThreads) {
    int r = e & (kSub - 1), c = e >> 7;
    if (r < mm) {
      long gr = r0 + r;
      Yout[gr + (long)c * ldy] = Qs[r * 33 + c];
      Wout[gr + (long)c * ldw] = Ws[r * 33 + c];
      if (Aband) {
        double v = 0.0;
        if (gr < kNB && c >= gr) v = __ldcg(Rin + gr + (long)c * ldr);
        Aband[gr + (long)c * ldband] = v;
      }
    }
  }
}

constexpr size_t kFinishDyn = 2 * kSub * 33 * sizeof(double);

int finish_attr() {
  EVD_TRY(smem_attr_once((const void*)tsqr_finish_kernel, (int)kFinishDyn));
  EVD_TRY(smem_attr_once((const void*)tsqr_up_kernel, (int)kTileSmem));
  EVD_TRY(smem_attr_once((const void*)tsqr_q_kernel, (int)kTileSmem));
  return EVD_SUCCESS;
}

}  // namespace

long panel_qr_ws_doubles(long m) { return make_plan(m).total; }

int panel_qr_check(long m, long n, long lda) {
  if (n != kNB || m < kNB || (m % kNB) != 0 || lda < m) return EVD_ERR_INVALID_ARG;
  if (m > (1L << 30)) return EVD_ERR_INVALID_ARG;
  return EVD_SUCCESS;
}

int panel_counters_reset(long m, double* ws, cudaStream_t st) {
  TsqrPlan plan = make_plan(m);
  if (plan.ncnt > 0)
    EVD_CUDA_TRY(cudaMemsetAsync(ws + plan.cnt_off, 0, sizeof(int) * plan.ncnt, st));
  return EVD_SUCCESS;
}

int panel_qr_launch(long m, double* A, long lda, double* ws, int mode, double* Yout, long ldy,
                    double* Wout, long ldw, double* R, long ldr, double* Aband, long ldband,
                    cudaStream_t st) {
  TsqrPlan plan = make_plan(m);
  if (plan.nlev >= kMaxLevels) return EVD_ERR_INVALID_ARG;
  EVD_TRY(finish_attr());
  tsqr_up_kernel<<<plan.T[0], kThreads, kTileSmem, st>>>(plan, A, lda, ws, R, ldr);
  EVD_LAUNCHED();
  int nodes = 0;
  for (int l = 0; l < plan.nlev; ++l) nodes += plan.T[l];
  tsqr_q_kernel<<<nodes, kThreads, kTileSmem, st>>>(plan, A, lda, ws);
  EVD_LAUNCHED();
  tsqr_finish_kernel<<<ceil_div_i(m, kSub), kThreads, kFinishDyn, st>>>(
      plan, ws, A, lda, mode, Yout, ldy, Wout, ldw, R, ldr, Aband, ldband);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

}  // namespace evd

extern "C" long evd_panel_qr_work_size(long m, long n) {
  if (evd::panel_qr_check(m, n, m) != EVD_SUCCESS) return 0;
  return evd::panel_qr_ws_doubles(m);
}

extern "C" int evd_tsqr(long m, long n, double* A, long lda, double* R, long ldr, double* work,
                        long lwork, cudaStream_t stream) {
  EVD_TRY(evd::panel_qr_check(m, n, lda));
  if (!A || !R || !work || ldr < n) return EVD_ERR_INVALID_ARG;
  if (lwork < evd::panel_qr_ws_doubles(m)) return EVD_ERR_WORKSPACE;
  EVD_TRY(evd::panel_counters_reset(m, work, stream));
  return evd::panel_qr_launch(m, A, lda, work, 0, nullptr, 0, nullptr, 0, R, ldr, nullptr, 0,
                              stream);
}

extern "C" int evd_panel_qr(long m, long n, double* A, long lda, double* W, long ldw, double* R,
                            long ldr, double* work, long lwork, cudaStream_t stream) {
  EVD_TRY(evd::panel_qr_check(m, n, lda));
  if (!A || !W || !R || !work || ldr < n || ldw < m) return EVD_ERR_INVALID_ARG;
  if (lwork < evd::panel_qr_ws_doubles(m)) return EVD_ERR_WORKSPACE;
  EVD_TRY(evd::panel_counters_reset(m, work, stream));
  return evd::panel_qr_launch(m, A, lda, work, 1, A, lda, W, ldw, R, ldr, nullptr, 0, stream);
}
