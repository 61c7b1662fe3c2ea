// Stage-2 back transformation: apply the bulge-chasing reflectors to a block
// of vectors.
//
// Reflector (s, k) of sweep s, step k covers rows p = s+1+32k .. p+31 and is
// stored in U(p:p+32, s) (zero where the sweep stored nothing).  With
// Q2 = prod_s prod_k H_{s,k} (generation order):
//   forward  (evd_bc_back, the reference's my_BC_back_trans_v8_10_noBandU,
//             api/BC_backTransV8_10_noBandU.cu:60-313):  X <- Q2^T X
//   reverse  (evd_bc_back_apply, the eigenvector direction): X <- Q2 X
//
// Ordering.  Rows are cut into 128-row strips R = 0, 128, ...  In strip R
// sweep h touches exactly rows [R+h+1, R+h+129) (4 reflectors, k = R/32 ..
// R/32+3).  Strips run bottom-up (forward) or top-down (reverse); that
// respects the generation order because the overlap of strip R's sweep h with
// strip R+-128 occurs only for sweeps on the correct side.
//
// Blocking (B200 design, not the reference's).  Inside a strip, sweeps are
// taken 8 at a time (block bb: sweeps 8bb..8bb+7).  The 8 reflectors of one
// block on segment j form a "group": they live in the 40-row parallelogram
// starting at row R+8bb+1+32j, reflector p on rows p..p+31 of it.  Two
// reflectors of different groups of a block overlap only if their segments
// are adjacent, and then the one on the lower segment comes first in
// generation order, so a block is applied group by group from the bottom
// segment up (forward; top-down and block order reversed for reverse).  A
// group is applied as one compact-WY update on the FP64 tensor cores:
//   Y (40 x 8, zero outside the parallelogram), T = (I + striu(Y^T Y))^-1
//   (unit upper triangular; every stored reflector has tau = 1),
//   forward X <- X - Y T^T (Y^T X),  reverse X <- X - Y T (Y^T X),
// as DMMA m16n8k8 products with X^T in the accumulator layout: a warp owns 16
// columns and keeps the block's 17 x 8-row window in registers; the
// accumulator layout of an 8-row tile doubles as the A operand of the next
// product (the k index is permuted to rows 0,2,4,6,1,3,5,7 and the B operand
// is read with the same permutation), so the window is never shuffled.
// T (Y^T Y by m8n8k4, then a triangular solve by 8 lanes) is either built,
// together with V = Y T^T (forward) or Y T (reverse), by a separate fully
// parallel kernel into a caller workspace before the apply kernel runs
// (q2_tbuild_kernel; the apply kernel then stages -V with the reflectors and
// updates X^T += W (-V)^T, with no T product), or, without a workspace,
// built inside the apply kernel one block ahead.  U is staged by cp.async into zero-padded, bank-conflict-free
// segments three blocks deep.  Work: the
// 2 n^2 ncols flops of the reflector algebra are done as 2.75 n^2 ncols on
// the DMMA pipe (parallelogram padding 40/32, plus the T product), plus the
// Gram products.  Rows >= n are never read or written (the reference needs
// 346 zero rows of padding).
#include "common.cuh"

namespace evd {

namespace {

constexpr int kQW = 4;                   // warps per CTA
constexpr int kQCols = 16;               // columns per warp (MMA M)
constexpr int kQThreads = kQW * 32;
constexpr int kStrip = 128;              // strip height (rows)
constexpr int kGroups = kStrip / 32;     // segments (groups) per block
constexpr int kTiles = 4 * kGroups + 1;  // 8-row tiles in a block's window (135 rows used)
constexpr int kSeg = 64;                 // smem slots per (sweep, segment): 8 + 32 + 8 used
constexpr int kYBuf = 8 * kGroups * kSeg;  // 8 sweeps x kGroups segments
constexpr int kNYBuf = 3;
constexpr int kTBuf = kGroups * 32 * 2;  // per group: 32 lanes x 2 B-fragment values
constexpr int kVGroup = 5 * 32 * 2;      // per group: 5 tiles x 32 lanes x 2 B-fragment values
constexpr int kVBuf = kGroups * kVGroup;
constexpr int kGBuf = 64;                // per warp: one 8 x 8 Gram matrix
constexpr size_t kQSmem = (size_t)(kNYBuf * kYBuf + kNYBuf * kVBuf + kQW * kGBuf) * sizeof(double);
static_assert(kGroups == kQW, "one warp builds the T of one group");

__device__ __forceinline__ void cp_async8_zfill(double* smem, const double* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
               "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async16(double* smem, const double* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mma16(double (&d)[4], double a0, double a1, double a2, double a3,
                                      double b0, double b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}
__device__ __forceinline__ void mma8(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// Segment (sweep p, segment j) of a staged block: Y_j[r][p] is at
// seg_off(p, j) + r - p for r - p in [-8, 40) (zero outside [0, 32)).  The
// offset 10 * ((p >> 1) & 1) makes both fragment read patterns below
// conflict-free (each half-warp hits 16 distinct 8-byte banks).
__device__ __forceinline__ int seg_off(int p, int j) {
  return (p * kGroups + j) * kSeg + 10 * ((p >> 1) & 1) + 8;
}

// Stage block bb of strip R: Y values of sweeps 8bb..8bb+7 (zero for sweep
// >= H or row >= n).  Element i of sweep p's strip window goes to segment
// i / 32, offset i % 32.
__device__ __forceinline__ void stage_block(double* ys, const double* U, long ldU, int n, long R,
                                            int H, int bb) {
  for (int e = threadIdx.x; e < 8 * kStrip; e += kQThreads) {
    const int p = e / kStrip, i = e % kStrip;
    const int h = 8 * bb + p;
    const long row = R + h + 1 + i;
    const bool valid = (h < H) && (row < n);
    const double* src = valid ? (U + row + (long)h * ldU) : U;
    cp_async8_zfill(ys + seg_off(p, i >> 5) + (i & 31), src, valid);
  }
}

// -T fragment of group w of a staged block (warp w).  G = Y^T Y by DMMA (the
// Y fragment is both operands), then lane q solves (I + striu(G)) t = e_q for
// column q of T, and stores -T as the B operand of the W <- W T (forward:
// B[k][n] = T[k][n]) or W <- W T^T (reverse) product, k permuted as in the
// window tiles.
template <bool FWD>
__device__ __forceinline__ void build_t(const double* ys, double* ts, double* gs, int warp,
                                        int lane, int offW) {
  const int j = warp;
  {
    double ga[2] = {0.0, 0.0}, gb[2] = {0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const double y0 = ys[offW + j * kSeg + 8 * i];
      const double y1 = ys[offW + j * kSeg + 8 * i + 1];
      mma8(ga, y0, y0);
      mma8(gb, y1, y1);
    }
    const int g = lane >> 2, t = lane & 3;
    gs[g * 8 + 2 * t] = ga[0] + gb[0];
    gs[g * 8 + 2 * t + 1] = ga[1] + gb[1];
  }
  __syncwarp();
  if (lane < 8) {
    const int q = lane;
    const double* G = gs;
    double tq[8];
#pragma unroll
    for (int i = 7; i >= 0; --i) {
      double acc = 0.0;
#pragma unroll
      for (int k = i + 1; k < 8; ++k) acc = fma(G[i * 8 + k], tq[k], acc);
      tq[i] = (i < q) ? -acc : (i == q ? 1.0 : 0.0);
    }
    double* dst = ts + j * 64;
    if (FWD) {
      // lane (g, t) of the product needs T[2t][g], T[2t+1][g]: column g = q
#pragma unroll
      for (int t2 = 0; t2 < 4; ++t2) {
        dst[(4 * q + t2) * 2 + 0] = -tq[2 * t2];
        dst[(4 * q + t2) * 2 + 1] = -tq[2 * t2 + 1];
      }
    } else {
      // lane (g, t) needs T[g][2t], T[g][2t+1]: row g, columns 2t, 2t+1
#pragma unroll
      for (int i = 0; i < 8; ++i) dst[(4 * i + (q >> 1)) * 2 + (q & 1)] = -tq[i];
    }
  }
}

// -V fragments of group w of a staged block (warp w), V = Y T^T (forward) or
// Y T (reverse), so that the update X^T += W (-V)^T needs no T product:
// lane (g, t) of tile i gets (-V[8i+g][2t], -V[8i+g][2t+1]).  T comes from
// build_t's Gram/triangular solve (written to gs as T[i][q] at gs[i*8+q]).
template <bool FWD>
__device__ __forceinline__ void build_v(const double* ys, double* vs, double* gs, int warp,
                                        int lane, int offW) {
  const int j = warp;
  {
    double ga[2] = {0.0, 0.0}, gb[2] = {0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const double y0 = ys[offW + j * kSeg + 8 * i];
      const double y1 = ys[offW + j * kSeg + 8 * i + 1];
      mma8(ga, y0, y0);
      mma8(gb, y1, y1);
    }
    const int g = lane >> 2, t = lane & 3;
    gs[g * 8 + 2 * t] = ga[0] + gb[0];
    gs[g * 8 + 2 * t + 1] = ga[1] + gb[1];
  }
  __syncwarp();
  double tq[8];
  if (lane < 8) {
    const int q = lane;
#pragma unroll
    for (int i = 7; i >= 0; --i) {
      double acc = 0.0;
#pragma unroll
      for (int k = i + 1; k < 8; ++k) acc = fma(gs[i * 8 + k], tq[k], acc);
      tq[i] = (i < q) ? -acc : (i == q ? 1.0 : 0.0);
    }
  }
  __syncwarp();
  if (lane < 8) {
#pragma unroll
    for (int i = 0; i < 8; ++i) gs[i * 8 + lane] = tq[i];  // T[i][q]
  }
  __syncwarp();
  const int g = lane >> 2, t = lane & 3;
  double* dst = vs + j * kVGroup;
#pragma unroll
  for (int i = 0; i < 5; ++i) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = 8 * i + g, p = 2 * t + h;
      double v = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const double y = ys[seg_off(q, j) + r - q];  // zero outside the parallelogram
        const double tv = FWD ? gs[p * 8 + q] : gs[q * 8 + p];
        v = fma(y, tv, v);
      }
      dst[(i * 32 + lane) * 2 + h] = -v;
    }
  }
}

// Blocks of all strips, strip-major: strip s has nblk(s) = B0 - 16 s blocks
// (B0 = ceil((n-2)/8); every strip height is a multiple of 8 rows), so the
// precomputed fragments of block bb of strip s start at tblock(s, bb) * kVBuf.
__host__ __device__ __forceinline__ long tblock(long s, long bb, long B0) {
  return s * B0 - 8 * s * (s - 1) + bb;
}

// Sweeps [h0, h1) of the chase (h0 a multiple of 8; h1 a multiple of 8 or at
// least n - 2): the blocks of those sweeps in every strip.  Splitting the
// sweeps into consecutive ranges, each applied to all strips, keeps the
// generation order: every reflector of a range precedes, in that order,
// every reflector of a later range that it overlaps.
// ident (forward only): X was the identity before sweep k = ident_k (k <= h0).
// Then column c is zero below row c + 30 + (h - k) before sweep h (each sweep
// moves the lowest nonzero row of a column down by at most one after the
// first), and sweep h touches rows >= R + h + 1 of strip R, so a strip with
// R > c + 29 - k never meets a nonzero of column c: a CTA skips the strips
// that lie wholly below its columns (with a margin of 64 rows).
struct Q2Range {
  int h0, h1, ident, ident_k;
  int rev;  // CTA b takes column block gridDim.x - 1 - b (the heaviest first)
};

// Strips 0 .. q2_strips() - 1 are the ones a CTA processes: those with a
// block of the range's sweeps (R < n - 2 - h0) and, from the identity, not
// wholly below the CTA's columns (R <= first column + columns + 64 - k).
// Both conditions bound R from above, so the strips form a prefix.
__host__ __device__ __forceinline__ int q2_strips(const Q2Range& rg, int n, int nstrips,
                                                  long cta_col0, int cta_cols) {
  long rmax = (long)n - 3 - rg.h0;
  if (rg.ident) rmax = min(rmax, cta_col0 + cta_cols + 64 - (long)rg.ident_k);
  if (rmax < 0) return 0;
  return (int)min((long)nstrips, rmax / kStrip + 1);
}

// -V fragments of every block of every strip (one CTA per block, one warp
// per group), in the layout the apply kernel reads.
template <bool FWD>
__global__ void __launch_bounds__(kQThreads)
    q2_tbuild_kernel(int n, const double* __restrict__ U, long ldU, double* __restrict__ Tg,
                     int bb0) {
  __shared__ __align__(16) double ys[kYBuf];
  __shared__ double gsh[kQW * kGBuf];
  const int s = blockIdx.y, bb = bb0 + (int)blockIdx.x;
  const int B0 = (n - 2 + 7) / 8;
  const int nblk = B0 - (kStrip / 8) * s;
  if (bb >= nblk) return;
  const long R = (long)s * kStrip;
  const int H = n - 2 - (int)R;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  for (int e = threadIdx.x; e < kYBuf; e += kQThreads) ys[e] = 0.0;
  __syncthreads();
  stage_block(ys, U, ldU, n, R, H, bb);
  cp_commit();
  cp_wait<0>();
  __syncthreads();
  build_v<FWD>(ys, Tg + tblock(s, bb, B0) * kVBuf, gsh + warp * kGBuf, warp, lane,
               seg_off(g, 0) + 2 * t - g);
}

// W += X^T Y over tiles i in [i0, i1) of group J (two accumulator chains by
// tile parity).
__device__ __forceinline__ void w_part(const double (&x)[kTiles][4], const double* ys, int offW,
                                       int J, int i0, int i1, double (&wa)[4], double (&wb)[4]) {
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    if (i < i0 || i >= i1) continue;
    const int ti = 4 * J + i;
    const double b0 = ys[offW + J * kSeg + 8 * i];
    const double b1 = ys[offW + J * kSeg + 8 * i + 1];
    if (i & 1)
      mma16(wb, x[ti][0], x[ti][2], x[ti][1], x[ti][3], b0, b1);
    else
      mma16(wa, x[ti][0], x[ti][2], x[ti][1], x[ti][3], b0, b1);
  }
}

// One block: its 4 groups in dependency order (segments 3..0 forward, 0..3
// reverse), each W = X^T Y, W <- W (-T or -T^T), X^T += W Y^T.  Consecutive
// groups share one tile (forward: tile 4J = the next group's last tile;
// reverse: tile 4J+4 = the next group's first), so the next group's W over
// its other four tiles is issued between this group's T product and its
// update, and the shared tile is updated first.
template <bool FWD, bool VPRE>
__device__ __forceinline__ void apply_block(double (&x)[kTiles][4], const double* ys,
                                            const double* ts, int lane, int offW, int offU0,
                                            int offU1) {
  double wa[4] = {0.0, 0.0, 0.0, 0.0}, wb[4] = {0.0, 0.0, 0.0, 0.0};
  w_part(x, ys, offW, FWD ? kGroups - 1 : 0, 0, 5, wa, wb);
#pragma unroll
  for (int s = 0; s < kGroups; ++s) {
    const int J = FWD ? kGroups - 1 - s : s;
    const int JN = FWD ? J - 1 : J + 1;
#pragma unroll
    for (int q = 0; q < 4; ++q) wa[q] += wb[q];
    double wt[4] = {0.0, 0.0, 0.0, 0.0};
    if (VPRE) {
#pragma unroll
      for (int q = 0; q < 4; ++q) wt[q] = wa[q];  // the update reads -V instead of -T Y^T
    } else {
      const double2 tf = *reinterpret_cast<const double2*>(ts + J * 64 + lane * 2);
      mma16(wt, wa[0], wa[2], wa[1], wa[3], tf.x, tf.y);
    }
    double na[4] = {0.0, 0.0, 0.0, 0.0}, nb[4] = {0.0, 0.0, 0.0, 0.0};
    if (s + 1 < kGroups) w_part(x, ys, offW, JN, FWD ? 0 : 1, FWD ? 4 : 5, na, nb);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const int i = FWD ? k : 4 - k;  // shared tile first
      const int ti = 4 * J + i;
      double b0, b1;
      if (VPRE) {
        const double2 vf = *reinterpret_cast<const double2*>(ts + J * kVGroup + (i * 32 + lane) * 2);
        b0 = vf.x;
        b1 = vf.y;
      } else {
        b0 = ys[offU0 + J * kSeg + 8 * i];
        b1 = ys[offU1 + J * kSeg + 8 * i];
      }
      mma16(x[ti], wt[0], wt[2], wt[1], wt[3], b0, b1);
    }
    if (s + 1 < kGroups) {
      w_part(x, ys, offW, JN, FWD ? 4 : 0, FWD ? 5 : 1, na, nb);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        wa[q] = na[q];
        wb[q] = nb[q];
      }
    }
  }
}

// Window tile i of a frame starting at row `base`: rows base+8i .. base+8i+7.
// Lane (g, t) holds X(rows 2t, 2t+1 of the tile; columns g, g+8 of the warp).
struct TileIO {
  double* cg;   // column c0+g (or a dummy)
  double* cg8;  // column c0+g+8
  bool okg, okg8;
  int t2;
};

__device__ __forceinline__ void load_tile(double (&v)[4], const TileIO& io, long row0, int n) {
  const long r = row0 + io.t2;
  const bool r0 = r >= 0 && r < n, r1 = r + 1 >= 0 && r + 1 < n;
  v[0] = (io.okg && r0) ? io.cg[r] : 0.0;
  v[1] = (io.okg && r1) ? io.cg[r + 1] : 0.0;
  v[2] = (io.okg8 && r0) ? io.cg8[r] : 0.0;
  v[3] = (io.okg8 && r1) ? io.cg8[r + 1] : 0.0;
}
__device__ __forceinline__ void store_tile(const double (&v)[4], const TileIO& io, long row0,
                                           int n) {
  const long r = row0 + io.t2;
  const bool r0 = r >= 0 && r < n, r1 = r + 1 >= 0 && r + 1 < n;
  if (io.okg && r0) io.cg[r] = v[0];
  if (io.okg && r1) io.cg[r + 1] = v[1];
  if (io.okg8 && r0) io.cg8[r] = v[2];
  if (io.okg8 && r1) io.cg8[r + 1] = v[3];
}

// PRE: the -T fragments were precomputed into Tg by q2_tbuild_kernel and are
// staged with the reflectors; otherwise each block's T is built here, one
// block ahead, by the same warps.  rg restricts the kernel to a range of
// sweeps (and marks an identity start, see Q2Range).
template <bool FWD, bool PRE, bool RANGE>
__global__ void __launch_bounds__(kQThreads, 2)
    q2_mma_kernel(int n, int ncols, const double* __restrict__ U, long ldU,
                  const double* __restrict__ Tg, double* __restrict__ X, long ldX, Q2Range rg) {
  extern __shared__ __align__(16) double smem[];
  double* Ys = smem;                 // kNYBuf x kYBuf
  double* Ts = Ys + kNYBuf * kYBuf;  // kNYBuf x kVBuf (PRE: -V) or 2 x kTBuf (-T)
  double* Gs = Ts + kNYBuf * kVBuf;  // kQW x kGBuf
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  double* gs = Gs + warp * kGBuf;

  // the zero padding of the staged segments is written once; staging never
  // touches it
  for (int e = threadIdx.x; e < kNYBuf * kYBuf; e += kQThreads) Ys[e] = 0.0;

  // per-lane fragment offsets (segment 0 of the block)
  const int offW = seg_off(g, 0) + 2 * t - g;               // Y[8i+2t(+1)][g]
  const int offU0 = seg_off(2 * t, 0) + g - 2 * t;          // Y[8i+g][2t]
  const int offU1 = seg_off(2 * t + 1, 0) + g - 2 * t - 1;  // Y[8i+g][2t+1]

  // RANGE = false: every sweep, no identity start (the plain solve's launch)
  const int cblk = (RANGE && rg.rev) ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
  const int c0 = cblk * (kQW * kQCols) + warp * kQCols;
  TileIO io;
  io.okg = c0 + g < ncols;
  io.okg8 = c0 + g + 8 < ncols;
  io.cg = X + (long)(io.okg ? c0 + g : 0) * ldX;
  io.cg8 = X + (long)(io.okg8 ? c0 + g + 8 : 0) * ldX;
  io.t2 = 2 * t;

  double x[kTiles][4];
  const int nstrips = (n - 2 + kStrip - 1) / kStrip;
  const int B0 = (n - 2 + 7) / 8;
  // stage the -V fragments of block bb of strip sidx (16-byte copies)
  auto stage_t = [&](double* dst, int sidx, int bb) {
    const double* src = Tg + tblock(sidx, bb, B0) * kVBuf;
    for (int e = threadIdx.x; e < kVBuf / 2; e += kQThreads) cp_async16(dst + 2 * e, src + 2 * e);
  };
  const long cta_col0 = (long)cblk * (kQW * kQCols);
  const int ns = RANGE ? q2_strips(rg, n, nstrips, cta_col0, kQW * kQCols) : nstrips;
  for (int si = 0; si < ns; ++si) {
    const int sidx = FWD ? (ns - 1 - si) : si;
    const long R = (long)sidx * kStrip;
    const int H = n - 2 - (int)R;  // sweeps with reflectors in this strip
    const int nblk = (H + 7) / 8;
    const int bbA = RANGE ? rg.h0 / 8 : 0, bbB = RANGE ? min(nblk, (rg.h1 + 7) / 8) : nblk;
    const int cnt = bbB - bbA;  // blocks of this launch's sweeps in the strip (>= 1)
    auto bb_of = [&](int it) { return FWD ? (bbA + it) : (bbB - 1 - it); };

    __syncthreads();  // previous strip done with Ys / Ts; zero fill visible
    {
      const long base = R + 8L * bb_of(0) + 1;
#pragma unroll
      for (int i = 0; i < kTiles; ++i) load_tile(x[i], io, base + 8 * i, n);
    }
    stage_block(Ys, U, ldU, n, R, H, bb_of(0));
    if (PRE) stage_t(Ts, sidx, bb_of(0));
    cp_commit();
    if (cnt > 1) {
      stage_block(Ys + kYBuf, U, ldU, n, R, H, bb_of(1));
      if (PRE) stage_t(Ts + kVBuf, sidx, bb_of(1));
    }
    cp_commit();
    cp_wait<1>();
    __syncthreads();
    if (!PRE) build_t<FWD>(Ys, Ts, gs, warp, lane, offW);

#pragma unroll 1
    for (int it = 0; it < cnt; ++it) {
      const int bb = bb_of(it);
      const long base = R + 8L * bb + 1;
      cp_wait<0>();
      __syncthreads();  // block it+1 staged; T of block it complete
      if (it + 2 < cnt) {
        stage_block(Ys + ((it + 2) % 3) * kYBuf, U, ldU, n, R, H, bb_of(it + 2));
        if (PRE) stage_t(Ts + ((it + 2) % 3) * kVBuf, sidx, bb_of(it + 2));
      }
      cp_commit();
      double inc[4];
      load_tile(inc, io, FWD ? (base + 8 * kTiles) : (base - 8), n);
      const double* ys = Ys + (it % 3) * kYBuf;
      const double* ts = Ts + (PRE ? (it % 3) * kVBuf : (it & 1) * kTBuf);
      if (!PRE && it + 1 < cnt)
        build_t<FWD>(Ys + ((it + 1) % 3) * kYBuf, Ts + ((it + 1) & 1) * kTBuf, gs, warp, lane,
                     offW);
      apply_block<FWD, PRE>(x, ys, ts, lane, offW, offU0, offU1);
      // slide the window one tile: the tile leaving it is final for this strip
      if (FWD) {
        store_tile(x[0], io, base, n);
#pragma unroll
        for (int i = 0; i + 1 < kTiles; ++i)
#pragma unroll
          for (int q = 0; q < 4; ++q) x[i][q] = x[i + 1][q];
#pragma unroll
        for (int q = 0; q < 4; ++q) x[kTiles - 1][q] = inc[q];
      } else {
        store_tile(x[kTiles - 1], io, base + 8 * (kTiles - 1), n);
#pragma unroll
        for (int i = kTiles - 1; i > 0; --i)
#pragma unroll
          for (int q = 0; q < 4; ++q) x[i][q] = x[i - 1][q];
#pragma unroll
        for (int q = 0; q < 4; ++q) x[0][q] = inc[q];
      }
    }
    // the window now holds the frame one block past the last one
    {
      const long base = FWD ? (R + 8L * bbB + 1) : (R + 8L * bbA - 7);
#pragma unroll
      for (int i = 0; i < kTiles; ++i) store_tile(x[i], io, base + 8 * i, n);
    }
  }
}

// ---- 8-column warps (m8n8k4), precomputed -V fragments ----
// The same strips, blocks, group order and staged fragments as q2_mma_kernel
// (PRE), with a warp owning 8 columns: the window tile (8 columns x 8 rows)
// is the m8n8k4 accumulator (lane (g, t): column g, rows 2t and 2t+1), which
// is the A operand of the W product for the rows {0, 2, 4, 6} (x[i][0]) and
// {1, 3, 5, 7} (x[i][1]) with the B operand read from the same staged
// reflector segments; W (column g, reflectors 2t, 2t+1) is in turn the A
// operand of the update for the even and odd reflectors against the -V
// fragments.  The window takes 68 registers instead of 136, so twice as many
// warps share each sub-partition's tensor pipe (the kernel above is bound by
// its dependent DMMA chains with two warps per sub-partition).
constexpr int kQ8Cols = 8;

__device__ __forceinline__ void w_part8(const double (&x)[kTiles][2], const double* ys, int offW,
                                        int J, int i0, int i1, double (&wa)[2],
                                        double (&wb)[2]) {
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    if (i < i0 || i >= i1) continue;
    const int ti = 4 * J + i;
    const double b0 = ys[offW + J * kSeg + 8 * i];
    const double b1 = ys[offW + J * kSeg + 8 * i + 1];
    if (i & 1) {
      mma8(wb, x[ti][0], b0);
      mma8(wb, x[ti][1], b1);
    } else {
      mma8(wa, x[ti][0], b0);
      mma8(wa, x[ti][1], b1);
    }
  }
}

template <bool FWD>
__device__ __forceinline__ void apply_block8(double (&x)[kTiles][2], const double* ys,
                                             const double* ts, int lane, int offW) {
  double wa[2] = {0.0, 0.0}, wb[2] = {0.0, 0.0};
  w_part8(x, ys, offW, FWD ? kGroups - 1 : 0, 0, 5, wa, wb);
#pragma unroll
  for (int s = 0; s < kGroups; ++s) {
    const int J = FWD ? kGroups - 1 - s : s;
    const int JN = FWD ? J - 1 : J + 1;
    const double wt0 = wa[0] + wb[0], wt1 = wa[1] + wb[1];
    double na[2] = {0.0, 0.0}, nb[2] = {0.0, 0.0};
    if (s + 1 < kGroups) w_part8(x, ys, offW, JN, FWD ? 0 : 1, FWD ? 4 : 5, na, nb);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const int i = FWD ? k : 4 - k;  // shared tile first
      const int ti = 4 * J + i;
      const double2 vf =
          *reinterpret_cast<const double2*>(ts + J * kVGroup + (i * 32 + lane) * 2);
      mma8(x[ti], wt0, vf.x);
      mma8(x[ti], wt1, vf.y);
    }
    if (s + 1 < kGroups) {
      w_part8(x, ys, offW, JN, FWD ? 4 : 0, FWD ? 5 : 1, na, nb);
      wa[0] = na[0];
      wa[1] = na[1];
      wb[0] = nb[0];
      wb[1] = nb[1];
    }
  }
}

__device__ __forceinline__ void load_tile8(double (&v)[2], const double* cg, bool ok, long row0,
                                           int t2, int n) {
  const long r = row0 + t2;
  v[0] = (ok && r >= 0 && r < n) ? cg[r] : 0.0;
  v[1] = (ok && r + 1 >= 0 && r + 1 < n) ? cg[r + 1] : 0.0;
}
__device__ __forceinline__ void store_tile8(const double (&v)[2], double* cg, bool ok, long row0,
                                            int t2, int n) {
  const long r = row0 + t2;
  if (ok && r >= 0 && r < n) cg[r] = v[0];
  if (ok && r + 1 >= 0 && r + 1 < n) cg[r + 1] = v[1];
}

template <bool FWD, int NW, bool RANGE>
__global__ void __launch_bounds__(NW * 32, 2)
    q2_mma8_kernel(int n, int ncols, const double* __restrict__ U, long ldU,
                   const double* __restrict__ Tg, double* __restrict__ X, long ldX, Q2Range rg) {
  extern __shared__ __align__(16) double smem[];
  double* Ys = smem;                 // kNYBuf x kYBuf
  double* Ts = Ys + kNYBuf * kYBuf;  // kNYBuf x kVBuf (-V fragments)
  const int nthr = NW * 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  for (int e = threadIdx.x; e < kNYBuf * kYBuf; e += nthr) Ys[e] = 0.0;
  const int offW = seg_off(g, 0) + 2 * t - g;  // Y[8i+2t(+1)][g]
  const int cblk = (RANGE && rg.rev) ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
  const int c0 = cblk * (NW * kQ8Cols) + warp * kQ8Cols;
  const bool okg = c0 + g < ncols;
  double* cg = X + (long)(okg ? c0 + g : 0) * ldX;
  const int t2 = 2 * t;

  double x[kTiles][2];
  const int nstrips = (n - 2 + kStrip - 1) / kStrip;
  const int B0 = (n - 2 + 7) / 8;
  auto stage_y = [&](double* ys, long R, int H, int bb) {
    for (int e = threadIdx.x; e < 8 * kStrip; e += nthr) {
      const int p = e / kStrip, i = e % kStrip;
      const int h = 8 * bb + p;
      const long row = R + h + 1 + i;
      const bool valid = (h < H) && (row < n);
      const double* src = valid ? (U + row + (long)h * ldU) : U;
      cp_async8_zfill(ys + seg_off(p, i >> 5) + (i & 31), src, valid);
    }
  };
  auto stage_t = [&](double* dst, int sidx, int bb) {
    const double* src = Tg + tblock(sidx, bb, B0) * kVBuf;
    for (int e = threadIdx.x; e < kVBuf / 2; e += nthr) cp_async16(dst + 2 * e, src + 2 * e);
  };
  const long cta_col0 = (long)cblk * (NW * kQ8Cols);
  const int ns = RANGE ? q2_strips(rg, n, nstrips, cta_col0, NW * kQ8Cols) : nstrips;
  for (int si = 0; si < ns; ++si) {
    const int sidx = FWD ? (ns - 1 - si) : si;
    const long R = (long)sidx * kStrip;
    const int H = n - 2 - (int)R;
    const int nblk = (H + 7) / 8;
    const int bbA = RANGE ? rg.h0 / 8 : 0, bbB = RANGE ? min(nblk, (rg.h1 + 7) / 8) : nblk;
    const int cnt = bbB - bbA;
    auto bb_of = [&](int it) { return FWD ? (bbA + it) : (bbB - 1 - it); };

    __syncthreads();
    {
      const long base = R + 8L * bb_of(0) + 1;
#pragma unroll
      for (int i = 0; i < kTiles; ++i) load_tile8(x[i], cg, okg, base + 8 * i, t2, n);
    }
    stage_y(Ys, R, H, bb_of(0));
    stage_t(Ts, sidx, bb_of(0));
    cp_commit();
    if (cnt > 1) {
      stage_y(Ys + kYBuf, R, H, bb_of(1));
      stage_t(Ts + kVBuf, sidx, bb_of(1));
    }
    cp_commit();
    cp_wait<1>();
    __syncthreads();

#pragma unroll 1
    for (int it = 0; it < cnt; ++it) {
      const int bb = bb_of(it);
      const long base = R + 8L * bb + 1;
      cp_wait<0>();
      __syncthreads();
      if (it + 2 < cnt) {
        stage_y(Ys + ((it + 2) % 3) * kYBuf, R, H, bb_of(it + 2));
        stage_t(Ts + ((it + 2) % 3) * kVBuf, sidx, bb_of(it + 2));
      }
      cp_commit();
      double inc[2];
      load_tile8(inc, cg, okg, FWD ? (base + 8 * kTiles) : (base - 8), t2, n);
      apply_block8<FWD>(x, Ys + (it % 3) * kYBuf, Ts + (it % 3) * kVBuf, lane, offW);
      if (FWD) {
        store_tile8(x[0], cg, okg, base, t2, n);
#pragma unroll
        for (int i = 0; i + 1 < kTiles; ++i) {
          x[i][0] = x[i + 1][0];
          x[i][1] = x[i + 1][1];
        }
        x[kTiles - 1][0] = inc[0];
        x[kTiles - 1][1] = inc[1];
      } else {
        store_tile8(x[kTiles - 1], cg, okg, base + 8 * (kTiles - 1), t2, n);
#pragma unroll
        for (int i = kTiles - 1; i > 0; --i) {
          x[i][0] = x[i - 1][0];
          x[i][1] = x[i - 1][1];
        }
        x[0][0] = inc[0];
        x[0][1] = inc[1];
      }
    }
    {
      const long base = FWD ? (R + 8L * bbB + 1) : (R + 8L * bbA - 7);
#pragma unroll
      for (int i = 0; i < kTiles; ++i) store_tile8(x[i], cg, okg, base + 8 * i, t2, n);
    }
  }
}

constexpr size_t kQ8Smem = (size_t)(kNYBuf * kYBuf + kNYBuf * kVBuf) * sizeof(double);

template <bool FWD, int NW, bool RANGE>
int launch_q2_8(long n, long ncols, const double* U, long ldU, const double* Tg, double* X,
                long ldX, Q2Range rg, cudaStream_t st) {
  EVD_TRY(smem_attr_once((const void*)q2_mma8_kernel<FWD, NW, RANGE>, (int)kQ8Smem));
  const int grid = ceil_div_i((int)ncols, NW * kQ8Cols);
  q2_mma8_kernel<FWD, NW, RANGE><<<grid, NW * 32, kQ8Smem, st>>>((int)n, (int)ncols, U, ldU, Tg,
                                                                 X, ldX, rg);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

template <bool FWD, bool PRE, bool RANGE>
int launch_q2(long n, long ncols, const double* U, long ldU, const double* Tg, double* X,
              long ldX, Q2Range rg, cudaStream_t st) {
  EVD_TRY(smem_attr_once((const void*)q2_mma_kernel<FWD, PRE, RANGE>, (int)kQSmem));
  int grid = ceil_div_i((int)ncols, kQW * kQCols);
  q2_mma_kernel<FWD, PRE, RANGE><<<grid, kQThreads, kQSmem, st>>>((int)n, (int)ncols, U, ldU, Tg,
                                                                  X, ldX, rg);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

// With fewer 64-column CTAs than SMs (ncols < 64 x SMs: n <= 8192 on B200)
// the 16-column kernel leaves SMs idle; the 8-column kernel (4 warps, 32
// columns per CTA) doubles the warps (n = 4096: 19.8 -> 14.0 ms).  Above that
// the 16-column kernel is faster (n = 16384: 436 ms against 461 ms with
// 8-column warps, whose m8n8k4 operands double the shared-memory reads per
// flop).  A launch over every sweep without an identity start takes the
// kernels compiled without the range logic.
template <bool FWD>
int launch_q2_pre(long n, long ncols, const double* U, long ldU, const double* Tg, double* X,
                  long ldX, Q2Range rg, cudaStream_t st) {
  const bool whole = !rg.ident && rg.h0 == 0 && rg.h1 >= n - 2;
  if (ncols >= 64L * device_sm_count())
    return whole ? launch_q2<FWD, true, false>(n, ncols, U, ldU, Tg, X, ldX, rg, st)
                 : launch_q2<FWD, true, true>(n, ncols, U, ldU, Tg, X, ldX, rg, st);
  return whole ? launch_q2_8<FWD, 4, false>(n, ncols, U, ldU, Tg, X, ldX, rg, st)
               : launch_q2_8<FWD, 4, true>(n, ncols, U, ldU, Tg, X, ldX, rg, st);
}

// -V fragments of the blocks of sweeps [h0, h1) in every strip.
template <bool FWD>
int launch_tbuild(long n, const double* U, long ldU, double* Tg, long h0, long h1,
                  cudaStream_t st) {
  const int nstrips = (int)((n - 2 + kStrip - 1) / kStrip);
  const int B0 = (int)((n - 2 + 7) / 8);
  const int bbA = (int)(h0 / 8), bbB = (int)std::min<long>(B0, (h1 + 7) / 8);
  if (bbB <= bbA) return EVD_SUCCESS;
  q2_tbuild_kernel<FWD><<<dim3(bbB - bbA, nstrips), kQThreads, 0, st>>>((int)n, U, ldU, Tg, bbA);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

}  // namespace

long q2_tbuf_doubles(long n) {
  if (n < 3) return 0;
  const long nstrips = (n - 2 + kStrip - 1) / kStrip;
  const long B0 = (n - 2 + 7) / 8;
  return tblock(nstrips, 0, B0) * kVBuf;
}

int q2_apply_range(bool forward, long n, long ncols, const double* U, long ldU, double* X,
                   long ldX, double* tbuf, long h0, long h1, long ident_k, cudaStream_t st) {
  const bool ident = ident_k >= 0;
  if (n < 0 || ncols < 0 || ldU < n || ldX < n) return EVD_ERR_INVALID_ARG;
  if (n > (1L << 30) || ncols > (1L << 30)) return EVD_ERR_INVALID_ARG;
  if (h0 < 0 || h0 % 8 != 0 || h1 < h0 || (h1 % 8 != 0 && h1 < n - 2)) return EVD_ERR_INVALID_ARG;
  if (ident && (!forward || ident_k > h0)) return EVD_ERR_INVALID_ARG;
  if (n < 3 || ncols == 0 || h0 >= n - 2 || h1 == h0) return EVD_SUCCESS;
  if (!U || !X) return EVD_ERR_INVALID_ARG;
  if (tbuf && ((uintptr_t)tbuf & 15)) return EVD_ERR_INVALID_ARG;
  // from the identity the work of a column block grows with its index: the
  // heaviest blocks are dispatched first
  const Q2Range rg{(int)h0, (int)std::min(h1, n), ident ? 1 : 0, ident ? (int)ident_k : 0,
                   ident ? 1 : 0};
  if (tbuf) {
    if (forward) {
      EVD_TRY(launch_tbuild<true>(n, U, ldU, tbuf, h0, h1, st));
      return launch_q2_pre<true>(n, ncols, U, ldU, tbuf, X, ldX, rg, st);
    }
    EVD_TRY(launch_tbuild<false>(n, U, ldU, tbuf, h0, h1, st));
    return launch_q2_pre<false>(n, ncols, U, ldU, tbuf, X, ldX, rg, st);
  }
  return forward ? launch_q2<true, false, true>(n, ncols, U, ldU, nullptr, X, ldX, rg, st)
                 : launch_q2<false, false, true>(n, ncols, U, ldU, nullptr, X, ldX, rg, st);
}

int q2_apply(bool forward, long n, long ncols, const double* U, long ldU, double* X, long ldX,
             double* tbuf, cudaStream_t st) {
  return q2_apply_range(forward, n, ncols, U, ldU, X, ldX, tbuf, 0, n, -1, st);
}

}  // namespace evd

extern "C" long evd_bc_back_work_size(long n) { return evd::q2_tbuf_doubles(n < 0 ? 0 : n); }

extern "C" int evd_bc_back(double* Q, long ldQ, const double* U, long ldU, long n, int b,
                           cudaStream_t stream) {
  if (b != 32) return EVD_ERR_INVALID_ARG;
  return evd::q2_apply(true, n, n, U, ldU, Q, ldQ, nullptr, stream);
}

extern "C" int evd_bc_back_apply(long n, long ncols, const double* U, long ldU, double* X,
                                 long ldX, int b, double* work, long lwork, cudaStream_t stream) {
  if (b != 32) return EVD_ERR_INVALID_ARG;
  if (work && lwork < evd::q2_tbuf_doubles(n)) return EVD_ERR_WORKSPACE;
  return evd::q2_apply(false, n, ncols, U, ldU, X, ldX, work, stream);
}
