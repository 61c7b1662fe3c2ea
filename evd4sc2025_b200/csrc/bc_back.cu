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
// Ordering.  Rows are cut into 256-row strips R = 0, 256, ...  In strip R
// sweep h touches exactly rows [R+h+1, R+h+257) (8 reflectors, k = R/32 ..
// R/32+7).  Overlapping reflectors of sweeps s < s' must be applied s first
// (forward) or s' first (reverse); processing strips bottom-up with sweeps
// ascending (forward), or top-down with sweeps descending (reverse), respects
// that: the overlap of strip R's sweep h with strip R+-256 occurs only for
// sweeps on the correct side.  (The reference uses the forward order.)
//
// B200 layout (not the reference's): a warp owns 8 columns of X and holds the
// 256-row window in registers, lane l holding rows 8l..8l+7 of each column,
// so a 32-row reflector is 4 lanes (2 shuffle steps per dot product, eight
// independent dot products per sweep) and each reflector value read from
// shared memory feeds 8 columns.  The window slides one row per sweep through
// a ring of 8 registers (the phase is a compile-time constant inside an
// 8-sweep block): one rotation shuffle per column, no register moves, no
// divergent branches; the row leaving the window is written back and the row
// entering is prefetched one block ahead.  Reflector chunks (16 sweeps x 256
// rows) are double-buffered in shared memory with cp.async, in a rotated
// layout that is bank-conflict free for both the copy and the reads; 4-warp
// CTAs so that two or more fit per SM.  Exactly 2 n^2 ncols flops, FP64 FMA; rows >= n are never read or
// written (the reference needs 346 zero rows of padding).
#include "common.cuh"

namespace evd {

namespace {

constexpr int kWin = 256;   // window rows (8 reflectors of 32)
constexpr int kCols = 8;    // columns per warp
constexpr int kWarps = 4;   // warps per CTA
constexpr int kChunk = 16;  // sweeps per staged reflector chunk
constexpr int kThreadsBC = kWarps * 32;

__device__ __forceinline__ void cp_async8_zfill(double* smem, const double* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
               "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Shared-memory slot of window row i = 8l + j of one staged sweep: lane l reads
// its 8 values at j*32 + rot(l, j); the rotation by 4j keeps both the staging
// writes (consecutive rows) and the per-sweep reads (consecutive lanes) free
// of bank conflicts.
__device__ __forceinline__ int uslot(int l, int j) { return j * 32 + ((l + 4 * j) & 31); }

// Stage reflectors of sweeps [h0, h0+kChunk) for strip R (zero for h >= H or
// row >= n): buf[hc*256 + uslot(l, j)] = U(R+h+1 + 8l+j, h).
__device__ __forceinline__ void stage_chunk(double* buf, const double* U, long ldU, int n, long R,
                                            int H, int h0) {
  for (int e = threadIdx.x; e < kChunk * kWin; e += kThreadsBC) {
    int hc = e >> 8, i = e & 255;
    int h = h0 + hc;
    long row = R + h + 1 + i;
    bool valid = (h < H) && (row < n);
    const double* src = valid ? (U + row + (long)h * ldU) : U;
    cp_async8_zfill(buf + hc * kWin + uslot(i >> 3, i & 7), src, valid);
  }
}

template <bool FWD>
__global__ void __launch_bounds__(kThreadsBC, 2)
    q2_apply_kernel(int n, int ncols, const double* __restrict__ U, long ldU,
                    double* __restrict__ X, long ldX) {
  extern __shared__ double smem[];
  double* Ubuf = smem;                                   // 2 x kChunk x kWin
  double* iobase = smem + 2 * kChunk * kWin;             // per warp: in[2][8][C], out[8][C]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* inbuf = iobase + warp * (3 * 8 * kCols);
  double* outbuf = inbuf + 2 * 8 * kCols;
  const int col0 = blockIdx.x * (kWarps * kCols) + warp * kCols;

  // block transfers of 8 rows x 8 columns: lane -> (row r = lane/4, columns c0, c0+4)
  const int io_r = lane >> 2, io_c = lane & 3;
  const int io_colA = col0 + io_c, io_colB = col0 + io_c + 4;
  const bool okA = io_colA < ncols, okB = io_colB < ncols;
  double* colA = X + (long)(okA ? io_colA : 0) * ldX;
  double* colB = X + (long)(okB ? io_colB : 0) * ldX;

  const int nstrips = (n - 2 + kWin - 1) / kWin;
  for (int si = 0; si < nstrips; ++si) {
    const int sidx = FWD ? (nstrips - 1 - si) : si;
    const long R = (long)sidx * kWin;
    const int H = n - 2 - (int)R;            // sweeps with reflectors in this strip
    if (H <= 0) continue;
    const int nchunks = (H + kChunk - 1) / kChunk;
    const int Hp = nchunks * kChunk;

    // ---- load the initial window ----
    // FWD: window of sweep 0 starts at row R+1.  REV: of sweep Hp-1 at R+Hp.
    const long ws0 = FWD ? (R + 1) : (R + Hp);
    double x[kCols][8];
#pragma unroll
    for (int c = 0; c < kCols; ++c) {
      const int col = col0 + c;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        long row = ws0 + 8 * lane + j;
        x[c][j] = (col < ncols && row < n) ? X[row + (long)col * ldX] : 0.0;
      }
    }
    __syncthreads();
    stage_chunk(Ubuf, U, ldU, n, R, H, FWD ? 0 : (nchunks - 1) * kChunk);
    cp_commit();
    // incoming rows for block 0: FWD rows R+257+r; REV rows R+Hp-1-r
    {
      long row = FWD ? (R + 257 + io_r) : (R + Hp - 1 - io_r);
      const bool rok = row < n && row >= 0;
      inbuf[io_r * kCols + io_c] = (okA && rok) ? colA[row] : 0.0;
      inbuf[io_r * kCols + io_c + 4] = (okB && rok) ? colB[row] : 0.0;
    }

    for (int ck = 0; ck < nchunks; ++ck) {
      const int chunk = FWD ? ck : (nchunks - 1 - ck);
      const double* cur = Ubuf + (ck & 1) * (kChunk * kWin);
      cp_wait_all();
      __syncthreads();
      if (ck + 1 < nchunks)
        stage_chunk(Ubuf + ((ck + 1) & 1) * (kChunk * kWin), U, ldU, n, R, H,
                    (FWD ? (chunk + 1) : (chunk - 1)) * kChunk);
      cp_commit();

#pragma unroll 1
      for (int blk = 0; blk < kChunk / 8; ++blk) {
        const int hb = FWD ? (chunk * kChunk + blk * 8) : (chunk * kChunk + kChunk - 1 - blk * 8);
        const int gblk = ck * (kChunk / 8) + blk;
        const double* in_cur = inbuf + (gblk & 1) * (8 * kCols);
        double* in_nxt = inbuf + ((gblk + 1) & 1) * (8 * kCols);
        // prefetch the next block's incoming rows
        double preA, preB;
        {
          long row = FWD ? (R + hb + 8 + 257 + io_r) : (R + hb - 8 - io_r);
          const bool rok = row < n && row >= 0;
          preA = (okA && rok) ? colA[row] : 0.0;
          preB = (okB && rok) ? colB[row] : 0.0;
        }
#pragma unroll
        for (int P = 0; P < 8; ++P) {
          const int h = FWD ? (hb + P) : (hb - P);
          const double* us = cur + (h - chunk * kChunk) * kWin;
          double u[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) u[j] = us[uslot(lane, j)];
          double d[kCols];
#pragma unroll
          for (int c = 0; c < kCols; ++c) {
            double d0 = 0.0, d1 = 0.0;
#pragma unroll
            for (int j = 0; j < 8; j += 2) {
              d0 = fma(u[j], x[c][FWD ? ((j + P) & 7) : ((j - P) & 7)], d0);
              d1 = fma(u[j + 1], x[c][FWD ? ((j + 1 + P) & 7) : ((j + 1 - P) & 7)], d1);
            }
            d[c] = d0 + d1;
          }
#pragma unroll
          for (int c = 0; c < kCols; ++c) d[c] += __shfl_xor_sync(0xffffffffu, d[c], 1);
#pragma unroll
          for (int c = 0; c < kCols; ++c) d[c] += __shfl_xor_sync(0xffffffffu, d[c], 2);
#pragma unroll
          for (int c = 0; c < kCols; ++c)
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int pj = FWD ? ((j + P) & 7) : ((j - P) & 7);
              x[c][pj] = fma(-d[c], u[j], x[c][pj]);
            }
          // slide the window by one row (register ring, phase P is a constant):
          // FWD: logical row 0 (physical P) leaves through lane 0 and every lane
          //      takes lane l+1's; REV: logical row 7 (physical (7-P)&7) leaves
          //      through lane 31 and every lane takes lane l-1's.  The rotation
          //      hands the leaving value to the lane that receives the new row.
          const int pp = FWD ? (P & 7) : ((7 - P) & 7);
          const int src = FWD ? ((lane + 1) & 31) : ((lane + 31) & 31);
          const bool edge = FWD ? (lane == 31) : (lane == 0);
#pragma unroll
          for (int c = 0; c < kCols; ++c) {
            const double t = __shfl_sync(0xffffffffu, x[c][pp], src);
            const double inv = in_cur[P * kCols + c];
            if (edge) outbuf[P * kCols + c] = t;
            x[c][pp] = edge ? inv : t;
          }
        }
        __syncwarp();
        // write back the 8 rows that left the window, stage the next incoming rows
        {
          long row = FWD ? (R + hb + 1 + io_r) : (R + hb + 256 - io_r);
          if (row < n) {
            if (okA) colA[row] = outbuf[io_r * kCols + io_c];
            if (okB) colB[row] = outbuf[io_r * kCols + io_c + 4];
          }
          in_nxt[io_r * kCols + io_c] = preA;
          in_nxt[io_r * kCols + io_c + 4] = preB;
        }
        __syncwarp();
      }
    }
    // Every sweep is followed by a one-row slide and Hp % 8 == 0 (phase back
    // to 0): FWD ends with the window at R+Hp+1, REV at R (one above sweep 0's).
    const long wsf = FWD ? (R + Hp + 1) : R;
#pragma unroll
    for (int c = 0; c < kCols; ++c) {
      const int col = col0 + c;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        long row = wsf + 8 * lane + j;
        if (col < ncols && row < n) X[row + (long)col * ldX] = x[c][j];
      }
    }
    __syncthreads();
  }
}

constexpr size_t kBCSmem =
    (2 * kChunk * kWin + kWarps * 3 * 8 * kCols) * sizeof(double);

template <bool FWD>
int launch_q2(long n, long ncols, const double* U, long ldU, double* X, long ldX,
              cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    EVD_CUDA_TRY(cudaFuncSetAttribute(q2_apply_kernel<FWD>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBCSmem));
    attr = true;
  }
  int grid = ceil_div_i(ncols, kWarps * kCols);
  q2_apply_kernel<FWD><<<grid, kThreadsBC, kBCSmem, st>>>((int)n, (int)ncols, U, ldU, X, ldX);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

}  // namespace

int q2_apply(bool forward, long n, long ncols, const double* U, long ldU, double* X, long ldX,
             cudaStream_t st) {
  if (n < 0 || ncols < 0 || ldU < n || ldX < n) return EVD_ERR_INVALID_ARG;
  if (n > (1L << 30) || ncols > (1L << 30)) return EVD_ERR_INVALID_ARG;
  if (n < 3 || ncols == 0) return EVD_SUCCESS;
  if (!U || !X) return EVD_ERR_INVALID_ARG;
  return forward ? launch_q2<true>(n, ncols, U, ldU, X, ldX, st)
                 : launch_q2<false>(n, ncols, U, ldU, X, ldX, st);
}

}  // namespace evd

extern "C" int evd_bc_back(double* Q, long ldQ, const double* U, long ldU, long n, int b,
                           cudaStream_t stream) {
  if (b != 32) return EVD_ERR_INVALID_ARG;
  return evd::q2_apply(true, n, n, U, ldU, Q, ldQ, stream);
}

extern "C" int evd_bc_back_apply(long n, long ncols, const double* U, long ldU, double* X,
                                 long ldX, int b, cudaStream_t stream) {
  if (b != 32) return EVD_ERR_INVALID_ARG;
  return evd::q2_apply(false, n, ncols, U, ldU, X, ldX, stream);
}
