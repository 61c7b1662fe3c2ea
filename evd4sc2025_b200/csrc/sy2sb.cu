// Stage 1: full -> band reduction with the two-sided ZY update.
//
// Same algorithm as my_ZY_ZY_SBR_Vector<double> (api/zy_zy_sy2sb.cu:24-486):
// nb-wide frames; inside a frame, b-wide panels i = b, 2b, ..., nb:
//   (Y, W, R) = panelQR(A[i:, i-b:i])                              (:100-125)
//   Z  = OA[i:, i:] W - Y_prev (Z_prev^T W) - Z_prev (Y_prev^T W)  (:134-304)
//   Z -= 1/2 Y (W^T Z)                                              (:307-347)
//   A[i:, i:i+b] -= Y Z[i:i+b]^T + Z Y[i:i+b]^T   (lazy next panel, :351-395)
// then OA_trail -= Y Z^T + Z Y^T (lower, :422-433) and recursion on the
// trailing frame (:466-485).
//
// B200 differences (same arithmetic, fewer passes):
//  * the panel kernel writes Y -> dY, W -> dW and the band panel (R over
//    zeros) -> dA directly (no copyMatrix / getU kernels);
//  * the lazy update is ONE two-operand-pair GEMM (K = 2i) instead of two, and
//    likewise Z_prev^T W / Y_prev^T W (one GEMM stacked along M) and the two
//    corrections of Z (one GEMM with K = 2(i-b));
//  * the trailing SYR2K computes lower tiles only and its epilogue mirrors them
//    (no separate copyMatrixL2U pass);
//  * instead of copying the whole trailing matrix OA -> dA after each frame
//    (:443-450), only the next frame's nb-wide column block is copied: every
//    other element of dA is rewritten by a later panel epilogue;
//  * skinny products (n = 32) use split-K with a deterministic reduction.
#include "common.cuh"
#include "gemm_f64.cuh"
#include "ozaki.cuh"
#include "panel_qr.cuh"

namespace evd {

namespace {

__global__ void copy_block_kernel(long m, long n, const double* __restrict__ src, long lds,
                                  double* __restrict__ dst, long ldd) {
  for (long j = blockIdx.y; j < n; j += gridDim.y)
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m;
         i += (long)gridDim.x * blockDim.x)
      dst[i + j * ldd] = src[i + j * lds];
}

// upper triangle <- lower triangle (copyMatrixL2U, util/kernelOther/kernelOther.cu:73-90),
// tiled through shared memory so both sides are coalesced.
__global__ void mirror_l2u_kernel(long n, double* A, long lda) {
  __shared__ double t[32][33];
  long bi = blockIdx.x, bj = blockIdx.y;  // tile row / col
  if (bj > bi) return;                    // only lower tiles are sources
  long r0 = bi * 32, c0 = bj * 32;
  int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int k = ty; k < 32; k += 8) {
    long r = r0 + tx, c = c0 + k;
    t[k][tx] = (r < n && c < n) ? A[r + c * lda] : 0.0;
  }
  __syncthreads();
  // write A[c, r] = A[r, c] for r > c
  for (int k = ty; k < 32; k += 8) {
    long c = c0 + tx, r = r0 + k;  // destination row c, column r
    if (r < n && c < n && r > c) A[c + r * lda] = t[tx][k];
  }
}

}  // namespace

struct Sy2sbLayout {
  long panel_off, panel_n;
  long s1_off, s2_off, s3_off, small_n;
  long sk_off, sk_n;
  long total;
};

static Sy2sbLayout sy2sb_layout(long M, long b, long nb) {
  Sy2sbLayout L{};
  L.panel_off = 0;
  L.panel_n = panel_qr_ws_doubles(M);
  L.small_n = 2 * nb * b;  // [S1; S2] is 2kp x b
  L.s1_off = L.panel_off + L.panel_n;
  L.s2_off = L.s1_off + L.small_n;
  L.s3_off = L.s2_off + L.small_n;
  L.sk_off = L.s3_off + L.small_n;
  L.sk_n = std::max(8 * M * b, 32 * nb * b);
  L.total = L.sk_off + L.sk_n;
  return L;
}

long sy2sb_ws_doubles(long M, long b, long nb) { return sy2sb_layout(M, b, nb).total; }

// oz != nullptr: the trailing SYR2K is an emulated FP64 product on the
// integer tensor cores (oz->nmod moduli) instead of the DMMA GEMM.
int sy2sb(long M, long N, long b, long nb, double* OA, long ldOA, double* dA, long ldA,
          double* dW, long ldW, double* dY, long ldY, double* dZ, long ldZ, double* dR, long ldR,
          double* work, long lwork, cudaStream_t st, const OzWork* oz) {
  if (M <= 0) return EVD_SUCCESS;
  if (M != N || b != 32 || nb <= 0 || nb % b != 0 || M % nb != 0) return EVD_ERR_INVALID_ARG;
  if (ldOA < M || ldA < M || ldW < M || ldY < M || ldZ < M || ldR < M) return EVD_ERR_INVALID_ARG;
  if (!OA || !dA || !dW || !dY || !dZ || !dR || !work) return EVD_ERR_INVALID_ARG;
  Sy2sbLayout L = sy2sb_layout(M, b, nb);
  if (lwork < L.total) return EVD_ERR_WORKSPACE;
  double* pws = work + L.panel_off;
  double* S1 = work + L.s1_off;
  double* S2 = work + L.s2_off;
  double* S3 = work + L.s3_off;
  double* SK = work + L.sk_off;
  const size_t skn = (size_t)L.sk_n;
  EVD_TRY(panel_counters_reset(M, pws, st));

  for (long off = 0;; off += nb) {
    const long Nf = M - off;
    if (off > 0) {
      // this frame's first nb columns of the updated trailing matrix -> dA
      dim3 grid(ceil_div_i(Nf, 256), (unsigned)std::min<long>(nb, 65535));
      copy_block_kernel<<<grid, 256, 0, st>>>(Nf, nb, OA + off + off * ldOA, ldOA,
                                              dA + off + off * ldA, ldA);
      EVD_LAUNCHED();
    }
    for (long i = b; i <= nb && i < Nf; i += b) {
      const long m = Nf - i;
      const long g0 = off + i;
      double* panel = dA + g0 + (g0 - b) * ldA;
      double* Yp = dY + g0 + (g0 - b) * ldY;
      double* Wp = dW + g0 + (g0 - b) * ldW;
      double* Rp = dR + g0 + (i - b) * ldR;
      double* Zp = dZ + i + (i - b) * ldZ;
      EVD_TRY(panel_qr_launch(m, panel, ldA, pws, 1, Yp, ldY, Wp, ldW, Rp, ldR, panel, ldA, st));

      // Z = OA[g0:, g0:] W
      EVD_TRY(dgemm('n', 'n', m, b, m, 1.0, OA + g0 + g0 * ldOA, ldOA, Wp, ldW, 0.0, Zp, ldZ,
                    st, 0, SK, skn));
      if (i > b) {
        const long kp = i - b;
        const double* Zprev = dZ + i;             // rows i.., cols 0..kp-1
        const double* Yprev = dY + g0 + off * ldY;
        // [S1; S2] = [Zprev | Yprev]^T W  (2kp x b, one GEMM stacked along M)
        GemmPair g1{'t', 'n', 2 * kp, b, m, 1.0, 0.0, Zprev, ldZ, Wp, ldW, S1, 2 * kp};
        g1.Am2 = Yprev;
        g1.ldam2 = ldY;
        g1.m1 = kp;
        EVD_TRY(dgemm_pair(g1, st, 0, SK, skn));
        // Z -= [Yprev, Zprev] [S1; S2]  (one GEMM, operands switched at K = kp)
        GemmPair g2{'n', 'n', m, b, 2 * kp, -1.0, 1.0, Yprev, ldY, S1, 2 * kp, Zp, ldZ};
        g2.A2 = Zprev;
        g2.lda2 = ldZ;
        g2.k1 = kp;
        EVD_TRY(dgemm_pair(g2, st, 0, SK, skn));
      }
      // Z -= 1/2 Y (W^T Z)
      EVD_TRY(dgemm('t', 'n', b, b, m, 1.0, Wp, ldW, Zp, ldZ, 0.0, S3, b, st, 0, SK, skn));
      EVD_TRY(dgemm('n', 'n', m, b, b, -0.5, Yp, ldY, S3, b, 1.0, Zp, ldZ, st, 0, SK, skn));
      if (i < nb) {
        // A[g0:, g0:g0+b] -= Y[g0:, off:off+i] Z[i:i+b, 0:i]^T + Z[i:, 0:i] Y[g0:g0+b, off:off+i]^T
        const double* Yi = dY + g0 + off * ldY;
        const double* Zi = dZ + i;
        EVD_TRY(dgemm_nt_pair(m, b, i, i, -1.0, Yi, ldY, Zi, ldZ, Zi, ldZ, Yi, ldY, 1.0,
                              dA + g0 + g0 * ldA, ldA, st, 0, SK, skn));
      }
    }
    if (Nf - nb <= 0) break;
    // trailing update of the working copy (lower tiles, mirrored)
    const long t0 = off + nb;
    if (oz) {
      EVD_TRY(oz_syr2k_lower(Nf - nb, nb, -1.0, dY + t0 + off * ldY, ldY, dZ + nb, ldZ, 1.0,
                             OA + t0 + t0 * ldOA, ldOA, oz->nmod, oz->ws, oz->bytes, st));
    } else {
      EVD_TRY(syr2k_lower_mirror(Nf - nb, nb, -1.0, dY + t0 + off * ldY, ldY, dZ + nb, ldZ, 1.0,
                                 OA + t0 + t0 * ldOA, ldOA, st));
    }
  }
  // dA <- symmetric band (copyMatrixL2U, src/EVD/myEVD.cu:346)
  dim3 g2(ceil_div_i(M, 32), ceil_div_i(M, 32));
  mirror_l2u_kernel<<<g2, dim3(32, 8), 0, st>>>(M, dA, ldA);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

int mirror_l2u(long n, double* A, long lda, cudaStream_t st) {
  if (n <= 0) return EVD_SUCCESS;
  dim3 g2(ceil_div_i(n, 32), ceil_div_i(n, 32));
  mirror_l2u_kernel<<<g2, dim3(32, 8), 0, st>>>(n, A, lda);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

int copy_matrix(long m, long n, const double* src, long lds, double* dst, long ldd,
                cudaStream_t st) {
  if (m <= 0 || n <= 0) return EVD_SUCCESS;
  dim3 grid(ceil_div_i(m, 256), (unsigned)std::min<long>(n, 65535));
  copy_block_kernel<<<grid, 256, 0, st>>>(m, n, src, lds, dst, ldd);
  EVD_LAUNCHED();
  return EVD_SUCCESS;
}

}  // namespace evd

extern "C" long evd_sy2sb_work_size(long M, long b, long nb) {
  if (M <= 0 || b != 32 || nb <= 0) return 0;
  return evd::sy2sb_ws_doubles(M, b, nb);
}

extern "C" int evd_sy2sb(long M, long N, long b, long nb, double* dOriA, long ldOriA, double* dA,
                         long ldA, double* dW, long ldW, double* dY, long ldY, double* dZ,
                         long ldZ, double* dR, long ldR, double* work, long lwork,
                         cudaStream_t stream) {
  return evd::sy2sb(M, N, b, nb, dOriA, ldOriA, dA, ldA, dW, ldW, dY, ldY, dZ, ldZ, dR, ldR,
                    work, lwork, stream, nullptr);
}
