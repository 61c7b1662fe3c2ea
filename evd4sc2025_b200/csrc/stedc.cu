// Symmetric tridiagonal eigensolver: divide and conquer on the device.
//
// Replaces the reference's host call LAPACKE_dstedc('I', ...) (MKL,
// src/EVD/myEVD.cu:529), which the reference overlaps with its GPU back
// transformation on a second host thread.  Same mathematics as LAPACK's
// divide and conquer (Cuppen's tear, deflation, secular equation, Gu-Eisenstat
// recomputation of z), written for the GPU:
//
//  * n is padded to n' = s * 2^L (leaf size s <= 32) with decoupled diagonal
//    entries larger than every eigenvalue; they deflate at every merge, sort to
//    the end and are dropped.  All merges of a level then have equal sizes and
//    the merge GEMMs run as uniform batched DMMA GEMMs.
//  * leaves: one warp per leaf, implicit QL with Wilkinson shift (the
//    classical tql2 iteration); every lane runs the scalar recurrence on its
//    own copy and applies the rotations to its own row of the leaf's
//    eigenvector matrix, so no lane ever waits on another.
//  * merge of [lo, mid) and [mid, hi) with coupling beta = e[mid-1]:
//      z = (last row of Q1, sign(beta) * first row of Q2) / sqrt(2),
//      rho = 2|beta|; merge-sort of the two eigenvalue lists (ranks by binary
//      search); sequential deflation per merge (small rho*|z_i| or Givens
//      rotation of close pairs, tol = 8 eps max(|d|,|z|)); secular roots with
//      the origin at the nearer pole and a two-pole rational model per
//      iteration, bracketed by bisection; z_hat_i from the Loewner formula
//      (products of (d_i - lambda_j)/(d_i - d_j)); U(:,j) = z_hat ./ (d - lambda_j)
//      normalised; Z_new = [Q1 0; 0 Q2] P U as two GEMMs that skip the zero
//      blocks (columns from Q1 only / mixed / Q2 only).
//  * every level is a fixed sequence of launches batched over its merges;
//    the host reads the per-merge sizes once per level to size the GEMMs.
#include <math.h>

#include <vector>

#include "common.cuh"
#include "gemm_f64.cuh"
#include "ozaki.cuh"

namespace evd {

namespace {

constexpr int kLeafMax = 32;
constexpr double kEps = 1.1102230246251565e-16;  // 2^-53

struct StedcPlan {
  long n, np;   // original and padded size
  int s, L;     // leaf size, levels
  // double offsets
  long o_d, o_e, o_Z, o_zv, o_ds, o_zs, o_dK, o_zK, o_tau, o_zh, o_dD, o_rc, o_rs, o_rho,
      o_scal, o_Qt, o_Qb, o_Ut, o_Ub, o_Zn, total_d;
  // int offsets
  long i_perm, i_colK, i_typK, i_pT, i_pB, i_colD, i_rA, i_rB, i_org, i_desc, total_i;
};

StedcPlan make_plan(long n) {
  StedcPlan p{};
  p.n = n;
  int L = 0;
  while ((n + (1L << L) - 1) / (1L << L) > kLeafMax) ++L;
  p.L = L;
  p.s = (int)((n + (1L << L) - 1) / (1L << L));
  p.np = (long)p.s << L;
  const long np = p.np;
  long o = 0;
  auto take = [&](long k) { long r = o; o += (k + 7) / 8 * 8; return r; };
  p.o_d = take(np);
  p.o_e = take(np);
  p.o_Z = take(np * np);
  p.o_zv = take(np);
  p.o_ds = take(np);
  p.o_zs = take(np);
  p.o_dK = take(np);
  p.o_zK = take(np);
  p.o_tau = take(np);
  p.o_zh = take(np);
  p.o_dD = take(np);
  p.o_rc = take(np);
  p.o_rs = take(np);
  p.o_rho = take(np);
  p.o_scal = take(1024);
  p.o_Qt = take(np * np / 2 + np);
  p.o_Qb = take(np * np / 2 + np);
  p.o_Ut = take(np * np);
  p.o_Ub = take(np * np);
  p.o_Zn = take(np * np);
  p.total_d = o;
  long q = 0;
  auto takei = [&](long k) { long r = q; q += (k + 3) / 4 * 4; return r; };
  p.i_perm = takei(np);
  p.i_colK = takei(np);
  p.i_typK = takei(np);
  p.i_pT = takei(np);
  p.i_pB = takei(np);
  p.i_colD = takei(np);
  p.i_rA = takei(np);
  p.i_rB = takei(np);
  p.i_org = takei(np);
  p.i_desc = takei(8 * (np / 2 + 1) + 64);
  p.total_i = q;
  return p;
}

// per-merge descriptor (ints)
enum { D_K = 0, D_K1, D_K2, D_K3, D_NDEF, D_NROT, D_ERR, D_PAD };

// ----------------------------------------------------------------- setup

__global__ void absmax_kernel(long n, const double* d, const double* e, double* out) {
  __shared__ double red[32];
  double m = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double a = fabs(d[i]), b = (i < n - 1) ? fabs(e[i]) : 0.0;
    // fmax drops NaN; keep it visible so the host can reject the input
    m = (isnan(a) || isnan(b)) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(m, fmax(a, b));
    if (isnan(m)) break;
  }
  // NaN-propagating max over the block
#pragma unroll
  for (int k = 16; k > 0; k >>= 1) {
    double o = __shfl_xor_sync(0xffffffffu, m, k);
    m = (isnan(o) || isnan(m)) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(m, o);
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) {
      double o = __shfl_xor_sync(0xffffffffu, t, k);
      t = (isnan(o) || isnan(t)) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(t, o);
    }
    if (threadIdx.x == 0) out[0] = t;
  }
}

// scaled copy + padding + tears at every leaf boundary
__global__ void init_kernel(long n, long np, int s, const double* d, const double* e,
                            const double* scal, double* dw, double* ew) {
  const double nrm = scal[0];
  const double inv = (nrm > 0.0) ? 1.0 / nrm : 1.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < np; i += (long)gridDim.x * blockDim.x) {
    double di = (i < n) ? d[i] * inv : 10.0 + (double)(i - n) * (1.0 / (double)np);
    double ei = (i < n - 1) ? e[i] * inv : 0.0;
    // tear at leaf boundaries: between rows k*s-1 and k*s subtract |e(k*s-1)|
    if (i < np - 1 && ((i + 1) % s) == 0) {
      // i is the last row of a leaf: di -= |e_i|
      di -= fabs(ei);
    }
    if (i > 0 && (i % s) == 0) {
      double ep = (i - 1 < n - 1) ? e[i - 1] * inv : 0.0;
      di -= fabs(ep);
    }
    dw[i] = di;
    ew[i] = ei;
  }
}

// ----------------------------------------------------------------- leaves

__device__ __forceinline__ double sign_of(double a, double b) { return (b >= 0.0) ? fabs(a) : -fabs(a); }

// One warp per leaf; lane r owns row r of the leaf eigenvector matrix.
__global__ void leaf_ql_kernel(int s, int nleaves, double* dw, const double* ew, double* Zw,
                               long ldz, int* err) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nleaves) return;
  const long lo = (long)warp * s;
  double d[kLeafMax], e[kLeafMax], z[kLeafMax];
  for (int i = 0; i < s; ++i) {
    d[i] = dw[lo + i];
    e[i] = (i < s - 1) ? ew[lo + i] : 0.0;
    z[i] = (i == lane) ? 1.0 : 0.0;
  }
  bool fail = false;
  for (int l = 0; l < s && !fail; ++l) {
    int iter = 0;
    for (;;) {
      int m = l;
      while (m < s - 1) {
        double dd = fabs(d[m]) + fabs(d[m + 1]);
        if (fabs(e[m]) <= kEps * dd) break;
        ++m;
      }
      if (m == l) break;
      if (++iter > 60) {
        fail = true;
        break;
      }
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + sign_of(r, g));
      double sn = 1.0, cs = 1.0, p = 0.0;
      bool underflow = false;
      for (int i = m - 1; i >= l; --i) {
        double f = sn * e[i];
        double bb = cs * e[i];
        r = hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          underflow = true;
          break;
        }
        sn = f / r;
        cs = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * sn + 2.0 * cs * bb;
        p = sn * r;
        d[i + 1] = g + p;
        g = cs * r - bb;
        double t = z[i + 1];
        z[i + 1] = sn * z[i] + cs * t;
        z[i] = cs * z[i] - sn * t;
      }
      if (underflow) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  if (fail && lane == 0) atomicCAS(err, 0, kDevNoConvergence);
  // selection sort ascending (identical in every lane), permuting z
  for (int i = 0; i < s - 1; ++i) {
    int k = i;
    double v = d[i];
    for (int j = i + 1; j < s; ++j)
      if (d[j] < v) {
        k = j;
        v = d[j];
      }
    if (k != i) {
      d[k] = d[i];
      d[i] = v;
      double t = z[i];
      z[i] = z[k];
      z[k] = t;
    }
  }
  if (lane < s) {
    for (int c = 0; c < s; ++c) Zw[(lo + lane) + (lo + c) * ldz] = z[c];
  }
  if (lane == 0)
    for (int i = 0; i < s; ++i) dw[lo + i] = d[i];
}

// ----------------------------------------------------------------- merges

struct LevelArgs {
  long np, ldz;
  int N, n1, n2, nm;
  double* dw;
  const double* ew;
  double* Zw;
  double *zv, *ds, *zs, *dK, *zK, *tau, *zh, *dD, *rc, *rs, *rho;
  int *perm, *colK, *typK, *pT, *pB, *colD, *rA, *rB, *org, *desc;
  int* err;
  double *Qt, *Qb, *Ut, *Ub, *Zn;
  int K12max, K23max, Kmax;
};

// z vector, rho and the merged sort order.  grid (ceil(N/256), nm)
__global__ void merge_setup_kernel(LevelArgs a) {
  const int m = blockIdx.y;
  const long lo = (long)m * a.N, mid = lo + a.n1;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.N) return;
  const double beta = a.ew[mid - 1];
  const double sgn = (beta < 0.0) ? -1.0 : 1.0;
  const double inv_sqrt2 = 0.70710678118654752440;
  double zc, dc = a.dw[lo + c];
  if (c < a.n1) zc = a.Zw[(mid - 1) + (lo + c) * a.ldz];
  else zc = sgn * a.Zw[mid + (lo + c) * a.ldz];
  zc *= inv_sqrt2;
  a.zv[lo + c] = zc;
  if (c == 0) a.rho[m] = 2.0 * fabs(beta);
  // rank in the merged ascending order (ties: first half first)
  int rank;
  if (c < a.n1) {
    const double* d2 = a.dw + mid;
    int l = 0, h = a.n2;  // count d2 < dc
    while (l < h) {
      int md = (l + h) >> 1;
      if (d2[md] < dc) l = md + 1; else h = md;
    }
    rank = c + l;
  } else {
    const double* d1 = a.dw + lo;
    int l = 0, h = a.n1;  // count d1 <= dc
    while (l < h) {
      int md = (l + h) >> 1;
      if (d1[md] <= dc) l = md + 1; else h = md;
    }
    rank = (c - a.n1) + l;
  }
  a.perm[lo + rank] = c;
  a.ds[lo + rank] = dc;
  a.zs[lo + rank] = zc;
}

// Deflation of one merge (LAPACK dlaed2's tests, the reference's host dstedc):
// small components of z, then Givens pair deflation of neighbours in the merged
// order.  The pair test chains through the previous undeflated entry, so one
// thread scans; the block stages the inputs in shared memory chunk by chunk
// (the scan never waits on global loads), reduces the tolerance in parallel and
// finishes the type-ordered GEMM positions in parallel.  grid nm, block
// kDefThreads.
constexpr int kDefThreads = 256;
constexpr int kDefChunk = 2048;

__global__ void __launch_bounds__(kDefThreads) merge_deflate_kernel(LevelArgs a) {
  __shared__ double s_d[kDefChunk], s_z[kDefChunk];
  __shared__ int s_c[kDefChunk];
  __shared__ double s_red[2][kDefThreads / 32];
  __shared__ int s_bad, s_K, s_K1, s_K2;
  const int m = blockIdx.x;
  const long lo = (long)m * a.N;
  const int N = a.N, n1 = a.n1;
  const double rho = a.rho[m];
  const double* ds = a.ds + lo;
  const double* zs = a.zs + lo;
  const int* perm = a.perm + lo;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double dmax = 0.0, zmax = 0.0;
  for (int k = tid; k < N; k += kDefThreads) {
    dmax = fmax(dmax, fabs(ds[k]));
    zmax = fmax(zmax, fabs(zs[k]));
  }
  dmax = warp_max(dmax);
  zmax = warp_max(zmax);
  if (lane == 0) {
    s_red[0][wid] = dmax;
    s_red[1][wid] = zmax;
  }
  if (tid == 0) s_bad = 0;
  __syncthreads();
  dmax = 0.0;
  zmax = 0.0;
  for (int w = 0; w < kDefThreads / 32; ++w) {
    dmax = fmax(dmax, s_red[0][w]);
    zmax = fmax(zmax, s_red[1][w]);
  }
  const double tol = 8.0 * kEps * fmax(dmax, zmax);
  int* d_ = a.desc + 8 * m;
  if (rho * zmax <= tol) {
    // everything deflates: the merged order is the result
    for (int k = tid; k < N; k += kDefThreads) {
      a.dD[lo + k] = ds[k];
      a.colD[lo + k] = perm[k];
    }
    if (tid == 0) {
      d_[D_K] = 0;
      d_[D_K1] = 0;
      d_[D_K2] = 0;
      d_[D_K3] = 0;
      d_[D_NDEF] = N;
      d_[D_NROT] = 0;
    }
    return;
  }
  // scan state (thread 0 only)
  int K = 0, nd = 0, nr = 0, c1 = 0, c2 = 0, c3 = 0;
  bool have = false;
  double pd = 0.0, pz = 0.0;
  int pc = 0, pt = 0;
  auto emit_root = [&](double dv, double zv, int cv, int tv) {
    a.dK[lo + K] = dv;
    a.zK[lo + K] = zv;
    a.colK[lo + K] = cv;
    a.typK[lo + K] = tv;
    a.pT[lo + K] = (tv == 1) ? c1++ : ((tv == 2) ? c2++ : c3++);  // index within its type
    ++K;
  };
  for (int c0 = 0; c0 < N; c0 += kDefChunk) {
    const int cn = min(kDefChunk, N - c0);
    __syncthreads();  // previous chunk consumed
    for (int k = tid; k < cn; k += kDefThreads) {
      s_d[k] = ds[c0 + k];
      s_z[k] = zs[c0 + k];
      s_c[k] = perm[c0 + k];
    }
    __syncthreads();
    if (tid == 0 && !s_bad) {
      for (int k = 0; k < cn; ++k) {
        const double dk = s_d[k], zk = s_z[k];
        const int ck = s_c[k];
        if (ck < 0 || ck >= N) {
          atomicCAS(a.err, 0, kDevBadShape);
          s_bad = 1;
          break;
        }
        const int tk = (ck < n1) ? 1 : 3;
        if (rho * fabs(zk) <= tol) {
          a.dD[lo + nd] = dk;
          a.colD[lo + nd] = ck;
          ++nd;
          continue;
        }
        if (!have) {
          have = true;
          pd = dk; pz = zk; pc = ck; pt = tk;
          continue;
        }
        double sv = pz, cv = zk;
        const double tau = hypot(cv, sv);
        const double t = dk - pd;
        cv /= tau;
        sv = -sv / tau;
        if (fabs(t * cv * sv) <= tol) {
          // rotate columns (pc, ck): x' = c x + s y, y' = c y - s x
          a.rA[lo + nr] = pc;
          a.rB[lo + nr] = ck;
          a.rc[lo + nr] = cv;
          a.rs[lo + nr] = sv;
          ++nr;
          const double cc = cv * cv, ss = sv * sv;
          const double dnew_p = pd * cc + dk * ss;
          const double dnew_k = pd * ss + dk * cc;
          const int tnew = (pt == tk) ? tk : 2;
          a.dD[lo + nd] = dnew_p;  // the previous entry deflates
          a.colD[lo + nd] = pc;
          ++nd;
          pd = dnew_k; pz = tau; pc = ck; pt = tnew;
        } else {
          emit_root(pd, pz, pc, pt);
          pd = dk; pz = zk; pc = ck; pt = tk;
        }
      }
    }
  }
  if (tid == 0) {
    if (have && !s_bad) emit_root(pd, pz, pc, pt);
    s_K = K;
    s_K1 = c1;
    s_K2 = c2;
    d_[D_K] = K;
    d_[D_K1] = c1;
    d_[D_K2] = c2;
    d_[D_K3] = c3;
    d_[D_NDEF] = nd;
    d_[D_NROT] = nr;
  }
  __syncthreads();
  if (s_bad) return;
  // type-ordered positions for the two structured GEMMs:
  // type 1 -> Qt column c1; type 2 -> Qt column K1 + c2 and Qb column c2;
  // type 3 -> Qb column K2 + c3
  const int Kf = s_K, K1f = s_K1, K2f = s_K2;
  for (int i = tid; i < Kf; i += kDefThreads) {
    const int tv = a.typK[lo + i], idx = a.pT[lo + i];
    if (tv == 1) {
      a.pB[lo + i] = -1;
    } else if (tv == 2) {
      a.pT[lo + i] = K1f + idx;
      a.pB[lo + i] = idx;
    } else {
      a.pT[lo + i] = -1;
      a.pB[lo + i] = K2f + idx;
    }
  }
}

// Apply the recorded rotations to the block's columns; thread = row.
__global__ void merge_rotate_kernel(LevelArgs a) {
  const int m = blockIdx.y;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.N) return;
  const long lo = (long)m * a.N;
  const int nr = a.desc[8 * m + D_NROT];
  double* row = a.Zw + (lo + r) + lo * a.ldz;
  for (int q = 0; q < nr; ++q) {
    long ca = a.rA[lo + q], cb = a.rB[lo + q];
    if (ca < 0 || ca >= a.N || cb < 0 || cb >= a.N) {
      atomicCAS(a.err, 0, kDevBadShape);
      return;
    }
    double c = a.rc[lo + q], s = a.rs[lo + q];
    double x = row[ca * a.ldz], y = row[cb * a.ldz];
    row[ca * a.ldz] = c * x + s * y;
    row[cb * a.ldz] = c * y - s * x;
  }
}

// Gather Q1/mixed columns (top rows) and mixed/Q2 columns (bottom rows) into
// zero-padded Qt (n1 x K12max) and Qb (n2 x K23max).  grid (ceil(N/256),
// ceil(Kcols/kColChunk), nm): thread = row, blockIdx.y = a chunk of columns.
constexpr int kColChunk = 64;

__global__ void merge_gather_kernel(LevelArgs a) {
  const int m = blockIdx.z;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.N) return;
  const int j0 = blockIdx.y * kColChunk;
  const long lo = (long)m * a.N;
  const int* d_ = a.desc + 8 * m;
  const int K = d_[D_K], K1 = d_[D_K1], K2 = d_[D_K2], K3 = d_[D_K3];
  const double* zrow = a.Zw + (lo + r) + lo * a.ldz;
  double* Qt = a.Qt + (long)m * a.n1 * a.K12max;
  double* Qb = a.Qb + (long)m * a.n2 * a.K23max;
  if (r < a.n1) {
    for (int j = max(j0, K1 + K2); j < min(a.K12max, j0 + kColChunk); ++j)
      Qt[r + (long)j * a.n1] = 0.0;
  } else {
    for (int j = max(j0, K2 + K3); j < min(a.K23max, j0 + kColChunk); ++j)
      Qb[(r - a.n1) + (long)j * a.n2] = 0.0;
  }
  const int i1 = min(K, j0 + kColChunk);
  for (int i = j0; i < i1; ++i) {
    long col = a.colK[lo + i];
    if (col < 0 || col >= a.N) {
      atomicCAS(a.err, 0, kDevBadShape);
      return;
    }
    double v = zrow[col * a.ldz];
    if (r < a.n1) {
      int p = a.pT[lo + i];
      if (p >= 0) Qt[r + (long)p * a.n1] = v;
    } else {
      int p = a.pB[lo + i];
      if (p >= 0) Qb[(r - a.n1) + (long)p * a.n2] = v;
    }
  }
}

// Deflated columns (after the rotations) -> Zn[:, K + t].  Runs after the
// merge GEMMs, which write Zn[:, 0:Kmax] for every merge of the level.
// grid (ceil(N/256), ceil(N/kColChunk), nm).
__global__ void merge_copy_deflated_kernel(LevelArgs a) {
  const int m = blockIdx.z;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.N) return;
  const int t0 = blockIdx.y * kColChunk;
  const long lo = (long)m * a.N;
  const int* d_ = a.desc + 8 * m;
  const int K = d_[D_K], nd = d_[D_NDEF];
  const double* zrow = a.Zw + (lo + r) + lo * a.ldz;
  double* Zn = a.Zn + (long)m * a.N * a.N;
  if (K + nd > a.N) {
    atomicCAS(a.err, 0, kDevBadShape);
    return;
  }
  const int t1 = min(nd, t0 + kColChunk);
  for (int t = t0; t < t1; ++t) {
    long col = a.colD[lo + t];
    if (col < 0 || col >= a.N) {
      atomicCAS(a.err, 0, kDevBadShape);
      return;
    }
    Zn[r + (long)(K + t) * a.N] = zrow[col * a.ldz];
  }
}

// f(tau) = 1/rho + sum_k z_k^2 / (Delta_k - tau), with Delta_k = d_k - d_o.
// Root j in (d_j, d_{j+1}) (or (d_{K-1}, d_{K-1} + rho z^T z) for the last).
// One warp per root: the lanes split the K terms and every sum is reduced
// across the warp, so the iteration control is uniform.
__device__ void secular_root_warp(int K, int j, const double* dK, const double* zK, double rho,
                                  double* tau_out, int* org_out) {
  const int lane = threadIdx.x & 31;
  const double dj = dK[j];
  const bool last = (j == K - 1);
  int o;
  double lo_b, hi_b, tau;
  if (!last) {
    const double gap = dK[j + 1] - dj;
    const double mid = 0.5 * gap;
    double f = 0.0;
    for (int k = lane; k < K; k += 32) f += zK[k] * zK[k] / ((dK[k] - dj) - mid);
    f = warp_sum(f) + 1.0 / rho;
    if (f >= 0.0) {  // root in (d_j, d_j + gap/2]
      o = j;
      lo_b = 0.0;
      hi_b = mid;
      tau = 0.5 * mid;
    } else {         // root in (d_j + gap/2, d_{j+1}); origin at the upper pole
      o = j + 1;
      lo_b = -mid;
      hi_b = 0.0;
      tau = -0.5 * mid;
    }
  } else {
    double zz = 0.0;
    for (int k = lane; k < K; k += 32) zz = fma(zK[k], zK[k], zz);
    zz = warp_sum(zz);
    o = j;
    lo_b = 0.0;
    hi_b = rho * zz;
    tau = 0.5 * hi_b;
  }
  const double d_o = dK[o];
  // poles adjacent to the root, relative to the origin
  const double pl = (o == j) ? 0.0 : (dj - d_o);                        // left pole (index j)
  const double pr = last ? 0.0 : ((o == j) ? (dK[j + 1] - d_o) : 0.0);  // right pole (j+1)
  for (int it = 0; it < 64; ++it) {
    double psi = 0.0, dpsi = 0.0, phi = 0.0, dphi = 0.0, erret = 0.0;
    for (int k = lane; k < K; k += 32) {
      const double del = (dK[k] - d_o) - tau;
      const double q = zK[k] / del;
      const double term = zK[k] * q;
      if (k <= j) { psi += term; dpsi = fma(q, q, dpsi); }
      else { phi += term; dphi = fma(q, q, dphi); }
      erret += fabs(term);
    }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
      psi += __shfl_xor_sync(0xffffffffu, psi, m);
      dpsi += __shfl_xor_sync(0xffffffffu, dpsi, m);
      phi += __shfl_xor_sync(0xffffffffu, phi, m);
      dphi += __shfl_xor_sync(0xffffffffu, dphi, m);
      erret += __shfl_xor_sync(0xffffffffu, erret, m);
    }
    const double f = 1.0 / rho + psi + phi;
    if (f < 0.0) lo_b = fmax(lo_b, tau); else hi_b = fmin(hi_b, tau);
    if (fabs(f) <= 8.0 * kEps * (1.0 / rho + erret)) break;
    if (hi_b - lo_b <= 4.0 * kEps * fmax(fabs(lo_b), fabs(hi_b))) break;
    // two-pole rational model through (tau, f, f')
    const double a1 = pl - tau;           // < 0
    double eta;
    if (!last) {
      const double a2 = pr - tau;         // > 0
      const double s1 = dpsi * a1 * a1;
      const double c1 = psi - dpsi * a1;
      const double s2 = dphi * a2 * a2;
      const double c2 = phi - dphi * a2;
      const double c = 1.0 / rho + c1 + c2;
      // c eta^2 - B eta + C = 0 with C = f a1 a2, root between a1 and a2
      const double B = c * (a1 + a2) + s1 + s2;
      const double C = f * a1 * a2;
      double disc = B * B - 4.0 * c * C;
      if (disc < 0.0) disc = 0.0;
      const double sq = sqrt(disc);
      if (c == 0.0) eta = C / B;
      else if (B >= 0.0) eta = (B + sq != 0.0) ? 2.0 * C / (B + sq) : 0.0;
      else eta = (B - sq) / (2.0 * c);
      if (!(eta > a1 && eta < a2) && c != 0.0) {
        double alt = (B >= 0.0) ? (B + sq) / (2.0 * c) : ((B - sq != 0.0) ? 2.0 * C / (B - sq) : 0.0);
        eta = alt;
      }
    } else {
      const double s1 = dpsi * a1 * a1;
      const double c1 = psi - dpsi * a1;
      const double c = 1.0 / rho + c1;
      eta = (c != 0.0) ? (a1 + s1 / c) : 0.0;
    }
    double tn = tau + eta;
    if (!(tn > lo_b && tn < hi_b) || !isfinite(tn)) tn = 0.5 * (lo_b + hi_b);
    if (tn == tau || fabs(tn - tau) <= 2.0 * kEps * fabs(tau)) {
      tau = tn;
      break;
    }
    tau = tn;
  }
  *tau_out = tau;
  *org_out = o;
}

// grid (ceil(Kmax*32/256), nm), block 256: one warp per root
__global__ void merge_secular_kernel(LevelArgs a) {
  const int m = blockIdx.y;
  const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long lo = (long)m * a.N;
  const int K = a.desc[8 * m + D_K];
  if (j >= K) return;
  double tau;
  int o;
  secular_root_warp(K, j, a.dK + lo, a.zK + lo, a.rho[m], &tau, &o);
  if ((threadIdx.x & 31) == 0) {
    a.tau[lo + j] = tau;
    a.org[lo + j] = o;
  }
}

// z_hat_i^2 = -(d_i - lambda_i) prod_{j != i} (d_i - lambda_j) / (d_i - d_j).
// One warp per i; each lane keeps its partial product as mantissa * 2^e so
// that no partial product over- or underflows.
__global__ void merge_loewner_kernel(LevelArgs a) {
  const int m = blockIdx.y;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long lo = (long)m * a.N;
  const int K = a.desc[8 * m + D_K];
  if (i >= K) return;
  const double* dK = a.dK + lo;
  const double di = dK[i];
  double w = 1.0;
  int ex = 0;
  for (int j = lane; j < K; j += 32) {
    const double delta = (di - dK[a.org[lo + j]]) - a.tau[lo + j];
    w *= (j == i) ? delta : delta / (di - dK[j]);
    int e2;
    w = frexp(w, &e2);
    ex += e2;
  }
#pragma unroll
  for (int mm = 16; mm > 0; mm >>= 1) {
    const double ow = __shfl_xor_sync(0xffffffffu, w, mm);
    const int oe = __shfl_xor_sync(0xffffffffu, ex, mm);
    int e2;
    w = frexp(w * ow, &e2);
    ex += oe + e2;
  }
  if (lane == 0) {
    const double wv = ldexp(w, ex);
    const double z = sqrt(fmax(0.0, -wv));
    a.zh[lo + i] = (a.zK[lo + i] >= 0.0) ? z : -z;
  }
}

// U(:, j): v_i = zhat_i / (d_i - lambda_j), normalised; rows placed in the
// type order of Ut (types 1,2) and Ub (types 2,3).  grid (Kmax, nm), block 256.
__global__ void merge_vectors_kernel(LevelArgs a) {
  const int m = blockIdx.y;
  const int j = blockIdx.x;
  const long lo = (long)m * a.N;
  const int* d_ = a.desc + 8 * m;
  const int K = d_[D_K], K1 = d_[D_K1], K2 = d_[D_K2], K3 = d_[D_K3];
  double* Ut = a.Ut + (long)m * a.K12max * a.Kmax;
  double* Ub = a.Ub + (long)m * a.K23max * a.Kmax;
  __shared__ double red[32];
  __shared__ double s_norm;
  if (j >= K) {
    for (int i = threadIdx.x; i < a.K12max; i += blockDim.x) Ut[i + (long)j * a.K12max] = 0.0;
    for (int i = threadIdx.x; i < a.K23max; i += blockDim.x) Ub[i + (long)j * a.K23max] = 0.0;
    return;
  }
  const double* dK = a.dK + lo;
  const double dorg = dK[a.org[lo + j]];
  const double tj = a.tau[lo + j];
  double ss = 0.0;
  for (int i = threadIdx.x; i < K; i += blockDim.x) {
    double v = a.zh[lo + i] / ((dK[i] - dorg) - tj);
    ss = fma(v, v, ss);
  }
  ss = warp_sum(ss);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) s_norm = (t > 0.0) ? 1.0 / sqrt(t) : 0.0;
  }
  __syncthreads();
  const double inv = s_norm;
  for (int i = threadIdx.x; i < K; i += blockDim.x) {
    double v = a.zh[lo + i] / ((dK[i] - dorg) - tj) * inv;
    int pt = a.pT[lo + i], pb = a.pB[lo + i];
    if (pt >= 0) Ut[pt + (long)j * a.K12max] = v;
    if (pb >= 0) Ub[pb + (long)j * a.K23max] = v;
  }
  for (int i = K1 + K2 + threadIdx.x; i < a.K12max; i += blockDim.x) Ut[i + (long)j * a.K12max] = 0.0;
  for (int i = K2 + K3 + threadIdx.x; i < a.K23max; i += blockDim.x) Ub[i + (long)j * a.K23max] = 0.0;
}

// Final ascending order of the merged eigenvalues and scatter of the vectors
// back into Zw[lo:hi, lo:hi].  grid (ceil(N/256), nm): thread = output source.
__global__ void merge_finalize_rank_kernel(LevelArgs a) {
  const int m = blockIdx.y;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;  // source index: roots then deflated
  if (q >= a.N) return;
  const long lo = (long)m * a.N;
  const int* d_ = a.desc + 8 * m;
  const int K = d_[D_K], nd = d_[D_NDEF];
  const double* dK = a.dK + lo;
  auto value = [&](int src) -> double {
    if (src < K) return dK[a.org[lo + src]] + a.tau[lo + src];
    return a.dD[lo + (src - K)];
  };
  if (q >= K + nd) return;
  const double v = value(q);
  int rank = 0;
  if (q < K) {
    rank = q;  // roots are ascending
    for (int t = 0; t < nd; ++t) rank += (a.dD[lo + t] < v) ? 1 : 0;
  } else {
    // roots <= v, deflated (< v or equal with smaller index)
    int l = 0, h = K;
    while (l < h) {
      int md = (l + h) >> 1;
      if (value(md) <= v) l = md + 1; else h = md;
    }
    rank = l;
    const int t0 = q - K;
    for (int t = 0; t < nd; ++t) {
      double w = a.dD[lo + t];
      rank += (w < v || (w == v && t < t0)) ? 1 : 0;
    }
  }
  a.zv[lo + rank] = v;          // new eigenvalue at its sorted position
  a.perm[lo + rank] = q;        // source column in Zn
}

// Zw[lo:hi, lo + p] = Zn[:, perm[p]], dw[lo + p] = sorted value.
// grid (ceil(N/256), ceil(N/kColChunk), nm): thread = row, blockIdx.y = columns.
__global__ void merge_scatter_kernel(LevelArgs a) {
  const int m = blockIdx.z;
  const int p0 = blockIdx.y * kColChunk;
  const long lo = (long)m * a.N;
  const int p1 = min(a.N, p0 + kColChunk);
  if (blockIdx.x == 0 && p0 + (int)threadIdx.x < p1)
    a.dw[lo + p0 + threadIdx.x] = a.zv[lo + p0 + threadIdx.x];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.N) return;
  const double* Zn = a.Zn + (long)m * a.N * a.N;
  for (int p = p0; p < p1; ++p) {
    int q = a.perm[lo + p];
    if (q < 0 || q >= a.N) {
      atomicCAS(a.err, 0, kDevBadShape);
      return;
    }
    a.Zw[(lo + r) + (lo + p) * a.ldz] = Zn[r + (long)q * a.N];
  }
}

__global__ void finish_kernel(long n, long np, const double* dw, const double* Zw, long ldzw,
                              const double* scal, double* d, double* Z, long ldz) {
  const double nrm = scal[0];
  const double s = (nrm > 0.0) ? nrm : 1.0;
  for (long j = blockIdx.y; j < n; j += gridDim.y) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
      Z[i + j * ldz] = Zw[i + j * ldzw];
    if (blockIdx.x == 0 && threadIdx.x == 0) d[j] = dw[j] * s;
  }
}

}  // namespace

long stedc_ws_doubles(long n) { return n <= 1 ? 8 : make_plan(n).total_d; }
long stedc_ws_ints(long n) { return n <= 1 ? 8 : make_plan(n).total_i; }

// oz != nullptr: merges whose products exceed kOzMergeMin multiply-adds run
// them as emulated FP64 products on the integer tensor cores (one per merge),
// the smaller ones stay on the batched DMMA GEMM.
constexpr double kOzMergeMin = 64.0 * 1024 * 1024 * 1024;

// Integer workspace (bytes) of the emulated merges of an order-n solve: the
// largest merge product is (np/2) x np x (np/2) (np: the padded order).
long stedc_oz_bytes(long n, int nmod) {
  if (n <= 1) return 0;
  const long np = make_plan(n).np;
  return oz_layout(np / 2, np, np / 2 + 2, nmod, true).bytes;
}

// out_after: an event the stream waits for before Z is written (the solve
// itself keeps its eigenvectors in its own workspace until the last kernel),
// so that Z may alias a buffer that other streams are still reading.
int stedc(long n, double* d, double* e, double* Z, long ldz, double* work, long lwork, int* iwork,
          long liwork, cudaStream_t st, const OzWork* oz, cudaEvent_t out_after) {
  if (n < 0 || ldz < std::max(1L, n)) return EVD_ERR_INVALID_ARG;
  if (n == 0) return EVD_SUCCESS;
  if (!d || !Z || !work || !iwork || (n > 1 && !e)) return EVD_ERR_INVALID_ARG;
  if (n > (1L << 20)) return EVD_ERR_INVALID_ARG;
  if (n == 1) {
    const double one = 1.0;
    if (out_after) EVD_CUDA_TRY(cudaStreamWaitEvent(st, out_after, 0));
    EVD_CUDA_TRY(cudaMemcpyAsync(Z, &one, sizeof(double), cudaMemcpyHostToDevice, st));
    EVD_CUDA_TRY(cudaStreamSynchronize(st));
    return EVD_SUCCESS;
  }
  StedcPlan P = make_plan(n);
  if (lwork < P.total_d || liwork < P.total_i) return EVD_ERR_WORKSPACE;
  const long np = P.np;
  double* scal = work + P.o_scal;
  int* err = iwork + P.i_desc + 8 * (np / 2 + 1) + 8;
  EVD_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
  absmax_kernel<<<1, 1024, 0, st>>>(n, d, e, scal);
  EVD_LAUNCHED();
  {
    // A NaN or Inf entry would break the merge ordering (ranks of NaN keys
    // collide); reject it before any merge runs.
    double h = 0.0;
    EVD_CUDA_TRY(cudaMemcpyAsync(&h, scal, sizeof(double), cudaMemcpyDeviceToHost, st));
    EVD_CUDA_TRY(cudaStreamSynchronize(st));
    if (!isfinite(h)) return EVD_ERR_INVALID_ARG;
  }
  double* dw = work + P.o_d;
  double* ew = work + P.o_e;
  double* Zw = work + P.o_Z;
  init_kernel<<<ceil_div_i(np, 256), 256, 0, st>>>(n, np, P.s, d, e, scal, dw, ew);
  EVD_LAUNCHED();
  EVD_CUDA_TRY(cudaMemsetAsync(Zw, 0, sizeof(double) * np * np, st));
  const int nleaves = 1 << P.L;
  leaf_ql_kernel<<<ceil_div_i((long)nleaves * 32, 128), 128, 0, st>>>(P.s, nleaves, dw, ew, Zw,
                                                                       np, err);
  EVD_LAUNCHED();

  std::vector<int> hdesc;
  for (int lev = 1; lev <= P.L; ++lev) {
    LevelArgs a{};
    a.np = np;
    a.ldz = np;
    a.N = P.s << lev;
    a.n1 = a.N / 2;
    a.n2 = a.N - a.n1;
    a.nm = (int)(np / a.N);
    a.dw = dw;
    a.ew = ew;
    a.Zw = Zw;
    a.zv = work + P.o_zv;
    a.ds = work + P.o_ds;
    a.zs = work + P.o_zs;
    a.dK = work + P.o_dK;
    a.zK = work + P.o_zK;
    a.tau = work + P.o_tau;
    a.zh = work + P.o_zh;
    a.dD = work + P.o_dD;
    a.rc = work + P.o_rc;
    a.rs = work + P.o_rs;
    a.rho = work + P.o_rho;
    a.perm = iwork + P.i_perm;
    a.colK = iwork + P.i_colK;
    a.typK = iwork + P.i_typK;
    a.pT = iwork + P.i_pT;
    a.pB = iwork + P.i_pB;
    a.colD = iwork + P.i_colD;
    a.rA = iwork + P.i_rA;
    a.rB = iwork + P.i_rB;
    a.org = iwork + P.i_org;
    a.desc = iwork + P.i_desc;
    a.err = err;
    a.Qt = work + P.o_Qt;
    a.Qb = work + P.o_Qb;
    a.Ut = work + P.o_Ut;
    a.Ub = work + P.o_Ub;
    a.Zn = work + P.o_Zn;
    dim3 gN(ceil_div_i(a.N, 256), a.nm);
    merge_setup_kernel<<<gN, 256, 0, st>>>(a);
    EVD_LAUNCHED();
    merge_deflate_kernel<<<a.nm, kDefThreads, 0, st>>>(a);
    EVD_LAUNCHED();
    hdesc.resize(8 * a.nm);
    EVD_CUDA_TRY(cudaMemcpyAsync(hdesc.data(), a.desc, sizeof(int) * 8 * a.nm,
                                 cudaMemcpyDeviceToHost, st));
    EVD_CUDA_TRY(cudaStreamSynchronize(st));
    int Kmax = 0, K12 = 0, K23 = 0, nrmax = 0;
    for (int m = 0; m < a.nm; ++m) {
      const int* dd = &hdesc[8 * m];
      Kmax = std::max(Kmax, dd[D_K]);
      K12 = std::max(K12, dd[D_K1] + dd[D_K2]);
      K23 = std::max(K23, dd[D_K2] + dd[D_K3]);
      nrmax = std::max(nrmax, dd[D_NROT]);
    }
    a.Kmax = Kmax;
    // leading dimensions of Qt/Ut and Qb/Ub rounded up to even: 16-byte
    // aligned columns and batch strides keep the merge GEMMs on the lean
    // kernel's 16-byte copies (the padding is zero-filled by gather/vectors)
    a.K12max = (K12 + 1) & ~1;
    a.K23max = (K23 + 1) & ~1;
    if (nrmax > 0) {
      merge_rotate_kernel<<<gN, 256, 0, st>>>(a);
      EVD_LAUNCHED();
    }
    {
      const int cols = std::max(Kmax, std::max(a.K12max, a.K23max));
      if (cols > 0) {
        dim3 gG(ceil_div_i(a.N, 256), ceil_div_i(cols, kColChunk), a.nm);
        merge_gather_kernel<<<gG, 256, 0, st>>>(a);
        EVD_LAUNCHED();
      }
    }
    if (Kmax > 0) {
      dim3 gK(ceil_div_i((long)Kmax * 32, 256), a.nm);
      merge_secular_kernel<<<gK, 256, 0, st>>>(a);
      EVD_LAUNCHED();
      merge_loewner_kernel<<<gK, 256, 0, st>>>(a);
      EVD_LAUNCHED();
      merge_vectors_kernel<<<dim3(Kmax, a.nm), 256, 0, st>>>(a);
      EVD_LAUNCHED();
      // Zn[0:n1, 0:Kmax] = Qt Ut ; Zn[n1:N, 0:Kmax] = Qb Ub   (batched over merges)
      const long sZ = (long)a.N * a.N;
      const bool emul = oz && (double)a.n1 * Kmax * std::max(K12, K23) >= kOzMergeMin;
      if (K12 > 0) {
        if (emul) {
          for (int m = 0; m < a.nm; ++m)
            EVD_TRY(oz_gemm('n', 'n', a.n1, Kmax, K12, 1.0, a.Qt + (long)m * a.n1 * a.K12max,
                            a.n1, a.Ut + (long)m * a.K12max * Kmax, a.K12max, 0.0, nullptr, a.N,
                            0.0, a.Zn + (long)m * sZ, a.N, oz->nmod, false, oz->ws, oz->bytes,
                            st));
        } else {
          EVD_TRY(dgemm_batched('n', 'n', a.n1, Kmax, K12, 1.0, a.Qt, a.n1,
                                (long)a.n1 * a.K12max, a.Ut, a.K12max, (long)a.K12max * Kmax,
                                0.0, a.Zn, a.N, sZ, a.nm, st));
        }
      }
      if (K23 > 0) {
        if (emul) {
          for (int m = 0; m < a.nm; ++m)
            EVD_TRY(oz_gemm('n', 'n', a.n2, Kmax, K23, 1.0, a.Qb + (long)m * a.n2 * a.K23max,
                            a.n2, a.Ub + (long)m * a.K23max * Kmax, a.K23max, 0.0, nullptr, a.N,
                            0.0, a.Zn + a.n1 + (long)m * sZ, a.N, oz->nmod, false, oz->ws,
                            oz->bytes, st));
        } else {
          EVD_TRY(dgemm_batched('n', 'n', a.n2, Kmax, K23, 1.0, a.Qb, a.n2,
                                (long)a.n2 * a.K23max, a.Ub, a.K23max, (long)a.K23max * Kmax,
                                0.0, a.Zn + a.n1, a.N, sZ, a.nm, st));
        }
      }
      if (K12 == 0 || K23 == 0) {
        // the missing half of the root columns is zero
        for (int m = 0; m < a.nm; ++m) {
          long off = (long)m * sZ + (K12 == 0 ? 0 : a.n1);
          long rows = (K12 == 0) ? a.n1 : a.n2;
          EVD_CUDA_TRY(cudaMemset2DAsync(a.Zn + off, sizeof(double) * a.N, 0, sizeof(double) * rows,
                                         Kmax, st));
        }
      }
    }
    dim3 gC(ceil_div_i(a.N, 256), ceil_div_i(a.N, kColChunk), a.nm);
    merge_copy_deflated_kernel<<<gC, 256, 0, st>>>(a);
    EVD_LAUNCHED();
    merge_finalize_rank_kernel<<<gN, 256, 0, st>>>(a);
    EVD_LAUNCHED();
    merge_scatter_kernel<<<gC, 256, 0, st>>>(a);
    EVD_LAUNCHED();
  }
  dim3 gf(ceil_div_i(n, 256), (unsigned)std::min<long>(n, 65535));
  if (out_after) EVD_CUDA_TRY(cudaStreamWaitEvent(st, out_after, 0));
  finish_kernel<<<gf, 256, 0, st>>>(n, np, dw, Zw, np, scal, d, Z, ldz);
  EVD_LAUNCHED();
  return read_device_error(err, st);
}

}  // namespace evd

extern "C" long evd_stedc_work_size(long n) { return evd::stedc_ws_doubles(n < 0 ? 0 : n); }
extern "C" long evd_stedc_iwork_size(long n) { return evd::stedc_ws_ints(n < 0 ? 0 : n); }

extern "C" int evd_stedc(long n, double* d, double* e, double* Z, long ldz, double* work,
                         long lwork, int* iwork, long liwork, cudaStream_t stream) {
  return evd::stedc(n, d, e, Z, ldz, work, lwork, iwork, liwork, stream, nullptr, nullptr);
}
