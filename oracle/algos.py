"""numpy restatement of the reference's two-stage EVD path (test oracle).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker; never by the product.

Conventions follow the reference exactly: column-major FP64 matrices (numpy
arrays are used as mathematical matrices here), Householder vectors with
||u||^2 = 2 (H = I - u u^T), band storage sub[i, j] = A[j+i, j] with 2b rows.
Citations are file:line in the hansheng1001/EVD4SC2025 source tree.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg as sla

# ----------------------------------------------------------------- Householder

def house(x: np.ndarray) -> np.ndarray:
    """Householder vector with ||u||^2 = 2 such that (I - u u^T) x = -sign(x0)||x|| e1.

    Same steps as the chasing kernel (util/inc/bugle_chasingV10.h:137-188) and
    the TSQR leaf (util/inc/kernelQR.h:262-305): u = x/||x||; u0 += sign(u0)
    (sign(0) = +1); u /= sqrt(|u0|).  A zero x gives u = 0 (H = I); the
    reference divides by zero there.
    """
    x = np.asarray(x, dtype=np.float64)
    nrm2 = float(np.dot(x, x))
    if nrm2 == 0.0:
        return np.zeros_like(x)
    scale = 1.0 / math.sqrt(nrm2)
    u = x * scale
    u[0] += 1.0 if u[0] >= 0.0 else -1.0
    u *= 1.0 / math.sqrt(abs(u[0]))
    return u


# ------------------------------------------------------------------ band storage

def band_pack(A: np.ndarray, b: int) -> np.ndarray:
    """sub[i, j] = A[j+i, j] for i <= b, zero elsewhere; shape (2b, n).

    kernel_bugle_chasing_cpydA2dSubA, src/EVD/myEVD.cu:53-78.
    """
    n = A.shape[0]
    sub = np.zeros((2 * b, n))
    for i in range(b + 1):
        if i < n:
            sub[i, : n - i] = np.diagonal(A, -i)
    return sub


def band_to_dense(sub: np.ndarray, n: int) -> np.ndarray:
    """Symmetric dense matrix from (lower) band storage."""
    A = np.zeros((n, n))
    for i in range(sub.shape[0]):
        if i < n:
            idx = np.arange(n - i)
            A[idx + i, idx] = sub[i, : n - i]
            A[idx, idx + i] = sub[i, : n - i]
    return A


# ---------------------------------------------------------------- bulge chasing

def bulge_chase(sub: np.ndarray, n: int, b: int):
    """Band -> tridiagonal; returns (d, e, U, sub_out).

    Restates chasing_kernel_one_timeV10<32> (util/inc/bugle_chasingV10.h:21-392)
    with sweeps run one after another (the reference pipelines them; its
    progress rule at :81 makes the pipelined order equivalent).  Per step at
    opRow r: u = house(B1[:,0]) stored in U[r:r+rb, s] (:137-196); B1 <- H B1
    (:207-226); S2 <- H S2 H (:262-310); B1' <- B1' H (:315-336); the sweep
    ends when fewer than two rows remain below (:341-374).
    """
    sub = np.array(sub, dtype=np.float64, copy=True)
    U = np.zeros((n, n))

    def get_block(r0, c0, nr, nc):
        blk = np.zeros((nr, nc))
        for c in range(nc):
            col = c0 + c
            off = r0 - col
            blk[:, c] = sub[off: off + nr, col]
        return blk

    def put_block(blk, r0, c0):
        nr, nc = blk.shape
        for c in range(nc):
            col = c0 + c
            off = r0 - col
            sub[off: off + nr, col] = blk[:, c]

    def get_sym(r0, nr):
        S = np.zeros((nr, nr))
        for c in range(nr):
            S[c:, c] = sub[0: nr - c, r0 + c]
        return np.tril(S) + np.tril(S, -1).T

    def put_sym_lower(S, r0):
        nr = S.shape[0]
        for c in range(nr):
            sub[0: nr - c, r0 + c] = S[c:, c]

    for s in range(n - 2):
        r = s + 1
        rb = min(b, n - r)
        cb = 1
        B1 = get_block(r, s, rb, cb)
        while True:
            u = house(B1[:, 0])
            U[r: r + rb, s] = u
            B1 = B1 - np.outer(u, u @ B1)
            put_block(B1, r, r - cb)
            S2 = get_sym(r, rb)
            y = S2 @ u
            v = y - 0.5 * float(u @ y) * u
            S2 = S2 - np.outer(u, v) - np.outer(v, u)
            put_sym_lower(S2, r)
            r2 = r + rb
            rb2 = min(b, n - r2)
            if rb2 > 0:
                Bn = get_block(r2, r, rb2, rb)
                Bn = Bn - np.outer(Bn @ u, u)
            if rb2 <= 1:
                if rb2 == 1:
                    put_block(Bn, r2, r)
                break
            cb, rb, r, B1 = rb, rb2, r2, Bn
    d = sub[0, :n].copy()
    e = sub[1, : n - 1].copy()
    return d, e, U, sub


def q2_apply(X: np.ndarray, U: np.ndarray, n: int, b: int, transpose: bool) -> np.ndarray:
    """Apply the chasing reflectors stored in U to the rows of X.

    transpose=True : X <- Q2^T X, reflectors in generation order (what
                     my_BC_back_trans_v8_10_noBandU computes,
                     api/BC_backTransV8_10_noBandU.cu:60-232).
    transpose=False: X <- Q2 X (reverse order; the eigenvector direction).
    Q2 = prod_s prod_k H_{s,k}; the reflectors of one sweep act on disjoint
    row blocks, so each sweep is applied as one block-diagonal operator.
    """
    X = np.array(X, dtype=np.float64, copy=True)
    order = range(n - 2) if transpose else range(n - 3, -1, -1)
    for s in order:
        # a sweep's reflectors sit in b-row segments from row s+1; entries of U
        # where the sweep stored nothing are zero, which applies as identity
        for r in range(s + 1, n, b):
            u = U[r: r + b, s]
            X[r: r + b] -= np.outer(u, u @ X[r: r + b])
    return X


# ------------------------------------------------------------- panel QR / TSQR

def hou_tile(T: np.ndarray):
    """my_hou_kernel<128,32> for double (util/inc/kernelQR.h:215-414).

    Householder QR of an mm x n tile (mm <= 128): returns the explicit thin Q
    (mm x n, :379-413) and R (n x n) with R[j,j] = -sign(x0)*||x|| (:283-287).
    """
    A = np.array(T, dtype=np.float64, copy=True)
    mm, n = A.shape
    RR = np.zeros(n)
    for col in range(n):
        x = A[col:, col]
        nrm = math.sqrt(float(x @ x))
        A[col:, col] *= 1.0 / nrm
        u1 = A[col, col]
        A[col, col] += 1.0 if u1 >= 0 else -1.0
        RR[col] = -nrm if u1 >= 0 else nrm
        A[col:, col] *= 1.0 / math.sqrt(abs(A[col, col]))
        u = A[col:, col]
        if col + 1 < n:
            utx = u @ A[col:, col + 1:]
            A[col:, col + 1:] -= np.outer(u, utx)
    R = np.triu(A[:n, :n], 1) + np.diag(RR)
    V = np.tril(A)  # Householder vectors (zeros above the diagonal)
    Q = np.zeros((mm, n))
    for h in range(n):
        q = np.zeros(mm)
        q[h] = 1.0
        for hh in range(h, -1, -1):
            u = V[:, hh]
            q -= (q @ u) * u
        Q[:, h] = q
    return Q, R


def tsqr(A: np.ndarray, tile: int = 128):
    """hou_tsqr_panel<double,128,32> (api/inc/TallShinnyQR.h:9-133).

    Leaf QR on 128-row tiles, R factors stacked (32 rows each) and factored
    recursively, then Q_tile <- Q_tile * Qstack[32t:32t+32] (:66-131).
    """
    m, n = A.shape
    if m <= tile:
        return hou_tile(A)
    if (m % tile) % n != 0:
        raise ValueError("hou_tsqr_panel requires (m % 128) % n == 0 (TallShinnyQR.h:37-41)")
    nblk = (m + tile - 1) // tile
    Q = np.zeros((m, n))
    stack = np.zeros((nblk * n, n))
    for t in range(nblk):
        r0, r1 = t * tile, min(m, t * tile + tile)
        Qt, Rt = hou_tile(A[r0:r1])
        Q[r0:r1] = Qt
        stack[t * n:(t + 1) * n] = Rt
    Qs, R = tsqr(stack, tile)
    for t in range(nblk):
        r0, r1 = t * tile, min(m, t * tile + tile)
        Q[r0:r1] = Q[r0:r1] @ Qs[t * n:(t + 1) * n]
    return Q, R


def lu_nopivot(A: np.ndarray):
    """Unpivoted LU of a tall m x n matrix: A = L U (L unit lower m x n)."""
    A = np.array(A, dtype=np.float64, copy=True)
    m, n = A.shape
    for k in range(n):
        A[k + 1:, k] /= A[k, k]
        if k + 1 < n:
            A[k + 1:, k + 1:] -= np.outer(A[k + 1:, k], A[k, k + 1:])
    L = np.tril(A, -1)[:, :n]
    L[np.arange(n), np.arange(n)] = 1.0
    U = np.triu(A[:n, :n])
    return L, U


def panel_qr(A: np.ndarray):
    """panelQR<double> leaf path (api/panelQR.cu:54-108) for n <= 32.

    TSQR -> I - Q -> unpivoted getrf -> Y = unit-lower L -> W = (I-Q) L1^{-T}.
    Returns (Y, W, R) with Q_full = I - W Y^T and Q_full^T A = [R; 0].
    """
    m, n = A.shape
    Q, R = tsqr(A)
    IQ = np.eye(m, n) - Q
    L, _ = lu_nopivot(IQ)
    W = sla.solve_triangular(L[:n, :n], IQ.T, lower=True, unit_diagonal=True).T
    return L, W, R


# --------------------------------------------------------------------- sy2sb

def sy2sb(A: np.ndarray, b: int, nb: int):
    """my_ZY_ZY_SBR_Vector<double> (api/zy_zy_sy2sb.cu:24-486).

    Returns (band, W, Y): band = symmetric banded B (after copyMatrixL2U,
    src/EVD/myEVD.cu:346) with A = Q1 B Q1^T, Q1 = prod_p (I - W_p Y_p^T); the
    factors of panel p are stored at rows (p+1)b.., columns pb..pb+b-1.
    """
    M = A.shape[0]
    if M % nb != 0 or nb % b != 0:
        raise ValueError("M must be divisible by nb (zy_zy_sy2sb.cu:51-55)")
    OA = np.array(A, dtype=np.float64, copy=True)   # dOriA (working copy)
    dA = np.array(A, dtype=np.float64, copy=True)   # band output / lazily updated panels
    W = np.zeros((M, M))
    Y = np.zeros((M, M))
    off = 0
    while True:
        N = M - off
        Z = np.zeros((N, nb))                          # frame-local dZ
        i = b
        while i <= nb and i < N:
            m = N - i
            g0 = off + i                               # global row/col of the trailing part
            panel = dA[g0:, g0 - b:g0]
            Yp, Wp, Rp = panel_qr(panel)               # :100-111
            Y[g0:, g0 - b:g0] = Yp                      # copyMatrix -> dY (:122-123)
            W[g0:, g0 - b:g0] = Wp
            dA[g0:, g0 - b:g0] = 0.0                    # getU -> band R (:125)
            dA[g0:g0 + b, g0 - b:g0] = np.triu(Rp)
            Zp = OA[g0:, g0:] @ Wp                      # :134-155 / :202-220
            if i > b:
                Zprev = Z[i:, : i - b]
                Yprev = Y[g0:, off: off + i - b]
                Zp -= Yprev @ (Zprev.T @ Wp)           # :223-263
                Zp -= Zprev @ (Yprev.T @ Wp)           # :266-304
            Zp -= 0.5 * Yp @ (Wp.T @ Zp)               # :158-197 / :307-347
            Z[i:, i - b:i] = Zp
            if i < nb:                                  # lazy next-panel update (:351-395)
                Yi = Y[g0:, off: off + i]
                Zi = Z[i:, :i]
                dA[g0:, g0:g0 + b] -= Yi @ Zi[:b].T + Zi @ Yi[:b].T
            i += b
        if N - nb <= 0:
            break
        t0 = off + nb                                  # trailing syr2k (:422-433) + L2U + copy (:436-450)
        Yt = Y[t0:, off: off + nb]
        Zt = Z[nb:, :nb]
        upd = Yt @ Zt.T
        OA[t0:, t0:] -= upd + upd.T
        OA[t0:, t0:] = np.tril(OA[t0:, t0:]) + np.tril(OA[t0:, t0:], -1).T
        dA[t0:, t0:] = OA[t0:, t0:]
        off += nb
    band = np.tril(dA) + np.tril(dA, -1).T
    return band, W, Y


def q1_apply(X: np.ndarray, W: np.ndarray, Y: np.ndarray, n: int, b: int) -> np.ndarray:
    """X <- Q1 X with Q1 = prod_p (I - W_p Y_p^T) (panel order), last panel first.

    The same operator the reference builds explicitly in my_SBRBack_BCBack
    (src/EVD/myEVD.cu:148-233) before its final GEMM (:564).
    """
    X = np.array(X, dtype=np.float64, copy=True)
    npan = (n - 1) // b
    for p in range(npan - 1, -1, -1):
        r0 = (p + 1) * b
        if r0 >= n:
            continue
        Wp = W[r0:, p * b:(p + 1) * b]
        Yp = Y[r0:, p * b:(p + 1) * b]
        X[r0:] -= Wp @ (Yp.T @ X[r0:])
    return X


def wy_from_slide(W: np.ndarray, Y: np.ndarray, slide: int) -> np.ndarray:
    """computerWYFromSlide (api/computerWYFromSlide.cu:5-25): sequential merge."""
    W = np.array(W, dtype=np.float64, copy=True)
    M, N = W.shape
    b = slide
    i = 2 * b
    while i <= N:
        work = Y[:, : i - b].T @ W[:, i - b:i]
        W[:, i - b:i] -= W[:, : i - b] @ work
        i += b
    return W


def q_from_wy(W: np.ndarray, Y: np.ndarray) -> np.ndarray:
    """computerQFromWY (api/computerQFromWY.cu:5-17): Q = I - W Y^T."""
    M = W.shape[0]
    return np.eye(M) - W @ Y.T


# ------------------------------------------------------------------- metrics

def orthogonality(A: np.ndarray, B: np.ndarray | None = None) -> float:
    """||A^T B - I||_F / M (util/tool/checkMetric.cu:5-24)."""
    B = A if B is None else B
    M = A.shape[1]
    G = A.T @ B - np.eye(M)
    return float(np.linalg.norm(G) / M)


def residual(A: np.ndarray, w: np.ndarray, X: np.ndarray) -> float:
    """||A X - X diag(w)||_F / (n ||A||_F)."""
    n = A.shape[0]
    return float(np.linalg.norm(A @ X - X * w) / (n * np.linalg.norm(A)))


# ----------------------------------------------------------- whole pipeline

def tridiag_eig(d: np.ndarray, e: np.ndarray):
    """LAPACK dstevd (divide and conquer) on the tridiagonal, the oracle for the
    reference's host LAPACKE_dstedc('I') (src/EVD/myEVD.cu:529)."""
    from scipy.linalg import lapack
    w, Z, info = lapack.dstevd(np.array(d, dtype=np.float64), np.array(e, dtype=np.float64),
                               compute_v=1)
    if info != 0:
        raise RuntimeError(f"dstevd info={info}")
    return w, Z


def syevd_two_stage(A: np.ndarray, b: int = 32, nb: int = 1024):
    """The reference pipeline of src/EVD/myEVD.cu:251-706 in numpy.

    sy2sb -> band pack -> bulge chasing -> dstedc -> X = Q1 Q2 Z.
    Returns (w, X, stages) with the intermediate results in `stages`.
    """
    n = A.shape[0]
    band, W, Y = sy2sb(A, b, nb)
    sub = band_pack(band, b)
    d, e, U, _ = bulge_chase(sub, n, b)
    w, Z = tridiag_eig(d, e)
    X = q2_apply(Z, U, n, b, transpose=False)
    X = q1_apply(X, W, Y, n, b)
    return w, X, {"band": band, "W": W, "Y": Y, "d": d, "e": e, "U": U, "Z": Z}


# ------------------------------------------------------------------- inputs

def sym_gaussian(n: int, seed: int) -> np.ndarray:
    """A = (G + G^T)/2, G i.i.d. N(0,1) from numpy default_rng(seed)."""
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    return (G + G.T) * 0.5


def haar_orthogonal(n: int, seed: int) -> np.ndarray:
    """Haar-distributed orthogonal Q: QR of a seeded Gaussian, sign(diag R) fixed."""
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    Q, R = np.linalg.qr(G)
    return Q * np.sign(np.diag(R))


def spectrum(kind: str, n: int, seed: int) -> np.ndarray:
    """Known spectra of the benchmark inputs (sorted ascending).

    geometric: |lambda| from 1 down to 1e-6 (or `geometric1e10`: to 1e-10), random signs;
    uniform: uniform on [-1, 1]; clustered: 100 clusters of width 1e-10.
    """
    rng = np.random.default_rng(seed + 7919)
    if kind in ("geometric", "geometric1e6"):
        mag = 10.0 ** (-6.0 * np.arange(n) / max(n - 1, 1))
        lam = mag * rng.choice([-1.0, 1.0], size=n)
    elif kind == "geometric1e10":
        mag = 10.0 ** (-10.0 * np.arange(n) / max(n - 1, 1))
        lam = mag * rng.choice([-1.0, 1.0], size=n)
    elif kind == "uniform":
        lam = rng.uniform(-1.0, 1.0, size=n)
    elif kind == "clustered":
        nclu = 100
        centers = np.linspace(-1.0, 1.0, nclu)
        per = -(-n // nclu)
        lam = np.concatenate([c + 1e-10 * rng.uniform(0, 1, per) for c in centers])[:n]
    else:
        raise ValueError(kind)
    return np.sort(lam)


def known_spectrum_matrix(kind: str, n: int, seed: int):
    """A = Q diag(lambda) Q^T with Haar Q; returns (A, lambda)."""
    lam = spectrum(kind, n, seed)
    Q = haar_orthogonal(n, seed)
    A = (Q * lam) @ Q.T
    A = 0.5 * (A + A.T)
    return A, lam


# ------------------------------------------------------------------ refinement

def refine_syev(A: np.ndarray, X: np.ndarray, iters: int = 1):
    """Ogita-Aishima refinement (RefSyEv, Japan J. Indust. Appl. Math. 35
    (2018), Algorithm 1) as the library's evd_refine_syev applies it; the
    reference has no refinement step.

    Per iteration: R = I - X^T X, S = X^T A X, l_i = s_ii / (1 - r_ii);
    delta = 2 (||S - diag(l)||_2 + ||A||_2 ||R||_2) with ||A||_2 taken as
    max |l_i|, floored at 1e8 sqrt(n) u max |l_i| (below it the rounding
    noise of S would dominate a correction); E_ij = (s + l_j r_ij) / (l_j - l_i)
    with s = (s_ij + s_ji) / 2 where |l_i - l_j| > delta, r_ij / 2 otherwise;
    X <- X + X E.  Norms are exact here (the library estimates them by
    power iteration).  Returns (l of the last iteration, X)."""
    A = np.asarray(A, dtype=np.float64)
    X = np.array(X, dtype=np.float64)
    n = A.shape[0]
    lam = np.zeros(n)
    u = np.finfo(np.float64).eps / 2
    for _ in range(iters):
        R = np.eye(n) - X.T @ X
        S = X.T @ (A @ X)
        lam = np.diag(S) / (1.0 - np.diag(R))
        normA = np.abs(lam).max() if n else 0.0
        D = S - np.diag(lam)
        delta = 2.0 * (np.linalg.norm(D, 2) + normA * np.linalg.norm(R, 2))
        delta = max(delta, 1e8 * math.sqrt(n) * u * normA)
        Ss = 0.5 * (S + S.T)
        gap = lam[None, :] - lam[:, None]           # gap[i, j] = l_j - l_i
        far = np.abs(gap) > delta
        np.fill_diagonal(far, False)
        with np.errstate(divide="ignore", invalid="ignore"):
            E = np.where(far, (Ss + lam[None, :] * R) / np.where(far, gap, 1.0), 0.5 * R)
        X = X + X @ E
    return lam, X
