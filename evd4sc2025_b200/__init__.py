"""B200-native two-stage symmetric eigensolver (FP64, sm_100a).

Host-side mirror of the hansheng1001/EVD4SC2025 entry points, over the C ABI
in ``include/evd_b200.h``.  Device memory and streams come from PyTorch
(plumbing only); every computation runs in ``libevd_b200.so``.

Matrices are column-major as in the reference.  A column-major ``m x n``
matrix is a torch tensor of shape ``(m, n)`` with ``stride(0) == 1`` (see
:func:`empty_cm` / :func:`to_cm`); its leading dimension is ``stride(1)``.

Reference name        -> function here
``myEVD n b nb``      -> :func:`syevd` (and the ``bin/myEVD`` CLI)
``my_ZY_ZY_SBR_Vector`` -> :func:`sy2sb`
``panelQR``           -> :func:`panel_qr`
``hou_tsqr_panel``    -> :func:`tsqr`
``tc_ozimmu_syr2k``   -> :func:`syr2k`
bulge chasing kernel  -> :func:`bulge_chase`
``my_BC_back_trans_v8_10_noBandU`` -> :func:`bc_back`
``computerWYFromSlide`` -> :func:`wy_from_slide`
``computerQFromWY``   -> :func:`q_from_wy`
``checkOrthogonality`` -> :func:`check_orthogonality`
host ``LAPACKE_dstedc`` -> :func:`stedc` (device divide and conquer)
``panelQR<float/half>``, ``tc_ozimmu_syr2k<float/half>``, ``tc_syr2k``
                      -> :mod:`evd4sc2025_b200.lowprec`
``writeMatrixToCsvV2`` / ``readMatrixFromFile`` -> :mod:`evd4sc2025_b200.matio`

Beyond the reference: :func:`syevd_values` (eigenvalues only), any order n in
:func:`syevd`, :func:`refine_syev` (Ogita-Aishima refinement),
:mod:`evd4sc2025_b200.serve` (batched solves, serving loop),
:mod:`evd4sc2025_b200.autotune` (nb per order).
"""
from __future__ import annotations

import ctypes as C

import torch

from ._native import EvdError, call, lib  # noqa: F401

__all__ = [
    "EvdError", "lib", "empty_cm", "to_cm", "dgemm", "syr2k", "band_pack", "bulge_chase",
    "tsqr", "panel_qr", "sy2sb", "stedc", "bc_back", "bc_back_apply", "wy_from_slide",
    "q_from_wy", "sbr_back", "check_orthogonality", "check_eig", "syevd", "last_timings",
    "syevd_values", "eigvalsh", "stebz", "refine_syev", "refine_work", "dgemm_ozaki",
    "dgemm_ozaki_work_size", "ozaki_bits", "refine_syev_ozaki", "refine_ozaki_work",
    "syevd_mixed", "syevd_s", "MixedWorkspace", "last_refine_ms", "mixed_last_timings",
    # reference-named aliases
    "my_ZY_ZY_SBR_Vector", "panelQR", "hou_tsqr_panel", "tc_ozimmu_syr2k",
    "my_BC_back_trans_v8_10_noBandU", "computerWYFromSlide", "computerQFromWY",
    "checkOrthogonality", "myEVD",
]

F64 = torch.float64


def _stream(stream=None) -> int:
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def empty_cm(m: int, n: int, device="cuda", dtype=F64, ld: int | None = None) -> torch.Tensor:
    """Uninitialised column-major ``m x n`` matrix with leading dimension ``ld``."""
    ld = m if ld is None else ld
    buf = torch.empty((n, max(ld, 1)), dtype=dtype, device=device)
    return buf[:, :m].t()


def zeros_cm(m: int, n: int, device="cuda", dtype=F64, ld: int | None = None) -> torch.Tensor:
    ld = m if ld is None else ld
    buf = torch.zeros((n, max(ld, 1)), dtype=dtype, device=device)
    return buf[:, :m].t()


def to_cm(t: torch.Tensor, device="cuda", ld: int | None = None) -> torch.Tensor:
    """Column-major FP64 copy of a 2-D tensor on ``device``."""
    m, n = t.shape
    out = empty_cm(m, n, device=device, ld=ld)
    out.copy_(t.to(device=device, dtype=F64))
    return out


def _cm(t: torch.Tensor, name: str, dtype=F64):
    """(pointer, leading dimension) of a column-major CUDA matrix of `dtype`."""
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {str(dtype).replace('torch.', '')}")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dim() == 1:
        return C.c_void_p(t.data_ptr()), max(1, t.shape[0])
    if t.shape[0] > 1 and t.stride(0) != 1:
        raise ValueError(f"{name} must be column-major (stride(0) == 1); use to_cm()")
    ld = t.stride(1) if t.shape[1] > 1 else max(1, t.shape[0])
    return C.c_void_p(t.data_ptr()), max(ld, t.shape[0], 1)


def _ptr(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


# --------------------------------------------------------------------------- GEMM
def dgemm(transa: str, transb: str, alpha: float, A: torch.Tensor, B: torch.Tensor,
          beta: float, Cm: torch.Tensor, stream=None) -> torch.Tensor:
    """C = alpha*op(A)*op(B) + beta*C on the FP64 DMMA kernel (in place)."""
    m, n = Cm.shape
    k = A.shape[0] if transa.lower() == "t" else A.shape[1]
    pa, lda = _cm(A, "A")
    pb, ldb = _cm(B, "B")
    pc, ldc = _cm(Cm, "C")
    call("evd_dgemm", transa.encode(), transb.encode(), m, n, k, alpha, pa, lda, pb, ldb,
         beta, pc, ldc, _stream(stream))
    return Cm


def dgemm_ozaki(transa: str, transb: str, alpha: float, A: torch.Tensor, B: torch.Tensor,
                beta: float, Cm: torch.Tensor, moduli: int = 14, work: torch.Tensor | None = None,
                stream=None) -> torch.Tensor:
    """C = alpha*op(A)*op(B) + beta*C (in place) as an emulated FP64 product on
    the integer tensor cores (Ozaki scheme II with ``moduli`` moduli; 14 give
    53-bit operands).  ``work``: a uint8 device tensor of at least
    :func:`dgemm_ozaki_work_size` bytes (allocated per call when omitted)."""
    m, n = Cm.shape
    k = A.shape[0] if transa.lower() == "t" else A.shape[1]
    need = dgemm_ozaki_work_size(transa, transb, m, n, k, moduli)
    if work is None:
        work = torch.empty(need, dtype=torch.uint8, device=Cm.device)
    pa, lda = _cm(A, "A")
    pb, ldb = _cm(B, "B")
    pc, ldc = _cm(Cm, "C")
    call("evd_dgemm_ozaki", transa.encode(), transb.encode(), m, n, k, alpha, pa, lda, pb, ldb,
         beta, pc, ldc, moduli, _ptr(work), work.numel(), _stream(stream))
    return Cm


def dgemm_ozaki_work_size(transa: str, transb: str, m: int, n: int, k: int,
                          moduli: int = 14) -> int:
    """Workspace bytes of :func:`dgemm_ozaki`."""
    need = int(lib().evd_dgemm_ozaki_work_size(transa.encode(), transb.encode(), m, n, k, moduli))
    if need <= 0:
        raise EvdError("evd_dgemm_ozaki_work_size", -1)
    return need


def ozaki_bits(moduli: int, k: int) -> int:
    """Integer bits P of the emulated product's operands."""
    return int(lib().evd_ozaki_bits(moduli, k))


def syr2k(alpha: float, A: torch.Tensor, B: torch.Tensor, beta: float, Cm: torch.Tensor,
          nb: int = 0, stream=None) -> torch.Tensor:
    """C(lower) = alpha*(A B^T + B A^T) + beta*C(lower); upper mirrored (tc_ozimmu_syr2k)."""
    n, k = A.shape
    pa, lda = _cm(A, "A")
    pb, ldb = _cm(B, "B")
    pc, ldc = _cm(Cm, "C")
    call("evd_syr2k_lower_mirror", n, k, alpha, pa, lda, pb, ldb, beta, pc, ldc, nb,
         _stream(stream))
    return Cm


tc_ozimmu_syr2k = syr2k


# ------------------------------------------------------------------ bulge chasing
def band_pack(A: torch.Tensor, b: int, stream=None) -> torch.Tensor:
    """Lower band of A in band storage (2b x n, sub[i, j] = A[j+i, j])."""
    n = A.shape[0]
    pa, lda = _cm(A, "A")
    sub = empty_cm(2 * b, n, device=A.device)
    ps, lds = _cm(sub, "sub")
    call("evd_band_pack", n, b, pa, lda, ps, lds, _stream(stream))
    return sub


def bulge_chase(sub: torch.Tensor, b: int = 32, ldU: int | None = None, stream=None):
    """Band (2b x n band storage, overwritten) -> (d, e, U).

    U (ldU x n, column s = reflectors of sweep s) is zero-initialised here, as
    the reference clears dU before its chasing kernel (src/EVD/myEVD.cu:413).
    """
    n = sub.shape[1]
    dev = sub.device
    ldU = n if ldU is None else ldU
    U = zeros_cm(n, n, device=dev, ld=ldU)
    d = torch.empty(n, dtype=F64, device=dev)
    e = torch.empty(max(n - 1, 1), dtype=F64, device=dev)
    iw = torch.empty(max(1, lib().evd_bulge_chase_iwork_size(n) // 4), dtype=torch.int32,
                     device=dev)
    ps, lds = _cm(sub, "sub")
    pu, ldu = _cm(U, "U")
    call("evd_bulge_chase", n, b, ps, lds, pu, ldu, _ptr(d), _ptr(e), _ptr(iw), _stream(stream))
    return d, e[: max(n - 1, 0)], U


# --------------------------------------------------------------- panel / TSQR
def _work(ndoubles: int, device) -> torch.Tensor:
    return torch.empty(max(int(ndoubles), 1), dtype=F64, device=device)


def tsqr(A: torch.Tensor, stream=None):
    """Tall-skinny QR (hou_tsqr_panel<double,128,32>): A (m x 32) <- explicit Q; returns R."""
    m, n = A.shape
    pa, lda = _cm(A, "A")
    R = zeros_cm(n, n, device=A.device)
    pr, ldr = _cm(R, "R")
    lw = lib().evd_panel_qr_work_size(m, n)
    if lw <= 0:
        raise EvdError("evd_panel_qr_work_size", -1)
    w = _work(lw, A.device)
    call("evd_tsqr", m, n, pa, lda, pr, ldr, _ptr(w), lw, _stream(stream))
    return A, R


hou_tsqr_panel = tsqr


def panel_qr(A: torch.Tensor, stream=None):
    """panelQR<double>: A (m x 32) <- Y (unit lower); returns (Y, W, R), Q = I - W Y^T."""
    m, n = A.shape
    pa, lda = _cm(A, "A")
    W = zeros_cm(m, n, device=A.device)
    R = zeros_cm(n, n, device=A.device)
    pw, ldw = _cm(W, "W")
    pr, ldr = _cm(R, "R")
    lw = lib().evd_panel_qr_work_size(m, n)
    if lw <= 0:
        raise EvdError("evd_panel_qr_work_size", -1)
    w = _work(lw, A.device)
    call("evd_panel_qr", m, n, pa, lda, pw, ldw, pr, ldr, _ptr(w), lw, _stream(stream))
    return A, W, R


panelQR = panel_qr


# --------------------------------------------------------------------- sy2sb
def sy2sb(A: torch.Tensor, b: int = 32, nb: int = 1024, stream=None):
    """my_ZY_ZY_SBR_Vector: returns (band, W, Y) for the symmetric A (not modified).

    band is the symmetric band matrix B with A = Q1 B Q1^T, Q1 = prod (I - W_p Y_p^T).
    """
    n = A.shape[0]
    dev = A.device
    OA = to_cm(A, device=dev)
    dA = to_cm(A, device=dev)
    W = zeros_cm(n, n, device=dev)
    Y = zeros_cm(n, n, device=dev)
    Z = zeros_cm(n, nb, device=dev)
    R = zeros_cm(n, nb, device=dev)
    lw = lib().evd_sy2sb_work_size(n, b, nb)
    if lw <= 0:
        raise EvdError("evd_sy2sb_work_size", -1)
    w = _work(lw, dev)
    args = []
    for t, name in ((OA, "OA"), (dA, "A"), (W, "W"), (Y, "Y"), (Z, "Z"), (R, "R")):
        args.extend(_cm(t, name))
    call("evd_sy2sb", n, n, b, nb, *args, _ptr(w), lw, _stream(stream))
    return dA, W, Y


my_ZY_ZY_SBR_Vector = sy2sb


# -------------------------------------------------------------------- stedc
def stedc(d: torch.Tensor, e: torch.Tensor, stream=None):
    """Device divide and conquer for the tridiagonal (d, e): returns (w ascending, Z)."""
    n = d.shape[0]
    dev = d.device
    w = d.to(dtype=F64).clone()
    ee = torch.zeros(max(n, 1), dtype=F64, device=dev)
    if n > 1:
        ee[: n - 1] = e[: n - 1]
    Z = empty_cm(n, n, device=dev)
    pz, ldz = _cm(Z, "Z")
    lw = lib().evd_stedc_work_size(n)
    liw = lib().evd_stedc_iwork_size(n)
    wk = _work(lw, dev)
    iw = torch.empty(max(int(liw), 1), dtype=torch.int32, device=dev)
    call("evd_stedc", n, _ptr(w), _ptr(ee), pz, ldz, _ptr(wk), lw, _ptr(iw), liw, _stream(stream))
    return w, Z


# ----------------------------------------------------------- back transforms
def bc_back(Q: torch.Tensor, U: torch.Tensor, b: int = 32, stream=None) -> torch.Tensor:
    """my_BC_back_trans_v8_10_noBandU: Q <- Q2^T Q (in place)."""
    n = Q.shape[0]
    pq, ldq = _cm(Q, "Q")
    pu, ldu = _cm(U, "U")
    call("evd_bc_back", pq, ldq, pu, ldu, n, b, _stream(stream))
    return Q


my_BC_back_trans_v8_10_noBandU = bc_back


def bc_back_apply(X: torch.Tensor, U: torch.Tensor, b: int = 32, stream=None,
                  work: torch.Tensor | bool | None = True) -> torch.Tensor:
    """X <- Q2 X (in place): the chasing reflectors in reverse generation order.

    ``work``: a float64 CUDA tensor of at least evd_bc_back_work_size(n)
    elements for the precomputed T factors, True to allocate one here, or
    None to let the kernel rebuild them (no workspace).
    """
    n, ncols = X.shape
    px, ldx = _cm(X, "X")
    pu, ldu = _cm(U, "U")
    if work is True:
        work = torch.empty(max(1, lib().evd_bc_back_work_size(n)), dtype=F64, device=X.device)
    pw, lw = (None, 0) if work is None else (_ptr(work), work.numel())
    call("evd_bc_back_apply", n, ncols, pu, ldu, px, ldx, b, pw, lw, _stream(stream))
    return X


def wy_from_slide(W: torch.Tensor, Y: torch.Tensor, slide: int, stream=None) -> torch.Tensor:
    """computerWYFromSlide: W (M x N) merged in place."""
    M, N = W.shape
    pw, ldw = _cm(W, "W")
    py, ldy = _cm(Y, "Y")
    work = _work(M * slide, W.device)
    call("evd_wy_from_slide", M, N, slide, pw, ldw, py, ldy, _ptr(work), _stream(stream))
    return W


computerWYFromSlide = wy_from_slide


def q_from_wy(W: torch.Tensor, Y: torch.Tensor, stream=None) -> torch.Tensor:
    """computerQFromWY: Q = I - W Y^T (M x M)."""
    M, N = W.shape
    Q = empty_cm(M, M, device=W.device)
    pq, ldq = _cm(Q, "Q")
    pw, ldw = _cm(W, "W")
    py, ldy = _cm(Y, "Y")
    call("evd_q_from_wy", M, N, pq, ldq, pw, ldw, py, ldy, _stream(stream))
    return Q


computerQFromWY = q_from_wy


def sbr_back(X: torch.Tensor, W: torch.Tensor, Y: torch.Tensor, b: int = 32, nk: int = 1024,
             stream=None) -> torch.Tensor:
    """X <- Q1 X with the stage-1 panels in W/Y (W is overwritten by the slab merge)."""
    n, ncols = X.shape
    px, ldx = _cm(X, "X")
    pw, ldw = _cm(W, "W")
    py, ldy = _cm(Y, "Y")
    lw = lib().evd_sbr_back_work_size(n, b, nk)
    work = _work(lw, X.device)
    call("evd_sbr_back", n, b, nk, pw, ldw, py, ldy, px, ldx, ncols, _ptr(work), lw,
         _stream(stream))
    return X


# ------------------------------------------------------------------- metrics
def check_orthogonality(A: torch.Tensor, B: torch.Tensor | None = None, stream=None) -> float:
    """checkOrthogonality: ||A^T B - I||_F / M (A, B: N x M)."""
    B = A if B is None else B
    N, M = A.shape
    pa, lda = _cm(A, "A")
    pb, ldb = _cm(B, "B")
    work = _work(M * M + 1024, A.device)
    out = (C.c_double * 1)()
    call("evd_check_orthogonality", M, N, pa, lda, pb, ldb, _ptr(work), out, _stream(stream))
    return float(out[0])


checkOrthogonality = check_orthogonality


def check_eig(A: torch.Tensor, w: torch.Tensor, X: torch.Tensor, stream=None):
    """(||A X - X diag(w)||_F / (n ||A||_F), ||X^T X - I||_F / n) on the device."""
    n = A.shape[0]
    pa, lda = _cm(A, "A")
    px, ldx = _cm(X, "X")
    work = _work(2 * n * n + 1024, A.device)
    out = (C.c_double * 2)()
    call("evd_check_eig", n, pa, lda, _ptr(w), px, ldx, _ptr(work), out, _stream(stream))
    return float(out[0]), float(out[1])


# -------------------------------------------------------------- whole solver
class Workspace:
    """Reusable device workspace for :func:`syevd` (bytes from evd_syevd_work_size)."""

    def __init__(self, n: int, b: int = 32, nb: int = 1024, device="cuda"):
        nbytes = lib().evd_syevd_work_size(n, b, nb)
        if nbytes <= 0:
            raise EvdError("evd_syevd_work_size", -1)
        self.key = (n, b, nb)
        self.nbytes = int(nbytes)
        self.buf = torch.empty(self.nbytes, dtype=torch.uint8, device=device)


def syevd(A: torch.Tensor, b: int = 32, nb: int = 1024, ws: Workspace | None = None,
          timed: bool = False, stream=None, w: torch.Tensor | None = None,
          X: torch.Tensor | None = None):
    """All eigenvalues (ascending) and eigenvectors of the symmetric FP64 matrix A.

    The plain-FP64 two-stage pipeline of `myEVD n b nb`; A is not modified.
    """
    n = A.shape[0]
    dev = A.device
    if ws is None or ws.key != (n, b, nb):
        ws = Workspace(n, b, nb, device=dev)
    if w is None:
        w = torch.empty(n, dtype=F64, device=dev)
    if X is None:
        X = empty_cm(n, n, device=dev)
    pa, lda = _cm(A, "A")
    px, ldx = _cm(X, "X")
    call("evd_syevd", n, b, nb, pa, lda, _ptr(w), px, ldx, _ptr(ws.buf), ws.nbytes,
         1 if timed else 0, _stream(stream))
    return w, X


myEVD = syevd


class MixedWorkspace:
    """Reusable device workspace for :func:`syevd_mixed`.  ``minimal``: the
    smallest workspace the solve accepts (one stage-2 chain, the divide and
    conquer after the Q1 formation: slower, about 3.4 n^2 doubles less)."""

    def __init__(self, n: int, b: int = 32, nb: int = 1024, moduli: int = 14,
                 refine_iters: int = 0, device="cuda", minimal: bool = False):
        size_fn = (lib().evd_syevd_mixed_work_size_min if minimal
                   else lib().evd_syevd_mixed_work_size)
        nbytes = size_fn(n, b, nb, moduli, refine_iters)
        if nbytes <= 0:
            raise EvdError("evd_syevd_mixed_work_size", -1)
        self.key = (n, b, nb, moduli, refine_iters)
        self.minimal = minimal
        self.nbytes = int(nbytes)
        self.buf = torch.empty(self.nbytes, dtype=torch.uint8, device=device)


def syevd_mixed(A: torch.Tensor, b: int = 32, nb: int = 1024, moduli: int = 14,
                refine_iters: int = 0, moduli_update: int = 14,
                ws: MixedWorkspace | None = None, timed: bool = False, stream=None,
                w: torch.Tensor | None = None, X: torch.Tensor | None = None):
    """All eigenpairs of the symmetric FP64 matrix A by the mixed form of the
    solve: the stage-1 trailing SYR2K and the stage-1 back transformation as
    emulated products on the integer tensor cores with ``moduli`` moduli (14:
    FP64-level), then ``refine_iters`` Ogita-Aishima iterations on emulated
    FP64 products (X E with ``moduli_update``).  A is not modified."""
    n = A.shape[0]
    dev = A.device
    if ws is None or ws.key != (n, b, nb, moduli, refine_iters):
        ws = MixedWorkspace(n, b, nb, moduli, refine_iters, device=dev)
    if w is None:
        w = torch.empty(n, dtype=F64, device=dev)
    if X is None:
        X = empty_cm(n, n, device=dev)
    pa, lda = _cm(A, "A")
    px, ldx = _cm(X, "X")
    call("evd_syevd_mixed", n, b, nb, pa, lda, _ptr(w), px, ldx, moduli, refine_iters,
         moduli_update, _ptr(ws.buf), ws.nbytes, 1 if timed else 0, _stream(stream))
    return w, X


def syevd_s(A: torch.Tensor, b: int = 32, nb: int = 1024, work: torch.Tensor | None = None,
            stream=None, w: torch.Tensor | None = None, X: torch.Tensor | None = None):
    """All eigenpairs of the symmetric FP32 matrix A (column-major), in FP32:
    the mixed form of the solve with 8 moduli and no refinement (the
    contractions on the integer tensor cores at FP32 accuracy; panels, chase
    and divide and conquer in FP64).  A is not modified."""
    n = A.shape[0]
    dev = A.device
    nbytes = int(lib().evd_syevd_s_work_size(n, b, nb))
    if nbytes <= 0:
        raise ValueError("unsupported shape")
    if work is None or work.numel() < nbytes:
        work = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    if w is None:
        w = torch.empty(n, dtype=torch.float32, device=dev)
    if X is None:
        X = empty_cm(n, n, device=dev, dtype=torch.float32)
    pa, lda = _cm(A, "A", torch.float32)
    px, ldx = _cm(X, "X", torch.float32)
    call("evd_syevd_s", n, b, nb, pa, lda, _ptr(w), px, ldx, _ptr(work), work.numel(),
         _stream(stream))
    return w, X


def mixed_last_timings() -> dict:
    """Stage times (ms) of the last timed :func:`syevd_mixed` on this thread.
    q1_formation and stage2_chains (the stage-2 reflectors accumulated from the
    identity, one chase range behind the chase) run on side streams beside the
    chase and the divide and conquer; final_products (from the end of the
    divide and conquer to X) includes waiting for them."""
    out = (C.c_double * 8)()
    lib().evd_syevd_mixed_last_timings(out)
    keys = ("sy2sb", "bulge_chasing", "tridiagonal_dc", "q1_formation", "stage2_chains",
            "final_products", "refine", "total")
    return {k: float(v) for k, v in zip(keys, out)}


def last_refine_ms() -> float:
    """Refinement time (ms) of the last timed :func:`syevd_mixed` on this thread."""
    return float(lib().evd_syevd_last_refine_ms())


def syevd_values(A: torch.Tensor, b: int = 32, nb: int = 1024, ws: Workspace | None = None,
                 timed: bool = False, stream=None, w: torch.Tensor | None = None) -> torch.Tensor:
    """Eigenvalues only (ascending) of the symmetric FP64 matrix A: stage 1,
    the chase without reflectors, Sturm-count multisection; no vectors."""
    n = A.shape[0]
    dev = A.device
    if ws is None or ws.key != (n, b, nb):
        ws = Workspace(n, b, nb, device=dev)
    if w is None:
        w = torch.empty(n, dtype=F64, device=dev)
    pa, lda = _cm(A, "A")
    call("evd_syevd_values", n, b, nb, pa, lda, _ptr(w), _ptr(ws.buf), ws.nbytes,
         1 if timed else 0, _stream(stream))
    return w


eigvalsh = syevd_values


def refine_work(n: int, device="cuda") -> torch.Tensor:
    """Workspace of :func:`refine_syev` for order n (allocate it once and pass
    it to every call to keep allocation out of a timed loop)."""
    nw = int(lib().evd_refine_syev_work_size(n))
    if nw <= 0:
        raise EvdError("evd_refine_syev_work_size", -1)
    return torch.empty(nw, dtype=F64, device=device)


def refine_syev(A: torch.Tensor, X: torch.Tensor, iters: int = 2, w: torch.Tensor | None = None,
                stream=None, work: torch.Tensor | None = None):
    """Ogita-Aishima refinement of approximate eigenvectors X (in place) of
    the symmetric FP64 matrix A; returns (w, X) with w the refined
    eigenvalues in the column order of X.  ``work`` (from
    :func:`refine_work`) is allocated per call when omitted."""
    n = A.shape[0]
    if work is None:
        work = refine_work(n, A.device)
    nw = work.numel()
    if w is None:
        w = torch.empty(n, dtype=F64, device=A.device)
    pa, lda = _cm(A, "A")
    px, ldx = _cm(X, "X")
    call("evd_refine_syev", n, pa, lda, _ptr(w), px, ldx, iters, _ptr(work), nw, _stream(stream))
    return w, X


def refine_ozaki_work(n: int, moduli: int = 14, device="cuda") -> torch.Tensor:
    """Workspace (bytes) of :func:`refine_syev_ozaki` for order n."""
    nb = int(lib().evd_refine_syev_ozaki_work_size(n, moduli))
    if nb <= 0:
        raise EvdError("evd_refine_syev_ozaki_work_size", -1)
    return torch.empty(nb, dtype=torch.uint8, device=device)


def refine_syev_ozaki(A: torch.Tensor, X: torch.Tensor, iters: int = 2, moduli: int = 14,
                      moduli_update: int = 14, w: torch.Tensor | None = None, stream=None,
                      work: torch.Tensor | None = None):
    """Ogita-Aishima refinement (in place) with every product emulated on the
    integer tensor cores: A X, X^T X and X^T A X with ``moduli`` moduli, the
    update X E with ``moduli_update``.  Returns (w, X)."""
    n = A.shape[0]
    if work is None:
        work = refine_ozaki_work(n, moduli, A.device)
    if w is None:
        w = torch.empty(n, dtype=F64, device=A.device)
    pa, lda = _cm(A, "A")
    px, ldx = _cm(X, "X")
    call("evd_refine_syev_ozaki", n, pa, lda, _ptr(w), px, ldx, iters, moduli, moduli_update,
         _ptr(work), work.numel(), _stream(stream))
    return w, X


def stebz(d: torch.Tensor, e: torch.Tensor, stream=None) -> torch.Tensor:
    """Eigenvalues (ascending) of the symmetric tridiagonal (d, e), no vectors."""
    n = d.shape[0]
    w = torch.empty(n, dtype=F64, device=d.device)
    nw = max(1, lib().evd_stebz_work_size(n))
    work = torch.empty(nw, dtype=F64, device=d.device)
    ep = _ptr(e) if e.numel() > 0 else None
    call("evd_stebz", n, _ptr(d), ep, _ptr(w), _ptr(work), nw, _stream(stream))
    return w


def fp64_peak_tflops(stream=None) -> float:
    """Measured FP64 DMMA peak of this GPU (TFLOP/s)."""
    out = (C.c_double * 1)()
    call("evd_fp64_peak_probe", out, _stream(stream))
    return float(out[0])


def last_timings() -> dict:
    """Stage times (ms) of the last timed syevd call on this thread."""
    out = (C.c_double * 6)()
    lib().evd_syevd_last_timings(out)
    keys = ("sy2sb", "bulge_chasing", "tridiagonal_dc", "bc_back", "sbr_back", "total")
    return {k: float(v) for k, v in zip(keys, out)}
