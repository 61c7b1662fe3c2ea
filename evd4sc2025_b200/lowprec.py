"""FP32 / FP16 entry points of the reference's API (``csrc/lowprec.cu``).

* :func:`tc_syr2k` — ``tc_syr2k`` (api/inc/tc_syr2k.h:6-18): FP32 matrices,
  FP16 products summed in FP32 on the tcgen05 tensor cores;
* :func:`syr2k_lower` — ``tc_ozimmu_syr2k<float>`` (FP32 arithmetic) and
  ``tc_ozimmu_syr2k<half>`` (FP16 data, FP32 accumulation on the tensor cores);
* :func:`panel_qr` / :func:`tsqr` — ``panelQR<float/half>`` and
  ``hou_tsqr_panel<float/half,128,32>``, computed in FP64 and rounded back.

All write the lower triangle of C only (with the diagonal).  Matrices are
column-major CUDA tensors of dtype float32 or float16.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _stream
from ._native import EvdError, call, lib


def _cm(t: torch.Tensor, name: str, dtypes=(torch.float32, torch.float16)):
    if t.dtype not in dtypes:
        raise TypeError(f"{name} must be one of {dtypes}")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    m, n = t.shape
    if m > 1 and t.stride(0) != 1:
        raise ValueError(f"{name} must be column-major")
    ld = t.stride(1) if n > 1 else max(1, m)
    if ld < max(1, m):
        raise ValueError(f"{name} must be column-major")
    return C.c_void_p(t.data_ptr()), ld


def empty_cm(m: int, n: int, dtype, device="cuda") -> torch.Tensor:
    return torch.empty((n, max(m, 1)), dtype=dtype, device=device)[:, :m].t()


def to_cm(t: torch.Tensor, dtype, device="cuda") -> torch.Tensor:
    out = empty_cm(t.shape[0], t.shape[1], dtype, device)
    out.copy_(t.to(device=device, dtype=dtype))
    return out


def tc_syr2k(alpha: float, A: torch.Tensor, B: torch.Tensor, beta: float, Cm: torch.Tensor,
             nb: int = 0, stream=None, hwork=True) -> torch.Tensor:
    """C(lower) = alpha (A B^T + B A^T) + beta C with FP16 products (FP32 data).

    ``hwork``: the reference's FP16 workspace (2 n k halves); True allocates
    it, None lets the library use a stream-ordered buffer."""
    n, k = A.shape
    pa, lda = _cm(A, "A", (torch.float32,))
    pb, ldb = _cm(B, "B", (torch.float32,))
    pc, ldc = _cm(Cm, "C", (torch.float32,))
    if hwork is True:
        hwork = torch.empty(max(1, 2 * n * k), dtype=torch.float16, device=A.device)
    ph = None if hwork is None else C.c_void_p(hwork.data_ptr())
    call("evd_tc_syr2k", n, k, alpha, pa, lda, pb, ldb, beta, pc, ldc, ph, nb, _stream(stream))
    return Cm


def syr2k_lower(alpha: float, A: torch.Tensor, B: torch.Tensor, beta: float, Cm: torch.Tensor,
                nb: int = 0, stream=None) -> torch.Tensor:
    """tc_ozimmu_syr2k<float> (FP32) or <half> (FP16 data, FP32 accumulation),
    chosen by the dtype of the tensors."""
    n, k = A.shape
    if not (A.dtype == B.dtype == Cm.dtype):
        raise TypeError("A, B and C must have one dtype")
    pa, lda = _cm(A, "A")
    pb, ldb = _cm(B, "B")
    pc, ldc = _cm(Cm, "C")
    fn = "evd_syr2k_lower_s" if A.dtype == torch.float32 else "evd_syr2k_lower_h"
    call(fn, n, k, alpha, pa, lda, pb, ldb, beta, pc, ldc, nb, _stream(stream))
    return Cm


def _work(m: int, n: int, device):
    nbytes = int(lib().evd_panel_qr_lp_work_size(m, n))
    if nbytes <= 0:
        raise EvdError("evd_panel_qr_lp_work_size", -1)
    return torch.empty(nbytes, dtype=torch.uint8, device=device), nbytes


def panel_qr(A: torch.Tensor, stream=None):
    """panelQR<float/half>: A (m x 32) <- Y; returns (Y, W, R), Q = I - W Y^T."""
    m, n = A.shape
    pa, lda = _cm(A, "A")
    W = empty_cm(m, n, A.dtype, A.device)
    W.zero_()
    R = empty_cm(n, n, A.dtype, A.device)
    R.zero_()
    pw, ldw = _cm(W, "W")
    pr, ldr = _cm(R, "R")
    w, nbytes = _work(m, n, A.device)
    fn = "evd_panel_qr_s" if A.dtype == torch.float32 else "evd_panel_qr_h"
    call(fn, m, n, pa, lda, pw, ldw, pr, ldr, C.c_void_p(w.data_ptr()), nbytes, _stream(stream))
    return A, W, R


def tsqr(A: torch.Tensor, stream=None):
    """hou_tsqr_panel<float/half,128,32>: A (m x 32) <- explicit Q; returns (Q, R)."""
    m, n = A.shape
    pa, lda = _cm(A, "A")
    R = empty_cm(n, n, A.dtype, A.device)
    R.zero_()
    pr, ldr = _cm(R, "R")
    w, nbytes = _work(m, n, A.device)
    fn = "evd_tsqr_s" if A.dtype == torch.float32 else "evd_tsqr_h"
    call(fn, m, n, pa, lda, pr, ldr, C.c_void_p(w.data_ptr()), nbytes, _stream(stream))
    return A, R
