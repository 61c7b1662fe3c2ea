"""Matrix and eigenpair files (binary records and the reference's CSV layout).

The reference writes matrices only as CSV, element by element
(writeMatrixToCsvV2, util/inc/fileOpTool.h:51-80) and reads them back with
readMatrixFromFile + fillMatrix (util/tool/fileOpTool.cu:127-174).  This
module wraps the library's file entry points (``evd_*_bin``, ``evd_*_csv``):

* binary: a sequence of records, each a 32-byte header
  ``{"EVDM", u32 1, u32 8, u32 0, i64 rows, i64 cols}`` followed by the FP64
  values column-major; an eigenpair file is two records, w (n x 1), X (n x n);
* CSV: one matrix row per line, comma separated, ``%.17g`` (round-trips FP64).

Tensors may live on the host or on a CUDA device; matrices are FP64 and are
read back column-major.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

from ._native import EvdError, call, lib

F64 = torch.float64


def _path(path) -> bytes:
    return os.fsencode(path)


def _cm_any(t: torch.Tensor, name: str):
    """(pointer, leading dimension, keep-alive tensor) of a column-major FP64
    matrix on the host or a device; other layouts are copied column-major."""
    if t.dtype != F64:
        raise TypeError(f"{name} must be float64")
    if t.dim() == 1:
        t = t.contiguous()
        return C.c_void_p(t.data_ptr()), max(1, t.shape[0]), t
    if t.dim() != 2:
        raise ValueError(f"{name} must be a matrix")
    m, n = t.shape
    if not (t.stride(0) == 1 and (n <= 1 or t.stride(1) >= max(1, m))):
        t = t.t().contiguous().t()
    ld = t.stride(1) if n > 1 else max(1, m)
    return C.c_void_p(t.data_ptr()), ld, t


def _empty_cm(m: int, n: int, device) -> torch.Tensor:
    return torch.empty((n, max(m, 1)), dtype=F64, device=device)[:, :m].t()


def save_matrix(path, A: torch.Tensor, append: bool = False) -> None:
    """Write A (m x n, or a vector as n x 1) as one binary record."""
    p, ld, keep = _cm_any(A, "A")
    m = A.shape[0]
    n = A.shape[1] if A.dim() == 2 else 1
    call("evd_write_matrix_bin", _path(path), 1 if append else 0, m, n, p, ld)
    del keep


def count_matrices(path) -> int:
    r = int(lib().evd_matrix_bin_count(_path(path)))
    if r < 0:
        raise EvdError("evd_matrix_bin_count", r)
    return r


def matrix_shape(path, index: int = 0) -> tuple[int, int]:
    rows, cols = C.c_long(0), C.c_long(0)
    call("evd_matrix_bin_shape", _path(path), index, C.byref(rows), C.byref(cols))
    return rows.value, cols.value


def load_matrix(path, index: int = 0, device="cpu") -> torch.Tensor:
    """Record ``index`` of a binary file as a column-major FP64 matrix."""
    m, n = matrix_shape(path, index)
    out = _empty_cm(m, n, device)
    call("evd_read_matrix_bin", _path(path), index, m, n, C.c_void_p(out.data_ptr()), max(m, 1))
    return out


def save_eigenpairs(path, w: torch.Tensor, X: torch.Tensor) -> None:
    """Write eigenvalues w (n) and eigenvectors X (n x n) as one file."""
    n = w.shape[0]
    if X.shape != (n, n):
        raise ValueError("X must be n x n")
    pw, _, kw = _cm_any(w, "w")
    px, ldx, kx = _cm_any(X, "X")
    call("evd_write_eigenpairs_bin", _path(path), n, pw, px, ldx)
    del kw, kx


def load_eigenpairs(path, device="cpu") -> tuple[torch.Tensor, torch.Tensor]:
    n, one = matrix_shape(path, 0)
    if one != 1:
        raise EvdError("evd_read_eigenpairs_bin", -6)
    w = torch.empty(n, dtype=F64, device=device)
    X = _empty_cm(n, n, device)
    call("evd_read_eigenpairs_bin", _path(path), n, C.c_void_p(w.data_ptr()),
         C.c_void_p(X.data_ptr()), max(n, 1))
    return w, X


def save_csv(path, A: torch.Tensor) -> None:
    """CSV in the reference's layout (row per line)."""
    p, ld, keep = _cm_any(A, "A")
    m = A.shape[0]
    n = A.shape[1] if A.dim() == 2 else 1
    call("evd_write_matrix_csv", _path(path), m, n, p, ld)
    del keep


def load_csv(path, device="cpu") -> torch.Tensor:
    rows, cols = C.c_long(0), C.c_long(0)
    call("evd_read_matrix_csv", _path(path), C.byref(rows), C.byref(cols), None, 1)
    out = _empty_cm(rows.value, cols.value, device)
    call("evd_read_matrix_csv", _path(path), C.byref(rows), C.byref(cols),
         C.c_void_p(out.data_ptr()), max(rows.value, 1))
    return out
