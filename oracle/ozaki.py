"""Exact-integer restatement of the emulated FP64 product (test oracle).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker; never by the
product.

The library's emulated product (Ozaki scheme II: Ozaki, Uchino, Imamura,
"Ozaki Scheme II: A GEMM-oriented emulation of floating-point matrix
multiplication using an integer modular technique", 2025) has no counterpart
in the reference, whose products are cuBLAS DGEMMs (api/TCblas/
tc_ozimmu_syr2k.cu:54-192).  What the product must return is fixed by its
definition, so this module computes it directly with Python integers instead
of residues:

  a_i = rint(2^e_i op(A)_i),  e_i = P - E_i,  ||op(A)_i||_2 < 2^E_i  (frexp)
  b_j = rint(2^f_j op(B)_j),  likewise for the columns of op(B)
  D_ij = alpha * 2^-(e_i + f_j) * (a_i . b_j)        (a_i . b_j exact)

The GPU forms a_i . b_j modulo each p_l and rebuilds it by the Chinese
remainder theorem; when |a_i . b_j| < Mod/2 (which the choice of P
guarantees) the two agree exactly, and the conversion of the integer to a
double is the same (40-bit limbs summed from the top down), so the results are
bit-for-bit equal.
"""
from __future__ import annotations

import math

import numpy as np

MODULI = (256, 255, 253, 251, 247, 241, 239, 233,
          229, 227, 223, 217, 211, 199, 197, 193)


def modulus_product(nmod: int) -> int:
    m = 1
    for p in MODULI[:nmod]:
        m *= p
    return m


def bits(nmod: int, k: int) -> int:
    """Largest P (<= 53) with (2^P + sqrt(k)/2)^2 < Mod/2."""
    M = modulus_product(nmod)
    lim = math.sqrt(M / 2.0) * (1.0 - 1e-12) - math.sqrt(k) / 2.0
    return min(int(math.floor(math.log2(lim))), 53)


def quantize_rows(S: np.ndarray, P: int):
    """Rows of S (a 2-D float64 array) -> (exponents, integer rows as int64)."""
    e = np.zeros(S.shape[0], dtype=np.int64)
    Q = np.zeros(S.shape, dtype=np.int64)
    for i in range(S.shape[0]):
        nrm = math.sqrt(float(np.dot(S[i], S[i])))
        if nrm > 0.0:
            _, E = math.frexp(nrm)
            e[i] = P - E
        Q[i] = np.rint(np.ldexp(S[i], int(e[i]))).astype(np.int64)
    return e, Q


def _to_double(x: int) -> float:
    """The device's conversion of the rebuilt integer: the magnitude's 40-bit
    limbs y3..y0 summed as y3 2^120 + (y2 2^80 + (y1 2^40 + y0)), one rounding
    per addition (the products by powers of two are exact)."""
    neg = x < 0
    x = -x if neg else x
    m = (1 << 40) - 1
    y0, y1, y2, y3 = x & m, (x >> 40) & m, (x >> 80) & m, x >> 120
    v = float(y3) * 2.0 ** 120 + (float(y2) * 2.0 ** 80 + (float(y1) * 2.0 ** 40 + float(y0)))
    return -v if neg else v


def gemm(opA: np.ndarray, opB: np.ndarray, nmod: int, alpha: float = 1.0) -> np.ndarray:
    """alpha * opA @ opB (opA m x k, opB k x n) as the emulated product returns it."""
    m, k = opA.shape
    P = bits(nmod, k)
    ea, qa = quantize_rows(np.asarray(opA, dtype=np.float64), P)
    eb, qb = quantize_rows(np.asarray(opB, dtype=np.float64).T, P)
    prod = qa.astype(object) @ qb.astype(object).T  # exact Python integers
    half = modulus_product(nmod) // 2
    out = np.empty((m, opB.shape[1]), dtype=np.float64)
    for i in range(m):
        for j in range(opB.shape[1]):
            x = int(prod[i, j])
            assert abs(x) < half, "CRT range exceeded"
            out[i, j] = alpha * math.ldexp(_to_double(x), -int(ea[i] + eb[j]))
    return out


def crt(residues: list[int], nmod: int) -> int:
    """The integer in (-Mod/2, Mod/2] with the given residues (for host checks
    of the moduli table)."""
    M = modulus_product(nmod)
    x = 0
    for r, p in zip(residues, MODULI[:nmod]):
        Mi = M // p
        x += r * Mi * pow(Mi, -1, p)
    x %= M
    return x - M if x > M // 2 else x
