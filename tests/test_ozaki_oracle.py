"""The emulated-FP64 product's oracle (oracle/ozaki.py) on the CPU: moduli,
CRT reconstruction and the accuracy of the definition against exact
rational products."""
import math
from fractions import Fraction

import numpy as np
import pytest

from oracle import ozaki as Z


def test_moduli_pairwise_coprime():
    for i, p in enumerate(Z.MODULI):
        assert p <= 256
        for q in Z.MODULI[i + 1:]:
            assert math.gcd(p, q) == 1


@pytest.mark.parametrize("nmod", [4, 8, 14, 16])
def test_crt_round_trip(nmod):
    rng = np.random.default_rng(nmod)
    M = Z.modulus_product(nmod)
    for _ in range(200):
        x = int(rng.integers(-(1 << 62), 1 << 62)) * int(rng.integers(1, 1 << 40))
        x %= M
        x = x - M if x > M // 2 else x
        res = [x % p for p in Z.MODULI[:nmod]]
        assert Z.crt(res, nmod) == x


@pytest.mark.parametrize("nmod,k", [(14, 1000), (14, 16384), (8, 4096), (4, 64)])
def test_bits_keep_products_in_range(nmod, k):
    P = Z.bits(nmod, k)
    assert P >= 4 * nmod - 4 or P == 53
    M = Z.modulus_product(nmod)
    assert (2 ** P + math.sqrt(k) / 2) ** 2 < M / 2


def test_fourteen_moduli_are_fp64_level():
    assert Z.bits(14, 16384) == 53
    assert Z.bits(14, 65536) == 53


@pytest.mark.parametrize("nmod", [8, 14])
def test_emulated_product_error_bound(nmod):
    rng = np.random.default_rng(5)
    m, k, n = 12, 40, 9
    A = rng.standard_normal((m, k)) * np.exp(rng.standard_normal((m, 1)))
    B = rng.standard_normal((k, n))
    D = Z.gemm(A, B, nmod)
    P = Z.bits(nmod, k)
    for i in range(m):
        for j in range(n):
            exact = sum(Fraction(float(A[i, t])) * Fraction(float(B[t, j])) for t in range(k))
            bound = math.sqrt(k) * 2.0 ** (-P) * np.linalg.norm(A[i]) * np.linalg.norm(B[:, j])
            assert abs(float(Fraction(float(D[i, j])) - exact)) <= bound + 1e-300
