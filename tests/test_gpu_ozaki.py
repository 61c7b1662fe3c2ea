"""Emulated FP64 products (Ozaki scheme II on tcgen05 kind::i8) through the C
ABI against the exact-integer oracle (bit for bit) and against FP64 DGEMM."""
import math

import numpy as np
import pytest
import torch

from oracle import ozaki as Z

pytestmark = pytest.mark.gpu


def _op(M, t):
    return M.T if t == "t" else M


@pytest.mark.parametrize("ta,tb", [("n", "n"), ("t", "n"), ("n", "t"), ("t", "t")])
@pytest.mark.parametrize("m,n,k,nmod", [(37, 29, 45, 14), (130, 70, 300, 14), (260, 258, 140, 6),
                                        (65, 300, 513, 9)])
def test_ozaki_matches_oracle_bitwise(cuda, evdlib, ta, tb, m, n, k, nmod):
    rng = np.random.default_rng(m * 1000 + n + k)
    A = rng.standard_normal((k, m) if ta == "t" else (m, k))
    B = rng.standard_normal((n, k) if tb == "t" else (k, n))
    A *= np.exp(2 * rng.standard_normal((A.shape[0], 1)))  # uneven row scales
    ref = Z.gemm(_op(A, ta), _op(B, tb), nmod)
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    Bd = evdlib.to_cm(torch.from_numpy(B), device=cuda)
    Cd = evdlib.empty_cm(m, n, device=cuda)
    evdlib.dgemm_ozaki(ta, tb, 1.0, Ad, Bd, 0.0, Cd, moduli=nmod)
    torch.cuda.synchronize()
    got = Cd.cpu().numpy()
    assert np.array_equal(got, ref), np.abs(got - ref).max()


@pytest.mark.parametrize("n,nmod", [(1024, 14), (2048, 14), (2048, 10), (3000, 14)])
def test_ozaki_accuracy_vs_dgemm(cuda, evdlib, n, nmod):
    g = torch.Generator(device=cuda).manual_seed(n + nmod)
    A = evdlib.to_cm(torch.randn(n, n, generator=g, dtype=torch.float64, device=cuda), cuda)
    B = evdlib.to_cm(torch.randn(n, n, generator=g, dtype=torch.float64, device=cuda), cuda)
    C = evdlib.to_cm(torch.randn(n, n, generator=g, dtype=torch.float64, device=cuda), cuda)
    ref = 0.5 * (A.t() @ B) - 2.0 * C
    D = C.clone(memory_format=torch.contiguous_format).t().contiguous().t()
    evdlib.dgemm_ozaki("t", "n", 0.5, A, B, -2.0, D, moduli=nmod)
    torch.cuda.synchronize()
    P = evdlib.ozaki_bits(nmod, n)
    assert P == Z.bits(nmod, n)
    bound = 0.5 * math.sqrt(n) * 2.0 ** -P * torch.outer(A.norm(dim=0), B.norm(dim=0))
    err = (D - ref).abs()
    # the emulation bound plus the DGEMM reference's own rounding
    assert bool((err <= 2 * bound + 4 * n * 1.2e-16 * (A.abs().t() @ B.abs()) * 0.5).all())


def test_ozaki_k_zero_and_alpha_zero(cuda, evdlib):
    n = 64
    C = evdlib.to_cm(torch.randn(n, n, dtype=torch.float64, device=cuda), cuda)
    A = evdlib.empty_cm(n, 0, device=cuda)
    D = C.clone().t().contiguous().t()
    evdlib.dgemm_ozaki("n", "n", 1.0, A, evdlib.empty_cm(0, n, device=cuda), 3.0, D)
    torch.cuda.synchronize()
    assert torch.equal(D, 3.0 * C)
