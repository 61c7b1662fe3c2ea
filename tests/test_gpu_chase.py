"""Bulge chasing kernel (C ABI) vs the oracle restatement of the reference kernel."""
import numpy as np
import pytest
import torch
from scipy.linalg import eigvalsh_tridiagonal

from oracle import algos as O

pytestmark = pytest.mark.gpu


def _banded(n, b, seed):
    A = O.sym_gaussian(n, seed)
    return np.tril(np.triu(A, -b), b)


@pytest.mark.parametrize("n", [3, 4, 5, 33, 34, 64, 65, 100, 257, 512])
def test_chase_matches_oracle(cuda, evdlib, n):
    b = 32
    B = _banded(n, b, seed=n)
    sub_ref = O.band_pack(B, b)
    d_ref, e_ref, U_ref, _ = O.bulge_chase(sub_ref, n, b)

    Bd = evdlib.to_cm(torch.from_numpy(B), device=cuda)
    sub = evdlib.band_pack(Bd, b)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(sub.cpu().numpy(), sub_ref)  # exact copy kernel

    d, e, U = evdlib.bulge_chase(sub, b)
    torch.cuda.synchronize()
    scale = np.abs(B).max()
    assert np.abs(d.cpu().numpy() - d_ref).max() <= 1e-12 * scale * n
    assert np.abs(e.cpu().numpy() - e_ref).max() <= 1e-12 * scale * n
    assert np.abs(U.cpu().numpy() - U_ref).max() <= 1e-10
    # invariants: same spectrum, reflectors reproduce T
    if n > 1:
        w_t = eigvalsh_tridiagonal(d.cpu().numpy(), e.cpu().numpy())
        w_b = np.linalg.eigvalsh(B)
        assert np.abs(w_t - w_b).max() <= 1e-12 * np.linalg.norm(B, 2) * 8
        Un = U.cpu().numpy()
        Q2 = O.q2_apply(np.eye(n), Un, n, b, transpose=False)
        T = np.diag(d.cpu().numpy()) + np.diag(e.cpu().numpy(), 1) + np.diag(e.cpu().numpy(), -1)
        assert np.abs(Q2.T @ B @ Q2 - T).max() <= 1e-13 * np.linalg.norm(B, 2) * 8


@pytest.mark.parametrize("n", [2048, 4100])
def test_chase_spectrum_large(cuda, evdlib, n):
    b = 32
    B = _banded(n, b, seed=7)
    Bd = evdlib.to_cm(torch.from_numpy(B), device=cuda)
    sub = evdlib.band_pack(Bd, b)
    d, e, U = evdlib.bulge_chase(sub, b)
    torch.cuda.synchronize()
    w_t = eigvalsh_tridiagonal(d.cpu().numpy(), e.cpu().numpy())
    w_b = np.linalg.eigvalsh(B)
    assert np.abs(w_t - w_b).max() <= 1e-12 * np.linalg.norm(B, 2) * 8
    # reflector norms: ||u||^2 = 2 for every stored reflector segment
    Un = U.cpu().numpy()
    seg = Un[1:33, 0]
    assert abs(seg @ seg - 2.0) < 1e-12


def test_chase_repeatable(cuda, evdlib):
    """Two calls in one process give identical results (the reference's
    g_overFlag made a second call return immediately)."""
    n, b = 300, 32
    B = _banded(n, b, seed=3)
    Bd = evdlib.to_cm(torch.from_numpy(B), device=cuda)
    out = []
    for _ in range(2):
        sub = evdlib.band_pack(Bd, b)
        d, e, U = evdlib.bulge_chase(sub, b)
        out.append((d.clone(), e.clone(), U.clone()))
    torch.cuda.synchronize()
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][2], out[1][2])
