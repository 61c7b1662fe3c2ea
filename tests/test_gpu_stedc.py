"""Device tridiagonal divide and conquer (C ABI) vs LAPACK dstevd (scipy)."""
import numpy as np
import pytest
import torch

from oracle import algos as O

pytestmark = pytest.mark.gpu


def _check(cuda, evdlib, d, e, tol_val=1e-13, tol_vec=1e-13):
    n = d.shape[0]
    w_ref = O.tridiag_eig(d, e)[0] if n > 1 else d.copy()
    w, Z = evdlib.stedc(torch.from_numpy(d).to(cuda), torch.from_numpy(e).to(cuda))
    torch.cuda.synchronize()
    w, Z = w.cpu().numpy(), Z.cpu().numpy()
    T = np.diag(d) + (np.diag(e, 1) + np.diag(e, -1) if n > 1 else 0)
    nrm = max(np.abs(w_ref).max(), 1e-300)
    assert np.all(np.diff(w) >= 0)
    assert np.abs(w - w_ref).max() <= tol_val * nrm * max(1.0, np.sqrt(n))
    assert np.linalg.norm(T @ Z - Z * w) / (n * max(np.linalg.norm(T), 1e-300)) <= tol_vec
    assert np.linalg.norm(Z.T @ Z - np.eye(n)) / n <= tol_vec
    return w, Z


@pytest.mark.parametrize("n", [1, 2, 3, 5, 31, 32, 33, 64, 65, 100, 257, 1000, 2048, 4097])
def test_stedc_random(cuda, evdlib, n):
    rng = np.random.default_rng(n)
    _check(cuda, evdlib, rng.standard_normal(n), rng.standard_normal(max(n - 1, 0)))


def test_stedc_from_chase(cuda, evdlib):
    n = 600
    A = O.sym_gaussian(n, 4)
    B = np.tril(np.triu(A, -32), 32)
    d, e, _, _ = O.bulge_chase(O.band_pack(B, 32), n, 32)
    _check(cuda, evdlib, d, e)


def test_stedc_zero_offdiag_blocks(cuda, evdlib):
    # decoupled blocks and exact zeros force deflation paths
    n = 500
    rng = np.random.default_rng(7)
    d = rng.standard_normal(n)
    e = rng.standard_normal(n - 1)
    e[::37] = 0.0
    _check(cuda, evdlib, d, e)


def test_stedc_repeated_eigenvalues(cuda, evdlib):
    # identity plus tiny coupling: heavy deflation with Givens rotations
    n = 700
    d = np.ones(n)
    e = np.full(n - 1, 1e-20)
    _check(cuda, evdlib, d, e)
    # Wilkinson-like matrix with close eigenvalue pairs
    m = 201
    d = np.abs(np.arange(m) - m // 2).astype(float)
    e = np.ones(m - 1)
    _check(cuda, evdlib, d, e)


def test_stedc_clustered_spectrum(cuda, evdlib):
    n = 1024
    lam = O.spectrum("clustered", n, 3)
    Q = O.haar_orthogonal(n, 3)
    A = (Q * lam) @ Q.T
    A = 0.5 * (A + A.T)
    from scipy.linalg import hessenberg
    # tridiagonal with the clustered spectrum (Householder tridiagonalisation)
    H = hessenberg(A)
    d = np.diag(H).copy()
    e = np.diag(H, -1).copy()
    _check(cuda, evdlib, d, e)


def test_stedc_rejects_nan(cuda, evdlib):
    d = np.ones(100)
    e = np.ones(99)
    e[40] = np.nan
    with pytest.raises(evdlib.EvdError):
        evdlib.stedc(torch.from_numpy(d).to(cuda), torch.from_numpy(e).to(cuda))


def test_stedc_scaling(cuda, evdlib):
    rng = np.random.default_rng(11)
    for s in (1e-150, 1e150):
        _check(cuda, evdlib, s * rng.standard_normal(300), s * rng.standard_normal(299))
