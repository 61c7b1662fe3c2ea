"""Eigenvalues-only path: the tridiagonal multisection solver against LAPACK
(scipy eigvalsh_tridiagonal), the chase without stored reflectors against the
chase with them, and the whole values-only solve against numpy eigvalsh."""
import numpy as np
import pytest
import torch
from scipy.linalg import eigvalsh_tridiagonal

from oracle import algos as O

pytestmark = pytest.mark.gpu


def _tri(kind, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "random":
        return rng.standard_normal(n), rng.standard_normal(max(n - 1, 0))
    if kind == "wilkinson":  # pairs of nearly equal eigenvalues
        m = (n - 1) / 2.0
        return np.abs(np.arange(n) - m), np.ones(max(n - 1, 0))
    if kind == "clustered":  # tiny off-diagonals: clusters and near-decoupled blocks
        d = np.repeat(rng.standard_normal(n // 16 + 1), 16)[:n]
        return d, 1e-12 * rng.standard_normal(max(n - 1, 0))
    if kind == "graded":
        return np.logspace(0, -14, n), np.logspace(-1, -15, max(n - 1, 0))
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["random", "wilkinson", "clustered", "graded"])
@pytest.mark.parametrize("n", [1, 2, 3, 17, 100, 1000, 5000])
def test_stebz_matches_lapack(cuda, evdlib, kind, n):
    d, e = _tri(kind, n, n)
    w = evdlib.stebz(torch.from_numpy(d).to(cuda), torch.from_numpy(e).to(cuda))
    torch.cuda.synchronize()
    ref = eigvalsh_tridiagonal(d, e) if n > 1 else d.copy()
    nrm = max(np.abs(d).max(), np.abs(e).max() if n > 1 else 0.0, 1e-300)
    assert np.abs(w.cpu().numpy() - ref).max() <= 1e-13 * nrm * max(1.0, np.log2(n))


def test_chase_without_reflectors_matches(cuda, evdlib):
    n, b = 700, 32
    A = O.sym_gaussian(n, 21)
    B = np.tril(np.triu(A, -b), b)
    Bd = evdlib.to_cm(torch.from_numpy(B), device=cuda)
    d1, e1, _ = evdlib.bulge_chase(evdlib.band_pack(Bd, b), b)
    sub = evdlib.band_pack(Bd, b)
    d2 = torch.empty(n, dtype=torch.float64, device=cuda)
    e2 = torch.empty(n, dtype=torch.float64, device=cuda)
    iw = torch.zeros(evdlib.lib().evd_bulge_chase_iwork_size(n) // 4 + 1, dtype=torch.int32,
                     device=cuda)
    import ctypes as C
    rc = evdlib.lib().evd_bulge_chase(n, b, C.c_void_p(sub.data_ptr()), 2 * b, None, n,
                                      C.c_void_p(d2.data_ptr()), C.c_void_p(e2.data_ptr()),
                                      C.c_void_p(iw.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert torch.equal(d1, d2) and torch.equal(e1[: n - 1], e2[: n - 1])


@pytest.mark.parametrize("n,nb", [(64, 32), (256, 64), (1024, 256), (2048, 1024)])
def test_values_only_solve(cuda, evdlib, n, nb):
    A = O.sym_gaussian(n, n + 3)
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    w = evdlib.syevd_values(Ad, 32, nb, timed=True)
    torch.cuda.synchronize()
    ref = np.linalg.eigvalsh(A)
    assert np.abs(w.cpu().numpy() - ref).max() <= 1e-12 * np.linalg.norm(A, 2)
    t = evdlib.last_timings()
    assert t["total"] > 0


@pytest.mark.parametrize("kind", ["geometric1e10", "clustered"])
def test_values_only_known_spectrum(cuda, evdlib, kind):
    n = 1024
    A, lam = O.known_spectrum_matrix(kind, n, seed=6)
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    w = evdlib.syevd_values(Ad, 32, 256)
    torch.cuda.synchronize()
    assert np.abs(w.cpu().numpy() - np.sort(lam)).max() <= 1e-12 * np.abs(lam).max() * 8


@pytest.mark.parametrize("n,nb", [(1000, 256), (77, 64), (1, 64)])
def test_values_only_any_order(cuda, evdlib, n, nb):
    A = O.sym_gaussian(n, n + 11)
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    w = evdlib.syevd_values(Ad, 32, nb)
    torch.cuda.synchronize()
    assert w.shape == (n,)
    ref = np.linalg.eigvalsh(A)
    assert np.abs(w.cpu().numpy() - ref).max() <= 1e-12 * max(np.linalg.norm(A, 2), 1e-300)
