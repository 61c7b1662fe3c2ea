"""Whole plain-FP64 pipeline (evd_syevd) vs LAPACK dsyevd and the oracle pipeline."""
import numpy as np
import pytest
import torch

from oracle import algos as O

pytestmark = pytest.mark.gpu

# accuracy bars: eigenvalues to 1e-12 relative to ||A||, residual and
# orthogonality below 1e-13 (normalised by n, as the reference's checkMetric)
TOL_VAL = 1e-12
TOL_RES = 1e-13
TOL_ORT = 1e-13


def _run(cuda, evdlib, A, nb):
    n = A.shape[0]
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    w, X = evdlib.syevd(Ad, 32, nb)
    res, orth = evdlib.check_eig(Ad, w, X)
    torch.cuda.synchronize()
    return w.cpu().numpy(), X.cpu().numpy(), res, orth


@pytest.mark.parametrize("n,nb", [(64, 32), (256, 64), (1024, 256), (1024, 1024), (2048, 1024),
                                  (4096, 1024)])
def test_syevd_gaussian(cuda, evdlib, n, nb):
    A = O.sym_gaussian(n, seed=2024 + n)
    w, X, res, orth = _run(cuda, evdlib, A, nb)
    w_ref = np.linalg.eigvalsh(A)
    nA = np.linalg.norm(A, 2)
    assert np.abs(w - w_ref).max() <= TOL_VAL * nA
    assert res <= TOL_RES and orth <= TOL_ORT
    # CPU-side residual for an independent check
    assert O.residual(A, w, X) <= TOL_RES


def test_syevd_matches_oracle_pipeline(cuda, evdlib):
    n, nb = 512, 256
    A = O.sym_gaussian(n, seed=77)
    w, X, res, orth = _run(cuda, evdlib, A, nb)
    w_o, X_o, _ = O.syevd_two_stage(A, 32, nb)
    assert np.abs(w - w_o).max() <= TOL_VAL * np.linalg.norm(A, 2)
    # eigenvectors agree up to sign (simple spectrum)
    s = np.sign(np.sum(X * X_o, axis=0))
    assert np.abs(X - X_o * s).max() <= 1e-9


@pytest.mark.parametrize("kind", ["geometric", "uniform", "clustered", "geometric1e10"])
def test_syevd_known_spectrum(cuda, evdlib, kind):
    n, nb = 1024, 256
    A, lam = O.known_spectrum_matrix(kind, n, seed=5)
    w, X, res, orth = _run(cuda, evdlib, A, nb)
    # lambda is known up to the error of forming A (~sqrt(n) eps ||A||)
    assert np.abs(w - lam).max() <= 1e-12 * np.abs(lam).max() * 4
    assert res <= TOL_RES and orth <= TOL_ORT


def test_syevd_repeatable_and_timed(cuda, evdlib):
    n = 1024
    A = evdlib.to_cm(torch.from_numpy(O.sym_gaussian(n, 1)), device=cuda)
    ws = evdlib.Workspace(n, 32, 256, device=cuda)
    w1, X1 = evdlib.syevd(A, 32, 256, ws=ws, timed=True)
    t = evdlib.last_timings()
    w2, X2 = evdlib.syevd(A, 32, 256, ws=ws)
    torch.cuda.synchronize()
    assert torch.equal(w1, w2) and torch.equal(X1, X2)  # deterministic
    assert t["total"] > 0 and all(v >= 0 for v in t.values())


@pytest.mark.parametrize("kind", ["diagonal", "block_diagonal", "tridiagonal"])
def test_structured_inputs(cuda, evdlib, kind):
    """Inputs whose panels are (partly) zero below the band: the panel
    factorisation must not break down (zero columns get the reflector
    sqrt(2) e_j)."""
    n = 256
    rng = np.random.default_rng(5)
    if kind == "diagonal":
        A = np.diag(rng.standard_normal(n))
    elif kind == "block_diagonal":
        A = np.zeros((n, n))
        G = rng.standard_normal((100, 100))
        A[:100, :100] = 0.5 * (G + G.T)
        A[100:, 100:] = np.diag(np.linspace(3.0, 4.0, n - 100))
    else:
        d, e = rng.standard_normal(n), rng.standard_normal(n - 1)
        A = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    w, X = evdlib.syevd(Ad, 32, 64)
    res, orth = evdlib.check_eig(Ad, w, X)
    torch.cuda.synchronize()
    w_ref = np.linalg.eigvalsh(A)
    assert np.abs(w.cpu().numpy() - w_ref).max() <= 1e-12 * np.abs(A).max() * 8
    assert res <= 1e-13 and orth <= 1e-13, (res, orth)


@pytest.mark.parametrize("n,nb", [(1000, 256), (300, 128), (1, 64), (20, 32), (32, 32),
                                  (33, 32), (77, 64), (1500, 1024)])
def test_syevd_any_order(cuda, evdlib, n, nb):
    """n not a multiple of nb: padded internally with a decoupled diagonal
    block above the spectrum; results must meet the same bars as n % nb == 0."""
    A = O.sym_gaussian(n, seed=3 * n + 1)
    w, X, res, orth = _run(cuda, evdlib, A, nb)
    assert w.shape == (n,) and X.shape == (n, n)
    w_ref = np.linalg.eigvalsh(A)
    nA = max(np.linalg.norm(A, 2), 1e-300)
    assert np.abs(w - w_ref).max() <= TOL_VAL * nA
    assert res <= TOL_RES and orth <= TOL_ORT, (res, orth)
    assert O.residual(A, w, X) <= TOL_RES


def test_syevd_any_order_zero_and_strided(cuda, evdlib):
    """A zero matrix (pad values fall back to 2 .. 3) and a strided A/X
    (lda, ldX > n) in the padded path; A is not modified."""
    n, nb = 200, 64
    Zd = evdlib.to_cm(torch.zeros(n, n, dtype=torch.float64), device=cuda)
    w, X = evdlib.syevd(Zd, 32, nb)
    torch.cuda.synchronize()
    Xh = X.cpu().numpy()
    assert np.all(w.cpu().numpy() == 0.0)
    assert np.linalg.norm(Xh.T @ Xh - np.eye(n)) / n <= TOL_ORT
    A = O.sym_gaussian(n, seed=9)
    big = evdlib.to_cm(torch.zeros(n + 7, n + 7, dtype=torch.float64), device=cuda)
    big[:n, :n].copy_(torch.from_numpy(A))
    Ad = big[:n, :n]
    Xbig = evdlib.to_cm(torch.zeros(n + 5, n + 5, dtype=torch.float64), device=cuda)
    Xd = Xbig[:n, :n]
    before = Ad.clone()
    w, X = evdlib.syevd(Ad, 32, nb, X=Xd)
    torch.cuda.synchronize()
    assert torch.equal(Ad, before)
    assert np.abs(w.cpu().numpy() - np.linalg.eigvalsh(A)).max() <= TOL_VAL * np.linalg.norm(A, 2)
    assert O.residual(A, w.cpu().numpy(), Xd.cpu().numpy()) <= TOL_RES
    assert float(Xbig[n:, :].abs().max()) == 0.0  # rows past n of X untouched


@pytest.mark.parametrize("bad", [float("nan"), float("inf")])
def test_non_finite_input_is_an_error(cuda, evdlib, bad):
    """A non-finite entry makes the solve fail with a status (the tridiagonal
    solver rejects non-finite input) instead of returning garbage; the
    context stays usable for the next solve."""
    n = 256
    A = O.sym_gaussian(n, seed=12)
    A[10, 3] = A[3, 10] = bad
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    with pytest.raises(evdlib.EvdError) as e:
        evdlib.syevd(Ad, 32, 64)
    assert e.value.status < 0
    w, X, res, orth = _run(cuda, evdlib, O.sym_gaussian(n, seed=13), 64)
    assert res <= TOL_RES and orth <= TOL_ORT
