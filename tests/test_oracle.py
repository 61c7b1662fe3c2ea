"""Oracle (numpy restatement of the reference path) checked against LAPACK.

CPU only.  The reference ships no golden vectors, so the restatement is pinned
here by exact invariants against scipy's LAPACK (dsyevd / dstevd): every stage
is an orthogonal similarity, so spectra must agree to rounding, and every
factor must be orthogonal.  Fixtures produced by the reference's own GPU build
(tests/golden/) pin it further in test_golden.py.
"""
import numpy as np
import pytest

from oracle import algos as O


def test_house_convention():
    x = np.array([3.0, 4.0, 0.0, -12.0])
    u = O.house(x)
    assert abs(u @ u - 2.0) < 1e-15
    y = x - u * (u @ x)
    assert abs(y[0] + np.linalg.norm(x)) < 1e-13 and np.abs(y[1:]).max() < 1e-13
    x2 = -x
    y2 = x2 - O.house(x2) * (O.house(x2) @ x2)
    assert abs(y2[0] - np.linalg.norm(x)) < 1e-13
    assert np.all(O.house(np.zeros(5)) == 0)


@pytest.mark.parametrize("n", [3, 4, 35, 64, 130])
def test_chase_is_similarity(n):
    b = 32
    A = O.sym_gaussian(n, n)
    B = np.tril(np.triu(A, -b), b)
    d, e, U, _ = O.bulge_chase(O.band_pack(B, b), n, b)
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    Q2 = O.q2_apply(np.eye(n), U, n, b, transpose=False)
    assert np.abs(Q2.T @ Q2 - np.eye(n)).max() < 1e-14 * n
    assert np.abs(Q2.T @ B @ Q2 - T).max() < 1e-13 * np.linalg.norm(B, 2)
    assert np.abs(np.linalg.eigvalsh(T) - np.linalg.eigvalsh(B)).max() < 1e-13 * np.linalg.norm(B, 2)
    # forward application is the transpose
    assert np.abs(O.q2_apply(np.eye(n), U, n, b, transpose=True) - Q2.T).max() < 1e-15 * n


@pytest.mark.parametrize("m", [32, 96, 128, 160, 544])
def test_panel_qr_householder_form(m):
    A = np.random.default_rng(m).standard_normal((m, 32))
    Y, W, R = O.panel_qr(A)
    Q = np.eye(m) - W @ Y.T
    assert np.abs(Q.T @ Q - np.eye(m)).max() < 1e-14 * 10
    assert np.abs((Q.T @ A)[:32] - R).max() < 1e-13 * 10
    assert np.allclose(np.triu(Y[:32], 1), 0) and np.allclose(np.diag(Y[:32]), 1)
    Qt, Rt = O.tsqr(A)
    assert np.allclose(R, Rt, atol=1e-13) and np.abs(Qt @ Rt - A).max() < 1e-13


def test_tsqr_rejects_bad_rows():
    with pytest.raises(ValueError):
        O.tsqr(np.ones((200, 32)))  # (200 % 128) % 32 != 0


@pytest.mark.parametrize("n,nb", [(128, 64), (256, 128)])
def test_sy2sb_is_similarity(n, nb):
    A = O.sym_gaussian(n, 3)
    band, W, Y = O.sy2sb(A, 32, nb)
    i, j = np.nonzero(band)
    assert np.abs(i - j).max() <= 32
    Q1 = O.q1_apply(np.eye(n), W, Y, n, 32)
    assert np.abs(Q1.T @ Q1 - np.eye(n)).max() < 1e-13
    assert np.abs(Q1 @ band @ Q1.T - A).max() < 1e-13 * np.linalg.norm(A, 2) * 4


def test_wy_merge_is_product():
    rng = np.random.default_rng(0)
    M, N, b = 50, 24, 8
    W = rng.standard_normal((M, N)) * 0.1
    Y = rng.standard_normal((M, N)) * 0.1
    Qm = O.q_from_wy(O.wy_from_slide(W, Y, b), Y)
    P = np.eye(M)
    for s in range(0, N, b):
        P = P @ (np.eye(M) - W[:, s:s + b] @ Y[:, s:s + b].T)
    assert np.abs(Qm - P).max() < 1e-14


@pytest.mark.parametrize("n,nb", [(256, 128), (512, 256)])
def test_pipeline_vs_dsyevd(n, nb):
    A = O.sym_gaussian(n, 5)
    w, X, _ = O.syevd_two_stage(A, 32, nb)
    assert np.abs(w - np.linalg.eigvalsh(A)).max() < 1e-12 * np.linalg.norm(A, 2)
    assert O.residual(A, w, X) < 1e-15
    assert O.orthogonality(X) < 1e-15


@pytest.mark.parametrize("kind", ["geometric", "uniform", "clustered", "geometric1e10"])
def test_known_spectrum_inputs(kind):
    A, lam = O.known_spectrum_matrix(kind, 200, 1)
    assert np.all(np.diff(lam) >= 0)
    assert np.abs(np.linalg.eigvalsh(A) - lam).max() < 1e-13 * 10


def test_oracle_refinement_converges():
    """The numpy RefSyEv (the oracle of evd_refine_syev): FP32 eigenpairs of a
    Gaussian matrix reach FP64 residual / orthogonality (quadratic decrease)."""
    n = 200
    A = O.sym_gaussian(n, seed=21)
    _, X32 = np.linalg.eigh(A.astype(np.float32))
    X = X32.astype(np.float64)
    w_ref, X_ref = np.linalg.eigh(A)
    errs = []
    for it in (1, 2, 3):
        lam, Xr = O.refine_syev(A, X, it)
        s = np.sign(np.sum(Xr * X_ref, axis=0))
        errs.append(np.abs(Xr * s - X_ref).max())
    # from about 1e-6 (FP32) one iteration reaches 1e-11 or better (quadratic),
    # then the error stays at the FP64 conditioning of the eigenvectors
    assert errs[0] <= 1e-11 and errs[2] <= 1e-12
    assert O.residual(A, lam, Xr) <= 1e-13
    assert O.orthogonality(Xr) <= 1e-13
    assert np.abs(np.sort(lam) - w_ref).max() <= 1e-12 * np.linalg.norm(A, 2)


def test_oracle_refinement_graded_spectrum():
    """Eigenvalues down to 1e-10 ||A||: from a 1e-8-perturbed start the
    noise-floored threshold keeps the iteration monotone (no oscillation of
    the orthogonality)."""
    n = 128
    A, lam = O.known_spectrum_matrix("geometric1e10", n, seed=3)
    _, Xe = np.linalg.eigh(A)
    X0 = Xe + 1e-8 * np.random.default_rng(2).standard_normal((n, n))
    orth = [O.orthogonality(O.refine_syev(A, X0, it)[1]) for it in (1, 2, 3, 4)]
    assert orth[-1] <= 1e-14 and orth[3] <= orth[1] * 10
