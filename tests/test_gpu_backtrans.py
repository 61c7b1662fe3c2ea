"""Back transformations (C ABI) vs the oracle: chasing reflectors (BC back), slab WY
(SBR back), computerWYFromSlide and computerQFromWY."""
import numpy as np
import pytest
import torch

from oracle import algos as O

pytestmark = pytest.mark.gpu


def _chase_U(n, seed):
    b = 32
    A = O.sym_gaussian(n, seed)
    B = np.tril(np.triu(A, -b), b)
    d, e, U, _ = O.bulge_chase(O.band_pack(B, b), n, b)
    return U


@pytest.mark.parametrize("n,ncols", [(3, 3), (4, 7), (33, 33), (100, 1), (257, 64), (300, 300),
                                     (517, 133), (1024, 40)])
@pytest.mark.parametrize("forward", [True, False])
def test_q2_apply_matches_oracle(cuda, evdlib, n, ncols, forward):
    U = _chase_U(n, seed=n)
    X = np.random.default_rng(ncols).standard_normal((n, ncols))
    ref = O.q2_apply(X, U, n, 32, transpose=forward)
    Xd = evdlib.to_cm(torch.from_numpy(X), device=cuda)
    Ud = evdlib.to_cm(torch.from_numpy(U), device=cuda)
    if forward:
        evdlib.bc_back(Xd, Ud) if ncols == n else _fwd(evdlib, Xd, Ud)
    else:
        evdlib.bc_back_apply(Xd, Ud)
    torch.cuda.synchronize()
    assert np.abs(Xd.cpu().numpy() - ref).max() <= 1e-12 * max(1.0, np.sqrt(n))


@pytest.mark.parametrize("n,ncols", [(5, 3), (257, 64), (517, 133), (1100, 300)])
def test_q2_apply_without_workspace(cuda, evdlib, n, ncols):
    """X <- Q2 X with the T factors rebuilt inside the kernel (work = NULL)
    agrees with the precomputed-T path and with the oracle."""
    U = _chase_U(n, seed=n + 1)
    X = np.random.default_rng(ncols).standard_normal((n, ncols))
    ref = O.q2_apply(X, U, n, 32, transpose=False)
    Ud = evdlib.to_cm(torch.from_numpy(U), device=cuda)
    X1 = evdlib.to_cm(torch.from_numpy(X), device=cuda)
    X2 = evdlib.to_cm(torch.from_numpy(X), device=cuda)
    evdlib.bc_back_apply(X1, Ud, work=None)
    evdlib.bc_back_apply(X2, Ud, work=True)
    torch.cuda.synchronize()
    a, b = X1.cpu().numpy(), X2.cpu().numpy()
    assert np.abs(a - ref).max() <= 1e-12 * max(1.0, np.sqrt(n))
    assert np.abs(a - b).max() <= 1e-13 * max(1.0, np.sqrt(n))


def test_q2_apply_rejects_small_workspace(cuda, evdlib):
    import ctypes as C
    n = 300
    U = evdlib.zeros_cm(n, n, device=cuda)
    X = evdlib.zeros_cm(n, 4, device=cuda)
    need = evdlib.lib().evd_bc_back_work_size(n)
    w = torch.empty(need, dtype=torch.float64, device=cuda)
    rc = evdlib.lib().evd_bc_back_apply(n, 4, C.c_void_p(U.data_ptr()), n, C.c_void_p(X.data_ptr()),
                                        n, 32, C.c_void_p(w.data_ptr()), need - 1, None)
    assert rc == -5  # EVD_ERR_WORKSPACE


def _fwd(evdlib, Xd, Ud):
    """Q2^T X for any column count through the square reference entry point:
    process X in chunks of at most n columns padded into an n x n block."""
    n, k = Xd.shape
    for c0 in range(0, k, n):
        c1 = min(k, c0 + n)
        P = evdlib.zeros_cm(n, n, device=Xd.device)
        P[:, : c1 - c0] = Xd[:, c0:c1]
        evdlib.bc_back(P, Ud)
        Xd[:, c0:c1] = P[:, : c1 - c0]


def test_bc_back_reference_semantics(cuda, evdlib):
    """Q <- Q2^T Q with Q = I gives Q2^T; Q2^T B Q2 is the tridiagonal."""
    n, b = 200, 32
    A = O.sym_gaussian(n, 9)
    B = np.tril(np.triu(A, -b), b)
    d, e, U, _ = O.bulge_chase(O.band_pack(B, b), n, b)
    Q = evdlib.to_cm(torch.eye(n, dtype=torch.float64), device=cuda)
    evdlib.bc_back(Q, evdlib.to_cm(torch.from_numpy(U), device=cuda))
    torch.cuda.synchronize()
    Q2t = Q.cpu().numpy()
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    assert np.abs(Q2t @ B @ Q2t.T - T).max() <= 1e-12 * np.linalg.norm(B, 2) * 8


@pytest.mark.parametrize("n,nb,nk", [(256, 64, 64), (512, 128, 128), (1024, 256, 256),
                                     (1024, 1024, 1024), (2048, 1024, 1024)])
def test_sbr_back_matches_oracle(cuda, evdlib, n, nb, nk):
    A = O.sym_gaussian(n, seed=3)
    band, W, Y = evdlib.sy2sb(evdlib.to_cm(torch.from_numpy(A), device=cuda), 32, nb)
    Wn, Yn = W.cpu().numpy(), Y.cpu().numpy()
    X = np.random.default_rng(5).standard_normal((n, 50))
    ref = O.q1_apply(X, Wn, Yn, n, 32)
    Xd = evdlib.to_cm(torch.from_numpy(X), device=cuda)
    evdlib.sbr_back(Xd, W, Y, 32, nk)
    torch.cuda.synchronize()
    assert np.abs(Xd.cpu().numpy() - ref).max() <= 1e-11


@pytest.mark.parametrize("M,N,b", [(64, 64, 32), (300, 128, 32), (1000, 256, 64), (513, 96, 32)])
def test_wy_from_slide_and_q_from_wy(cuda, evdlib, M, N, b):
    # the merge identity (I - W1 Y1^T)(I - W2 Y2^T) = I - [W1, W2 - W1 Y1^T W2][Y1, Y2]^T
    # holds for any slides; small random entries keep the product well scaled
    rng = np.random.default_rng(M)
    W = rng.standard_normal((M, N)) / np.sqrt(M * N)
    Y = rng.standard_normal((M, N)) / np.sqrt(M)
    Wm_ref = O.wy_from_slide(W, Y, b)
    Wd = evdlib.to_cm(torch.from_numpy(W), device=cuda)
    Yd = evdlib.to_cm(torch.from_numpy(Y), device=cuda)
    evdlib.wy_from_slide(Wd, Yd, b)
    torch.cuda.synchronize()
    assert np.abs(Wd.cpu().numpy() - Wm_ref).max() <= 1e-14 * max(1, N)
    Q = evdlib.q_from_wy(Wd, Yd)
    torch.cuda.synchronize()
    Qr = O.q_from_wy(Wm_ref, Y)
    assert np.abs(Q.cpu().numpy() - Qr).max() <= 1e-14 * max(1, N)
    P = np.eye(M)
    for s in range(0, N, b):
        P = P @ (np.eye(M) - W[:, s:s + b] @ Y[:, s:s + b].T)
    assert np.abs(Q.cpu().numpy() - P).max() <= 1e-13


def test_check_orthogonality(cuda, evdlib):
    Q, _ = np.linalg.qr(np.random.default_rng(1).standard_normal((300, 300)))
    Qd = evdlib.to_cm(torch.from_numpy(Q), device=cuda)
    v = evdlib.check_orthogonality(Qd)
    assert abs(v - O.orthogonality(Q)) <= 1e-15 + 1e-3 * O.orthogonality(Q)
    Qp = Q.copy()
    Qp[:, 0] *= 1.001
    v2 = evdlib.check_orthogonality(evdlib.to_cm(torch.from_numpy(Qp), device=cuda))
    assert abs(v2 - O.orthogonality(Qp)) <= 1e-6 * O.orthogonality(Qp)
