"""TSQR / panel QR kernels (C ABI) vs the oracle restatement of panelQR/hou_tsqr_panel."""
import numpy as np
import pytest
import torch

from oracle import algos as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m", [32, 64, 96, 128, 160, 256, 544, 1024, 4128, 16352])
def test_tsqr_matches_oracle(cuda, evdlib, m):
    A = np.random.default_rng(m).standard_normal((m, 32))
    Qr, Rr = O.tsqr(A)
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    Q, R = evdlib.tsqr(Ad)
    torch.cuda.synchronize()
    Q, R = Q.cpu().numpy(), R.cpu().numpy()
    assert np.abs(R - Rr).max() <= 1e-12 * np.abs(Rr).max()
    assert np.abs(Q - Qr).max() <= 1e-12
    assert np.abs(Q.T @ Q - np.eye(32)).max() <= 1e-13
    assert np.abs(Q @ R - A).max() <= 1e-12 * np.abs(A).max()


@pytest.mark.parametrize("m", [32, 96, 128, 160, 640, 1056, 8192])
def test_panel_qr_matches_oracle(cuda, evdlib, m):
    A = np.random.default_rng(100 + m).standard_normal((m, 32))
    Yr, Wr, Rr = O.panel_qr(A)
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    Y, W, R = evdlib.panel_qr(Ad)
    torch.cuda.synchronize()
    Y, W, R = Y.cpu().numpy(), W.cpu().numpy(), R.cpu().numpy()
    assert np.abs(R - Rr).max() <= 1e-12 * np.abs(Rr).max()
    assert np.abs(Y - Yr).max() <= 1e-11
    assert np.abs(W - Wr).max() <= 1e-11
    # Householder form: unit lower Y, Q = I - W Y^T orthogonal, Q^T A = [R; 0]
    assert np.abs(np.triu(Y[:32], 1)).max() == 0.0
    assert np.abs(np.diag(Y[:32]) - 1.0).max() == 0.0
    Qf = np.eye(m) - W @ Y.T
    assert np.abs(Qf.T @ Qf - np.eye(m)).max() <= 1e-13 * 10
    QtA = Qf.T @ A
    assert np.abs(QtA[:32] - R).max() <= 1e-12 * np.abs(A).max() * 4
    if m > 32:
        assert np.abs(QtA[32:]).max() <= 1e-12 * np.abs(A).max() * 4


def test_panel_rejects_bad_shapes(cuda, evdlib):
    A = evdlib.to_cm(torch.randn(100, 32, dtype=torch.float64), device=cuda)  # m % 32 != 0
    with pytest.raises(evdlib.EvdError):
        evdlib.panel_qr(A)
