"""sy2sb (full -> band, ZY) via the C ABI vs the oracle restatement of my_ZY_ZY_SBR_Vector."""
import numpy as np
import pytest
import torch

from oracle import algos as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,nb", [(64, 32), (128, 64), (256, 128), (512, 256), (512, 512),
                                  (1024, 256)])
def test_sy2sb_matches_oracle(cuda, evdlib, n, nb):
    A = O.sym_gaussian(n, seed=n + nb)
    band_r, W_r, Y_r = O.sy2sb(A, 32, nb)
    band, W, Y = evdlib.sy2sb(evdlib.to_cm(torch.from_numpy(A), device=cuda), 32, nb)
    torch.cuda.synchronize()
    band, W, Y = band.cpu().numpy(), W.cpu().numpy(), Y.cpu().numpy()
    scale = np.linalg.norm(A, 2)
    assert np.abs(band - band_r).max() <= 1e-11 * scale
    assert np.abs(Y - Y_r).max() <= 1e-9
    assert np.abs(W - W_r).max() <= 1e-9
    # exact structure: symmetric band of width 32
    assert np.array_equal(band, band.T)
    i, j = np.nonzero(band)
    assert np.abs(i - j).max() <= 32
    # similarity: A = Q1 B Q1^T and the spectrum is preserved
    Q1 = O.q1_apply(np.eye(n), W, Y, n, 32)
    assert np.abs(Q1 @ band @ Q1.T - A).max() <= 1e-12 * scale * 8
    assert np.abs(np.linalg.eigvalsh(band) - np.linalg.eigvalsh(A)).max() <= 1e-12 * scale * 8


def test_sy2sb_rejects_bad_sizes(cuda, evdlib):
    A = evdlib.to_cm(torch.eye(96, dtype=torch.float64), device=cuda)
    with pytest.raises(evdlib.EvdError):
        evdlib.sy2sb(A, 32, 64)  # 96 % 64 != 0 ("M must be diviable by nb!")
