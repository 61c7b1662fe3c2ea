"""The FP32 solve (evd_syevd_s): FP32 matrices in and out, the mixed form
with 8 moduli and no refinement inside.  Against LAPACK on the FP64 value of
the same FP32 input, at FP32 bars: eigenvalues within 1e-6 ||A||_2, residual
||AX - X diag(w)||_F / ||A||_F and orthogonality ||X^T X - I||_F within 1e-5
(1e-6 after the reference's 1/n normalisation, the FP32-tolerance class of
the serving workload)."""
import numpy as np
import pytest
import torch

import evd4sc2025_b200 as evd
from oracle import algos as O

pytestmark = pytest.mark.gpu


def _check(A32, w, X):
    A = A32.astype(np.float64)
    n = A.shape[0]
    w = w.cpu().numpy().astype(np.float64)
    X = X.cpu().numpy().astype(np.float64)
    nA2 = np.linalg.norm(A, 2)
    assert np.all(np.diff(w) >= 0)
    assert np.abs(w - np.linalg.eigvalsh(A)).max() <= 1e-6 * nA2
    res = np.linalg.norm(A @ X - X * w) / np.linalg.norm(A)
    orth = np.linalg.norm(X.T @ X - np.eye(n))
    assert res <= 1e-5 and orth <= 1e-5, (res, orth)
    assert res / n <= 1e-6 and orth / n <= 1e-6


@pytest.mark.parametrize("n,nb", [(1, 64), (5, 64), (64, 64), (100, 64), (1024, 256),
                                  (1500, 512), (2048, 512)])
def test_fp32_solve_matches_lapack(cuda, evdlib, n, nb):
    A32 = O.sym_gaussian(n, seed=n + 41).astype(np.float32)
    Ad = evd.empty_cm(n, n, device=cuda, dtype=torch.float32)
    Ad.copy_(torch.from_numpy(A32))
    w, X = evd.syevd_s(Ad, 32, nb)
    torch.cuda.synchronize()
    assert w.dtype == torch.float32 and X.dtype == torch.float32
    _check(A32, w, X)


def test_fp32_solve_known_spectrum(cuda, evdlib):
    n = 1024
    A, lam = O.known_spectrum_matrix("uniform", n, seed=4)
    A32 = A.astype(np.float32)
    Ad = evd.empty_cm(n, n, device=cuda, dtype=torch.float32)
    Ad.copy_(torch.from_numpy(A32))
    w, X = evd.syevd_s(Ad, 32, 256)
    torch.cuda.synchronize()
    _check(A32, w, X)
    # rounding A to FP32 moves its eigenvalues by about u_32 ||A||
    assert np.abs(np.sort(w.cpu().numpy()) - np.sort(lam)).max() <= 1e-6 * np.abs(lam).max()


def test_fp32_solve_agrees_with_the_fp64_solve(cuda, evdlib):
    n = 1024
    A32 = O.sym_gaussian(n, seed=77).astype(np.float32)
    Ad = evd.empty_cm(n, n, device=cuda, dtype=torch.float32)
    Ad.copy_(torch.from_numpy(A32))
    w, X = evd.syevd_s(Ad, 32, 256)
    A64 = evd.to_cm(torch.from_numpy(A32.astype(np.float64)), device=cuda)
    w64, X64 = evd.syevd(A64, 32, 256)
    torch.cuda.synchronize()
    nA = float(np.linalg.norm(A32.astype(np.float64), 2))
    assert float((w.double() - w64).abs().max()) <= 1e-6 * nA
    # eigenvectors agree up to sign (distinct eigenvalues of a Gaussian matrix)
    d = (X.double().t() @ X64).diagonal().abs()
    assert float((d - 1).abs().max()) <= 1e-4


def test_fp32_solve_rejects_bad_arguments(cuda, evdlib):
    lib = evd.lib()
    n, nb = 256, 256
    need = lib.evd_syevd_s_work_size(n, 32, nb)
    assert need > 0 and lib.evd_syevd_s_work_size(n, 16, nb) == 0
    A = evd.empty_cm(n, n, device=cuda, dtype=torch.float32)
    A.copy_(torch.from_numpy(O.sym_gaussian(n, seed=1).astype(np.float32)))
    w = torch.empty(n, dtype=torch.float32, device=cuda)
    X = evd.empty_cm(n, n, device=cuda, dtype=torch.float32)
    short = torch.empty(need - 1, dtype=torch.uint8, device=cuda)
    rc = lib.evd_syevd_s(n, 32, nb, A.data_ptr(), n, w.data_ptr(), X.data_ptr(), n,
                         short.data_ptr(), need - 1, None)
    assert rc == -5  # EVD_ERR_WORKSPACE
    rc = lib.evd_syevd_s(n, 32, nb, A.data_ptr(), n - 1, w.data_ptr(), X.data_ptr(), n,
                         short.data_ptr(), need - 1, None)
    assert rc == -1  # EVD_ERR_INVALID_ARG (lda < n)
