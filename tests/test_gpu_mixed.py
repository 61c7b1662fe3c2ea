"""The mixed form of the solve (evd_syevd_mixed): trailing SYR2K and stage-1
back transformation as emulated products on the integer tensor cores, then
optional Ogita-Aishima refinement.  Against LAPACK, the plain FP64 solve and
the reference build's eigenvalues, at the FP64 bars (eigenvalues 1e-12 ||A||,
residual and orthogonality 1e-13 in the reference's 1/n normalisation)."""
import pathlib

import numpy as np
import pytest
import torch

from oracle import algos as O

pytestmark = pytest.mark.gpu

GOLD = pathlib.Path(__file__).resolve().parent / "golden"


def _solve(evdlib, cuda, A, nb, **kw):
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    w, X = evdlib.syevd_mixed(Ad, 32, nb, **kw)
    res, orth = evdlib.check_eig(Ad, w, X)
    torch.cuda.synchronize()
    return w.cpu().numpy(), X, res, orth


@pytest.mark.parametrize("n,nb", [(1024, 256), (2048, 512), (4096, 1024)])
def test_mixed_fp64_level_products(cuda, evdlib, n, nb):
    A = O.sym_gaussian(n, seed=n + 5)
    nA = np.linalg.norm(A, 2)
    w, X, res, orth = _solve(evdlib, cuda, A, nb, moduli=14, refine_iters=0)
    assert res <= 1e-13 and orth <= 1e-13, (res, orth)
    assert np.abs(w - np.linalg.eigvalsh(A)).max() <= 1e-12 * nA
    # the plain solve on the same input
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    wp, Xp = evdlib.syevd(Ad, 32, nb)
    torch.cuda.synchronize()
    assert np.abs(w - wp.cpu().numpy()).max() <= 1e-13 * nA


@pytest.mark.parametrize("moduli,iters", [(8, 2), (10, 1), (12, 1)])
def test_mixed_reduced_products_refined(cuda, evdlib, moduli, iters):
    n = 2048
    A = O.sym_gaussian(n, seed=99)
    nA = np.linalg.norm(A, 2)
    w, X, res, orth = _solve(evdlib, cuda, A, 512, moduli=moduli, refine_iters=iters)
    assert res <= 1e-13 and orth <= 1e-13, (res, orth)
    assert np.abs(np.sort(w) - np.linalg.eigvalsh(A)).max() <= 1e-12 * nA


def test_mixed_reduced_products_unrefined_is_less_accurate(cuda, evdlib):
    """Without refinement 8 moduli (about 30-bit operands) leave an error far
    above FP64 level: the refinement is what wins the accuracy back."""
    n = 1024
    A = O.sym_gaussian(n, seed=3)
    w, X, res, orth = _solve(evdlib, cuda, A, 256, moduli=8, refine_iters=0)
    assert orth > 1e-12
    w2, X2, res2, orth2 = _solve(evdlib, cuda, A, 256, moduli=8, refine_iters=2)
    assert res2 <= 1e-13 and orth2 <= 1e-13, (res2, orth2)


@pytest.mark.parametrize("kind", ["uniform", "clustered", "geometric1e10"])
def test_mixed_known_spectra(cuda, evdlib, kind):
    n = 2048
    A, lam = O.known_spectrum_matrix(kind, n, seed=8)
    w, X, res, orth = _solve(evdlib, cuda, A, 512, moduli=14, refine_iters=0)
    assert res <= 1e-13 and orth <= 1e-13, (res, orth)
    # forming A rounds its spectrum by about sqrt(n) u ||A||
    assert np.abs(np.sort(w) - np.sort(lam)).max() <= 4e-13 * np.abs(lam).max()


def test_mixed_any_order(cuda, evdlib):
    n = 1500  # padded internally to 1536
    A = O.sym_gaussian(n, seed=15)
    w, X, res, orth = _solve(evdlib, cuda, A, 512, moduli=14, refine_iters=1)
    assert res <= 1e-13 and orth <= 1e-13, (res, orth)
    assert np.abs(np.sort(w) - np.linalg.eigvalsh(A)).max() <= 1e-12 * np.linalg.norm(A, 2)


@pytest.mark.parametrize("n,nb,moduli,iters", [(1, 64, 14, 0), (5, 64, 14, 0), (64, 64, 14, 0),
                                               (100, 64, 8, 2), (300, 128, 14, 1)])
def test_mixed_small_orders(cuda, evdlib, n, nb, moduli, iters):
    """Orders whose stage-2 T factors do not fit in the borrowed n x n buffer
    (the kernel then rebuilds them) and orders padded to 64."""
    A = O.sym_gaussian(n, seed=n + 3)
    w, X, res, orth = _solve(evdlib, cuda, A, nb, moduli=moduli, refine_iters=iters)
    assert res <= 1e-13 and orth <= 1e-13, (res, orth)
    assert np.abs(w - np.linalg.eigvalsh(A)).max() <= 1e-12 * max(np.linalg.norm(A, 2), 1.0)


def test_mixed_matches_reference_build(cuda, evdlib):
    f = np.load(GOLD / "ref_n4096_s13.npz")
    n, seed = int(f["n"]), int(f["seed"])
    A = O.sym_gaussian(n, seed)
    nA = np.linalg.norm(A, 2)
    w, X, res, orth = _solve(evdlib, cuda, A, 1024, moduli=14, refine_iters=0)
    assert np.abs(w - f["w"]).max() <= 1e-12 * nA
    X8 = X[:, :8].cpu().numpy()
    s = np.sign(np.sum(X8 * f["X8"], axis=0))
    assert np.abs(X8 - f["X8"] * s).max() <= 1e-9


@pytest.mark.parametrize("n,nb,moduli,iters", [(1024, 256, 14, 0), (1500, 256, 14, 0),
                                               (2048, 512, 8, 2)])
def test_mixed_minimal_workspace_one_chain(cuda, evdlib, n, nb, moduli, iters):
    """With the smallest workspace the solve runs one stage-2 chain and the
    divide and conquer after the Q1 formation (the schedule of orders above
    24576): same bars, same eigenvalues as the full-workspace schedule."""
    A = O.sym_gaussian(n, seed=n + 17)
    nA = np.linalg.norm(A, 2)
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    lmin = evdlib.lib().evd_syevd_mixed_work_size_min(n, 32, nb, moduli, iters)
    lfull = evdlib.lib().evd_syevd_mixed_work_size(n, 32, nb, moduli, iters)
    assert 0 < lmin < lfull
    wsm = evdlib.MixedWorkspace(n, 32, nb, moduli, iters, device=cuda, minimal=True)
    assert wsm.nbytes == lmin
    w1, X1 = evdlib.syevd_mixed(Ad, 32, nb, moduli, iters, ws=wsm)
    w2, X2 = evdlib.syevd_mixed(Ad, 32, nb, moduli, iters)
    r1, o1 = evdlib.check_eig(Ad, w1, X1)
    r2, o2 = evdlib.check_eig(Ad, w2, X2)
    torch.cuda.synchronize()
    assert r1 <= 1e-13 and o1 <= 1e-13, (r1, o1)
    assert r2 <= 1e-13 and o2 <= 1e-13, (r2, o2)
    w1, w2 = w1.cpu().numpy(), w2.cpu().numpy()
    assert np.abs(w1 - np.linalg.eigvalsh(A)).max() <= 1e-12 * nA
    assert np.abs(w1 - w2).max() <= 1e-13 * nA
    # one byte short of the minimum is rejected before any device work
    short = torch.empty(lmin - 1, dtype=torch.uint8, device=cuda)
    wd = torch.empty(n, dtype=torch.float64, device=cuda)
    Xd = evdlib.empty_cm(n, n, device=cuda)
    rc = evdlib.lib().evd_syevd_mixed(n, 32, nb, Ad.data_ptr(), n, wd.data_ptr(),
                                      Xd.data_ptr(), n, moduli, iters, 14, short.data_ptr(),
                                      lmin - 1, 0, None)
    assert rc == -5  # EVD_ERR_WORKSPACE
