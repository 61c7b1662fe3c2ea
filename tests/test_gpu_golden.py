"""The CUDA pipeline vs the reference's own GPU build on the same inputs
(fixtures in tests/golden/, produced by tests/golden/make_golden.py)."""
import pathlib

import numpy as np
import pytest
import torch

from oracle import algos as O

pytestmark = pytest.mark.gpu

GOLD = pathlib.Path(__file__).resolve().parent / "golden"
FIXTURES = sorted(GOLD.glob("ref_n*_s*.npz"))


@pytest.mark.parametrize("path", FIXTURES, ids=[p.stem for p in FIXTURES])
def test_pipeline_matches_reference_build(cuda, evdlib, path):
    f = np.load(path)
    n, seed = int(f["n"]), int(f["seed"])
    A = O.sym_gaussian(n, seed)
    nA = np.linalg.norm(A, 2)
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    # same stage-1/2 path: tridiagonal equal to the reference's up to rounding
    band, W, Y = evdlib.sy2sb(Ad, 32, 1024)
    d, e, U = evdlib.bulge_chase(evdlib.band_pack(band, 32), 32)
    torch.cuda.synchronize()
    assert np.abs(np.abs(d.cpu().numpy()) - np.abs(f["d"])).max() <= 1e-10 * nA
    assert np.abs(np.abs(e.cpu().numpy()) - np.abs(f["e"])).max() <= 1e-10 * nA
    # whole solver: eigenvalues to 1e-12 ||A||, eigenvectors up to sign
    w, X = evdlib.syevd(Ad, 32, 1024)
    res, orth = evdlib.check_eig(Ad, w, X)
    torch.cuda.synchronize()
    assert np.abs(w.cpu().numpy() - f["w"]).max() <= 1e-12 * nA
    assert res <= 1e-13 and orth <= 1e-13
    X8 = X[:, :8].cpu().numpy()
    s = np.sign(np.sum(X8 * f["X8"], axis=0))
    assert np.abs(X8 - f["X8"] * s).max() <= 1e-9
