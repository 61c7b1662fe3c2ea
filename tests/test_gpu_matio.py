"""Matrix and eigenpair files with device memory, and the myEVD CLI's file
options (--save-input, --input, --output) around a real solve."""
import pathlib
import subprocess

import numpy as np
import pytest
import torch

from evd4sc2025_b200 import matio
from oracle import algos as O

pytestmark = pytest.mark.gpu

BIN = pathlib.Path(__file__).resolve().parent.parent / "evd4sc2025_b200" / "bin" / "myEVD"


def test_device_round_trip(cuda, evdlib, tmp_path):
    A = evdlib.to_cm(torch.from_numpy(O.sym_gaussian(500, 1)), device=cuda)
    f = tmp_path / "a.bin"
    matio.save_matrix(f, A)
    B = matio.load_matrix(f, device=cuda)
    assert B.is_cuda and torch.equal(A, B)
    assert torch.equal(matio.load_matrix(f), A.cpu())  # host read of a device write


def test_solve_save_reload(cuda, evdlib, tmp_path):
    n = 384
    A = O.sym_gaussian(n, 2)
    Ad = evdlib.to_cm(torch.from_numpy(A), device=cuda)
    w, X = evdlib.syevd(Ad, 32, 128)
    torch.cuda.synchronize()
    f = tmp_path / "eig.bin"
    matio.save_eigenpairs(f, w, X)
    w2, X2 = matio.load_eigenpairs(f, device=cuda)
    assert torch.equal(w, w2) and torch.equal(X, X2)
    assert O.residual(A, w2.cpu().numpy(), X2.cpu().numpy()) <= 1e-13


@pytest.mark.parametrize("n,nb", [(256, 64), (300, 128)])
def test_cli_file_options(cuda, evdlib, tmp_path, n, nb):
    if not BIN.exists():
        pytest.fail(f"{BIN} is missing: build with python -m evd4sc2025_b200.build")
    a, e1, e2 = tmp_path / "A.bin", tmp_path / "e1.bin", tmp_path / "e2.bin"
    r1 = subprocess.run([str(BIN), str(n), "32", str(nb), "--dist", "gauss", "--seed", "11",
                         "--save-input", str(a), "--output", str(e1)],
                        capture_output=True, text=True, timeout=300)
    assert r1.returncode == 0, r1.stdout + r1.stderr
    A = matio.load_matrix(a).numpy()
    assert A.shape == (n, n) and np.array_equal(A, A.T)
    w, X = matio.load_eigenpairs(e1)
    assert np.abs(w.numpy() - np.linalg.eigvalsh(A)).max() <= 1e-12 * np.linalg.norm(A, 2)
    assert O.residual(A, w.numpy(), X.numpy()) <= 1e-13
    # the same matrix read back through --input gives the same eigenpairs
    r2 = subprocess.run([str(BIN), str(n), "32", str(nb), "--input", str(a), "--output", str(e2)],
                        capture_output=True, text=True, timeout=300)
    assert r2.returncode == 0, r2.stdout + r2.stderr
    w2, X2 = matio.load_eigenpairs(e2)
    assert torch.equal(w, w2) and torch.equal(X, X2)
    # a size that does not match the file is refused
    r3 = subprocess.run([str(BIN), str(n + 32), "32", str(nb), "--input", str(a)],
                        capture_output=True, text=True, timeout=300)
    assert r3.returncode == 1 and "cannot read" in r3.stdout
