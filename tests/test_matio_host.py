"""Matrix and eigenpair files on host memory (no GPU): binary record layout,
round trips, appended records, CSV in the reference's row-per-line layout,
and the error statuses."""
import struct

import numpy as np
import pytest
import torch

pytest.importorskip("evd4sc2025_b200")
from evd4sc2025_b200 import matio  # noqa: E402
from evd4sc2025_b200._native import EvdError  # noqa: E402


def _rand(m, n, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.randn(m, n, generator=g, dtype=torch.float64)


def test_binary_record_layout(tmp_path):
    A = _rand(5, 3, 1)
    f = tmp_path / "a.bin"
    matio.save_matrix(f, A)
    raw = f.read_bytes()
    assert len(raw) == 32 + 5 * 3 * 8
    magic, ver, eb, res, rows, cols = struct.unpack("<4sIIIqq", raw[:32])
    assert (magic, ver, eb, res, rows, cols) == (b"EVDM", 1, 8, 0, 5, 3)
    vals = np.frombuffer(raw[32:], dtype="<f8").reshape(3, 5).T  # column-major
    assert np.array_equal(vals, A.numpy())


def test_binary_round_trip_and_append(tmp_path):
    f = tmp_path / "m.bin"
    mats = [_rand(7, 7, 2), _rand(1, 9, 3), _rand(300, 40, 4), torch.zeros(0, 4, dtype=torch.float64)]
    for i, M in enumerate(mats):
        matio.save_matrix(f, M, append=i > 0)
    assert matio.count_matrices(f) == len(mats)
    for i, M in enumerate(mats):
        assert matio.matrix_shape(f, i) == tuple(M.shape)
        assert torch.equal(matio.load_matrix(f, i), M)


def test_strided_and_row_major_inputs(tmp_path):
    big = _rand(20, 20, 5)
    sub = big.t().contiguous().t()[2:9, 3:8]  # column-major view with ld 20
    f = tmp_path / "s.bin"
    matio.save_matrix(f, sub)
    assert torch.equal(matio.load_matrix(f), sub)
    rm = _rand(6, 4, 6)  # row-major tensor
    matio.save_matrix(f, rm)
    assert torch.equal(matio.load_matrix(f), rm)


def test_eigenpairs_round_trip(tmp_path):
    n = 33
    A = _rand(n, n, 7)
    A = 0.5 * (A + A.t())
    w, X = torch.linalg.eigh(A)
    f = tmp_path / "e.bin"
    matio.save_eigenpairs(f, w, X)
    assert matio.count_matrices(f) == 2
    w2, X2 = matio.load_eigenpairs(f)
    assert torch.equal(w, w2) and torch.equal(X, X2)


def test_csv_round_trip_is_exact(tmp_path):
    A = _rand(6, 5, 8) * torch.logspace(-300, 300, 5, dtype=torch.float64)
    f = tmp_path / "a.csv"
    matio.save_csv(f, A)
    lines = f.read_text().strip().split("\n")
    assert len(lines) == 6 and all(len(l.split(",")) == 5 for l in lines)
    assert torch.equal(matio.load_csv(f), A)


def test_csv_reads_reference_style_text(tmp_path):
    f = tmp_path / "r.csv"
    f.write_text("1,2,3\n4.5,5e-3, -6\r\n")
    A = matio.load_csv(f)
    assert torch.equal(A, torch.tensor([[1, 2, 3], [4.5, 5e-3, -6]], dtype=torch.float64))


def test_errors(tmp_path):
    with pytest.raises(EvdError) as e:
        matio.load_matrix(tmp_path / "missing.bin")
    assert e.value.status == -6
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"NOPE" + bytes(28))
    with pytest.raises(EvdError) as e:
        matio.count_matrices(bad)
    assert e.value.status == -6
    f = tmp_path / "one.bin"
    matio.save_matrix(f, _rand(3, 3, 9))
    with pytest.raises(EvdError):
        matio.load_matrix(f, index=1)          # no such record
    trunc = tmp_path / "trunc.bin"
    trunc.write_bytes(f.read_bytes()[:-8])
    with pytest.raises(EvdError):
        matio.load_matrix(trunc)               # short data
    rag = tmp_path / "rag.csv"
    rag.write_text("1,2\n3\n")
    with pytest.raises(EvdError):
        matio.load_csv(rag)
