"""Argument checks of the Python wrappers (no GPU): they refuse what the C
ABI cannot take before any device work."""
import pytest
import torch

pytest.importorskip("evd4sc2025_b200")
from evd4sc2025_b200 import autotune, lowprec, matio, serve  # noqa: E402


def test_lowprec_rejects_host_and_wrong_dtype():
    with pytest.raises(ValueError):
        lowprec._cm(torch.zeros(4, 4, dtype=torch.float32), "A")        # host tensor
    with pytest.raises(TypeError):
        lowprec._cm(torch.zeros(4, 4, dtype=torch.float64), "A")        # FP64 is not FP32/FP16


def test_matio_rejects_non_fp64(tmp_path):
    with pytest.raises(TypeError):
        matio.save_matrix(tmp_path / "x.bin", torch.zeros(3, 3, dtype=torch.float32))
    with pytest.raises(ValueError):
        matio.save_eigenpairs(tmp_path / "e.bin", torch.zeros(3, dtype=torch.float64),
                              torch.zeros(3, 4, dtype=torch.float64))


def test_orders_below_one_rejected():
    with pytest.raises(ValueError):
        serve.padded_shape(0)
    with pytest.raises(ValueError):
        autotune.choose_nb(0, {"entries": [{"n": 64, "nb": 64, "ms": {"64": 1.0}}]})


def test_row_major_matrices_are_written_column_major(tmp_path):
    A = torch.arange(12, dtype=torch.float64).reshape(3, 4)   # row-major
    matio.save_matrix(tmp_path / "a.bin", A)
    assert torch.equal(matio.load_matrix(tmp_path / "a.bin"), A)
