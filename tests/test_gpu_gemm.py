"""FP64 DMMA GEMM / SYR2K kernels vs a torch FP64 reference (floating-point kernels)."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rand(m, n, dev, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    return torch.randn(m, n, generator=g, dtype=torch.float64).to(dev)


def _tol(k):
    # FP64 dot products of length k with N(0,1) entries: error ~ eps * k
    return 64 * 2.2e-16 * max(k, 1) * 4


@pytest.mark.parametrize("ta", ["n", "t"])
@pytest.mark.parametrize("tb", ["n", "t"])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (128, 128, 16), (130, 33, 47),
                                   (257, 129, 300), (64, 32, 1000), (1000, 32, 2048),
                                   (517, 600, 129)])
def test_dgemm_matches_torch(cuda, evdlib, ta, tb, m, n, k):
    A = _rand(k if ta == "t" else m, m if ta == "t" else k, cuda, 1)
    B = _rand(n if tb == "t" else k, k if tb == "t" else n, cuda, 2)
    C0 = _rand(m, n, cuda, 3)
    opA = A.t() if ta == "t" else A
    opB = B.t() if tb == "t" else B
    ref = 1.5 * (opA @ opB) - 0.5 * C0
    Cm = evdlib.to_cm(C0)
    evdlib.dgemm(ta, tb, 1.5, evdlib.to_cm(A), evdlib.to_cm(B), -0.5, Cm)
    torch.cuda.synchronize()
    assert (Cm - ref).abs().max().item() <= _tol(k)


def test_dgemm_beta_zero_ignores_nan(cuda, evdlib):
    A = _rand(65, 40, cuda, 4)
    B = _rand(40, 70, cuda, 5)
    Cm = evdlib.to_cm(torch.full((65, 70), float("nan"), dtype=torch.float64, device=cuda))
    evdlib.dgemm("n", "n", 1.0, evdlib.to_cm(A), evdlib.to_cm(B), 0.0, Cm)
    torch.cuda.synchronize()
    assert torch.isfinite(Cm).all()
    assert (Cm - A @ B).abs().max().item() <= _tol(40)


def test_dgemm_odd_leading_dimension(cuda, evdlib):
    # ld odd -> 8-byte copies path
    A = evdlib.to_cm(_rand(99, 50, cuda, 6), ld=101)
    B = evdlib.to_cm(_rand(50, 77, cuda, 7), ld=53)
    Cm = evdlib.to_cm(torch.zeros(99, 77, dtype=torch.float64, device=cuda), ld=103)
    evdlib.dgemm("n", "n", 1.0, A, B, 0.0, Cm)
    torch.cuda.synchronize()
    assert (Cm - A @ B).abs().max().item() <= _tol(50)


@pytest.mark.parametrize("n,k", [(1, 1), (33, 7), (128, 64), (300, 1024), (1000, 96)])
def test_syr2k_lower_mirror(cuda, evdlib, n, k):
    A = _rand(n, k, cuda, 8)
    B = _rand(n, k, cuda, 9)
    C0 = _rand(n, n, cuda, 10)
    C0 = C0 + C0.t()
    ref = -1.0 * (A @ B.t() + B @ A.t()) + 1.0 * C0
    ref = torch.tril(ref) + torch.tril(ref, -1).t()
    Cm = evdlib.to_cm(C0)
    evdlib.syr2k(-1.0, evdlib.to_cm(A), evdlib.to_cm(B), 1.0, Cm)
    torch.cuda.synchronize()
    assert (Cm - ref).abs().max().item() <= _tol(2 * k)
    assert torch.equal(Cm, Cm.t())  # exact mirror


def test_strided_batched(cuda, evdlib):
    import ctypes as C
    batch, m, n, k = 5, 40, 24, 33
    A = _rand(m * batch, k, cuda, 11)   # batch member b = rows b*m.. (stride m)
    B = _rand(k * batch, n, cuda, 12)
    Am = evdlib.to_cm(A)
    Bm = evdlib.to_cm(B)
    Cm = evdlib.to_cm(torch.zeros(m * batch, n, dtype=torch.float64, device=cuda))
    evdlib.lib()
    from evd4sc2025_b200._native import call
    call("evd_dgemm_strided_batched", b"n", b"n", m, n, k, 1.0,
         C.c_void_p(Am.data_ptr()), Am.stride(1), m,
         C.c_void_p(Bm.data_ptr()), Bm.stride(1), k, 0.0,
         C.c_void_p(Cm.data_ptr()), Cm.stride(1), m, batch,
         C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    for bi in range(batch):
        ref = A[bi * m:(bi + 1) * m] @ B[bi * k:(bi + 1) * k]
        assert (Cm[bi * m:(bi + 1) * m] - ref).abs().max().item() <= _tol(k)
