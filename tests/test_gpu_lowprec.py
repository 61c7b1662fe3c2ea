"""FP32 / FP16 entry points (tc_syr2k, tc_ozimmu_syr2k<float/half>,
panelQR<float/half>, hou_tsqr_panel<float/half>) against FP64 references of
the same arithmetic.

Tolerances: with FP16 operands every product is exact in FP32 (11 x 11 bits),
so the FP32 accumulation is the only error: |C - C_ref| <= 4 k u32 (|alpha| S
+ |beta| |C|) elementwise, S = |A||B|^T + |B||A|^T, u32 = 2^-24; FP16 output
adds one FP16 rounding (2^-11 relative).  The FP32 SIMT product adds one FP32
rounding per product (same bound form).  Panel QR in FP32/FP16 is the FP64
panel on the converted input, rounded once: it must equal the rounded FP64
result bit for bit."""
import math

import pytest
import torch

from evd4sc2025_b200 import lowprec as LP

pytestmark = pytest.mark.gpu

U32 = 2.0 ** -24


def _data(n, k, seed, dev, dtype=torch.float32):
    g = torch.Generator().manual_seed(seed)
    A = torch.randn(n, k, generator=g, dtype=torch.float64)
    B = torch.randn(n, k, generator=g, dtype=torch.float64)
    Cm = torch.randn(n, n, generator=g, dtype=torch.float64)
    return (LP.to_cm(A, dtype, dev), LP.to_cm(B, dtype, dev), LP.to_cm(Cm, dtype, dev))


def _ref(alpha, Ad, Bd, beta, Cd):
    S = Ad.abs() @ Bd.abs().t() + Bd.abs() @ Ad.abs().t()
    ref = alpha * (Ad @ Bd.t() + Bd @ Ad.t()) + beta * Cd
    bound = abs(alpha) * S + abs(beta) * Cd.abs()
    return ref, bound


def _check_lower(Cout, C0, ref, bound, k, extra_rel=0.0):
    n = ref.shape[0]
    low = torch.tril(torch.ones(n, n, dtype=torch.bool))
    got = Cout.double().cpu()
    err = (got - ref).abs()
    tol = 4 * max(k, 1) * U32 * bound + extra_rel * ref.abs() + 1e-30
    assert bool((err[low] <= tol[low]).all()), float((err - tol)[low].max())
    # strictly upper triangle untouched
    up = ~low
    assert torch.equal(got[up], C0.double().cpu()[up])


@pytest.mark.parametrize("n,k", [(1, 1), (100, 7), (128, 64), (300, 200), (1000, 256),
                                 (513, 1024), (200, 40), (129, 8)])
@pytest.mark.parametrize("alpha,beta", [(-1.0, 1.0), (0.5, 0.0), (2.0, -0.25)])
@pytest.mark.parametrize("packed", [True, False])
def test_tc_syr2k(cuda, evdlib, n, k, alpha, beta, packed):
    """packed: operands packed into the caller's FP16 workspace (k % 64 == 0;
    other k use the library's buffer); else into the library's buffer."""
    A, B, Cm = _data(n, k, n * 7 + k, cuda)
    if beta == 0.0:
        Cm.fill_(float("nan"))  # beta == 0 must not read C (lower NaN, upper 0)
        Cm.tril_()
    C0 = Cm.clone()
    LP.tc_syr2k(alpha, A, B, beta, Cm, hwork=True if packed else None)
    torch.cuda.synchronize()
    Ah, Bh = A.half().double().cpu(), B.half().double().cpu()
    Cd = torch.nan_to_num(C0.double().cpu()) if beta == 0.0 else C0.double().cpu()
    ref, bound = _ref(alpha, Ah, Bh, beta, Cd)
    _check_lower(Cm, C0, ref, bound, k)


@pytest.mark.parametrize("n,k", [(1, 3), (100, 7), (300, 200), (1000, 256)])
def test_syr2k_lower_fp32(cuda, evdlib, n, k):
    alpha, beta = -1.0, 0.75
    A, B, Cm = _data(n, k, n + 3 * k, cuda)
    C0 = Cm.clone()
    LP.syr2k_lower(alpha, A, B, beta, Cm)
    torch.cuda.synchronize()
    ref, bound = _ref(alpha, A.double().cpu(), B.double().cpu(), beta, C0.double().cpu())
    _check_lower(Cm, C0, ref, bound, k)


@pytest.mark.parametrize("n,k", [(1, 2), (100, 7), (300, 64), (1000, 256)])
def test_syr2k_lower_fp16(cuda, evdlib, n, k):
    alpha, beta = -1.0, 1.0
    A, B, Cm = _data(n, k, 5 * n + k, cuda, torch.float16)
    A.mul_(0.25)
    B.mul_(0.25)
    C0 = Cm.clone()
    LP.syr2k_lower(alpha, A, B, beta, Cm)
    torch.cuda.synchronize()
    ref, bound = _ref(alpha, A.double().cpu(), B.double().cpu(), beta, C0.double().cpu())
    _check_lower(Cm, C0, ref, bound, k, extra_rel=2.0 ** -11)


def test_syr2k_degenerate_sizes(cuda, evdlib):
    A, B, Cm = _data(50, 4, 9, cuda)
    C0 = Cm.clone()
    Z = A[:, :0]
    LP.tc_syr2k(1.0, Z, B[:, :0], 0.5, Cm)     # k == 0: C(lower) = beta C
    LP.syr2k_lower(0.0, A, B, 2.0, Cm)           # alpha == 0: C(lower) *= 2
    torch.cuda.synchronize()
    low = torch.tril(torch.ones(50, 50, dtype=torch.bool))
    got = Cm.double().cpu()
    want = C0.double().cpu()[low] * 0.5 * 2.0   # beta 0.5, then 2
    assert torch.allclose(got[low], want, rtol=1e-6, atol=0)
    assert torch.equal(got[~low], C0.double().cpu()[~low])
    E = LP.empty_cm(0, 0, torch.float32, cuda)
    LP.tc_syr2k(1.0, LP.empty_cm(0, 3, torch.float32, cuda), LP.empty_cm(0, 3, torch.float32, cuda),
                0.0, E)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16])
@pytest.mark.parametrize("m", [128, 1024, 4096])
def test_panel_qr_lowprec_is_rounded_fp64(cuda, evdlib, dtype, m):
    g = torch.Generator().manual_seed(m)
    A = LP.to_cm(torch.randn(m, 32, generator=g, dtype=torch.float64), dtype, cuda)
    Ad = evdlib.to_cm(A.double(), device=cuda)
    Y, W, R = LP.panel_qr(A.clone())
    Yd, Wd, Rd = evdlib.panel_qr(Ad)
    Q, Rq = LP.tsqr(A.clone())
    Qd, Rqd = evdlib.tsqr(evdlib.to_cm(A.double(), device=cuda))
    torch.cuda.synchronize()
    for got, ref in ((Y, Yd), (W, Wd), (R, Rd), (Q, Qd), (Rq, Rqd)):
        if dtype == torch.float32:  # one FP64 -> FP32 rounding: bit-exact
            assert torch.equal(got, ref.to(dtype))
        else:  # FP64 -> FP16 rounded directly: within half an FP16 ulp
            err = (got.double() - ref).abs()
            assert bool((err <= 2.0 ** -11 * ref.abs() + 2.0 ** -25).all())
    # and the factorisation holds to the precision of the type
    eps = 2.0 ** -23 if dtype == torch.float32 else 2.0 ** -10
    QR = Q.double() @ Rq.double()
    assert float((QR - A.double()).abs().max()) <= 8 * eps * math.sqrt(m) * float(A.double().abs().max())
