"""Batched uneven sizes and the serving loop on the GPU: padded solves match
LAPACK, concurrent solves match solves run alone, and every request served in
the mix matches the same request served alone."""
import numpy as np
import pytest
import torch

from evd4sc2025_b200 import serve

pytestmark = pytest.mark.gpu


def _sym(n, seed):
    g = torch.Generator().manual_seed(seed)
    G = torch.randn(n, n, generator=g, dtype=torch.float64)
    return 0.5 * (G + G.t())


def _check(A, w, X):
    A = A.numpy()
    w = w.cpu().numpy()
    X = X.cpu().numpy()
    n = A.shape[0]
    nrm = np.linalg.norm(A, 2)
    w_ref = np.linalg.eigvalsh(A)
    assert np.abs(w - w_ref).max() <= 1e-12 * nrm
    res = np.linalg.norm(A @ X - X * w) / (n * np.linalg.norm(A))
    orth = np.linalg.norm(X.T @ X - np.eye(n)) / n
    assert res <= 1e-13 and orth <= 1e-13, (res, orth)


@pytest.mark.parametrize("n", [1, 2, 5, 33, 100, 257, 500, 1100])
def test_any_order_matches_lapack(cuda, evdlib, n):
    A = _sym(n, n)
    w, X = serve.syevd_any(A.to(cuda))
    _check(A, w, X)


def test_batched_matches_one_at_a_time(cuda, evdlib):
    sizes = [64, 70, 100, 129, 200, 257, 300, 333, 512, 640, 700, 1024]
    mats = [_sym(n, 100 + i).to(cuda) for i, n in enumerate(sizes)]
    out, ms = serve.syevd_batched(mats, nstreams=4)
    assert ms > 0
    one = serve.StreamSolver(cuda)
    for A, (w, X) in zip(mats, out):
        w1, X1 = serve.syevd_any(A, one)
        nrm = float(torch.linalg.matrix_norm(A, ord=2))
        assert float((w - w1).abs().max()) <= 1e-13 * nrm
        # eigenvectors agree up to sign (distinct eigenvalues)
        d = (X.t() @ X1).diagonal().abs()
        assert float((d - 1).abs().max()) <= 1e-10
        _check(A.cpu(), w, X)


def test_native_batched_matches_single_solves(cuda, evdlib):
    """evd_syevd_batched (threads and streams inside the library) gives, for
    every matrix, exactly what evd_syevd gives alone with the same nb."""
    sizes = [1, 33, 64, 100, 257, 512, 700, 1024, 90, 2]
    mats = [evdlib.to_cm(_sym(n, 300 + i), device=cuda) for i, n in enumerate(sizes)]
    out, ms = serve.syevd_batched_native(mats, nstreams=3)
    assert ms > 0
    for A, (w, X) in zip(mats, out):
        n = A.shape[0]
        _, nb = serve.padded_shape(n)
        w1, X1 = evdlib.syevd(A, 32, nb)
        torch.cuda.synchronize()
        assert torch.equal(w, w1) and torch.equal(X, X1)
        _check(A.cpu(), w, X)


def test_server_mix_matches_alone(cuda, evdlib):
    reqs = serve.poisson_stream(16, 400.0, 64, 600, seed=11)
    srv = serve.Server(nworkers=4, budget_bytes=8 * 10**9, device=cuda)
    stats = srv.run(reqs)
    assert stats["requests"] == len(reqs)
    assert stats["p99_s"] >= stats["p50_s"] > 0
    alone = serve.StreamSolver(cuda)
    for r, res in zip(sorted(reqs, key=lambda q: q.rid), srv.results):
        assert r.rid == res.rid
        w1, X1 = serve.syevd_any(r.A.to(cuda), alone)
        nrm = float(torch.linalg.matrix_norm(r.A, ord=2))
        assert float((res.w - w1.cpu()).abs().max()) <= 1e-13 * nrm
        _check(r.A, res.w, res.X)


def _check_class(A, w, X, tol):
    A = A.numpy()
    w = w.cpu().numpy()
    X = X.cpu().numpy()
    n = A.shape[0]
    res = np.linalg.norm(A @ X - X * w) / (n * np.linalg.norm(A))
    orth = np.linalg.norm(X.T @ X - np.eye(n)) / n
    bar = 1e-13 if tol == "fp64" else 1e-6
    assert res <= bar and orth <= bar, (tol, res, orth)
    nrm = np.linalg.norm(A, 2)
    ebar = 1e-12 if tol == "fp64" else 1e-6
    assert np.abs(np.sort(w) - np.linalg.eigvalsh(A)).max() <= ebar * nrm


def test_server_two_classes_mix_matches_alone(cuda, evdlib):
    """FP64-accurate and FP32-tolerance requests, some large enough for the
    mixed form: each result in the mix equals the same request solved alone
    by the same form, and meets its class's bars."""
    reqs = serve.poisson_stream(10, 200.0, 1200, 3000, seed=21, fp64_fraction=0.6)
    assert {r.tol for r in reqs} == {"fp64", "fp32"}
    assert any(r.A.shape[0] >= serve.MIXED_MIN_N for r in reqs)
    srv = serve.Server(nworkers=3, budget_bytes=40 * 10**9, device=cuda)
    stats = srv.run(reqs)
    assert stats["requests"] == len(reqs) and stats["failed"] == 0
    assert set(stats["per_class"]) == {"fp64", "fp32"}
    alone = serve.StreamSolver(cuda)
    for r, res in zip(sorted(reqs, key=lambda q: q.rid), srv.results):
        assert r.rid == res.rid and res.tol == r.tol
        w1, X1 = alone.solve(r.A.to(cuda), tol=r.tol)
        alone.stream.synchronize()
        nrm = float(torch.linalg.matrix_norm(r.A, ord=2))
        assert float((res.w - w1.cpu()).abs().max()) <= 1e-13 * nrm
        _check_class(r.A, res.w, res.X, r.tol)


def test_request_form_rule(evdlib):
    assert serve.request_form(1000, "fp64") == ("plain", 0)
    assert serve.request_form(4096, "fp64") == ("mixed", serve.FP64_MODULI)
    assert serve.request_form(4096, "fp32") == ("mixed", serve.FP32_MODULI)
    with pytest.raises(ValueError):
        serve.request_form(4096, "fp16")
