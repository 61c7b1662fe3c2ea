"""Host logic of the batched/serving layer (no GPU): padding rule, admission
under a memory budget, FIFO service, latency statistics."""
import threading
import time

import pytest
import torch

pytest.importorskip("evd4sc2025_b200")
from evd4sc2025_b200 import serve  # noqa: E402


@pytest.mark.parametrize("n,np_,nb", [(1, 64, 64), (64, 64, 64), (65, 96, 32), (100, 128, 128),
                                      (1000, 1024, 1024), (1025, 1056, 32), (3000, 3008, 64),
                                      (8192, 8192, 1024), (16384, 16384, 1024)])
def test_padded_shape(n, np_, nb):
    assert serve.padded_shape(n) == (np_, nb)
    assert np_ % nb == 0 and (nb // 32) & (nb // 32 - 1) == 0


def test_padding_keeps_the_spectrum():
    """The padded block-diagonal matrix has A's eigenpairs as its n smallest."""
    g = torch.Generator().manual_seed(3)
    n = 45
    G = torch.randn(n, n, generator=g, dtype=torch.float64)
    A = 0.5 * (G + G.t())
    np_, _ = serve.padded_shape(n)
    s = float(torch.linalg.matrix_norm(A, ord=1))
    k = np_ - n
    P = torch.zeros(np_, np_, dtype=torch.float64)
    P[:n, :n] = A
    P[n:, n:] = torch.diag(2 * s + s * torch.arange(k, dtype=torch.float64) / k)
    w_p, X_p = torch.linalg.eigh(P)
    w_a = torch.linalg.eigvalsh(A)
    assert torch.allclose(w_p[:n], w_a, atol=1e-12 * s)
    assert float(X_p[n:, :n].abs().max()) <= 1e-12


def _fake_requests(sizes, gap=0.002):
    return [serve.Request(i * gap, i, torch.zeros(n, n, dtype=torch.float64))
            for i, n in enumerate(sizes)]


def test_admission_respects_budget_and_serves_everything():
    in_flight = {"now": 0, "max": 0}
    lock = threading.Lock()

    def solve(k, A, tol):
        n = A.shape[0]
        with lock:
            in_flight["now"] += n
            in_flight["max"] = max(in_flight["max"], in_flight["now"])
        time.sleep(0.004)
        with lock:
            in_flight["now"] -= n
        return torch.zeros(n), torch.zeros(n, n)

    sizes = [30, 50, 20, 70, 10, 40, 60, 25, 35, 45]
    srv = serve.Server(nworkers=4, budget_bytes=100, solve_fn=solve, footprint_fn=lambda n, tol: n)
    stats = srv.run(_fake_requests(sizes))
    assert stats["requests"] == len(sizes)
    assert srv.max_in_flight_bytes <= 100
    assert in_flight["max"] <= 100
    res = srv.results
    assert [r.rid for r in res] == list(range(len(sizes)))
    for r in res:
        assert r.admitted >= r.arrival - 1e-6 and r.done >= r.admitted
    assert stats["p50_s"] <= stats["p99_s"]


def test_oversized_request_is_rejected():
    srv = serve.Server(nworkers=1, budget_bytes=10, solve_fn=lambda k, A, tol: (None, None),
                       footprint_fn=lambda n, tol: n)
    with pytest.raises(ValueError):
        srv.run(_fake_requests([5, 11]))


def test_poisson_stream_is_seeded():
    a = serve.poisson_stream(20, 100.0, 64, 256, seed=5)
    b = serve.poisson_stream(20, 100.0, 64, 256, seed=5)
    assert [r.A.shape[0] for r in a] == [r.A.shape[0] for r in b]
    assert all(64 <= r.A.shape[0] <= 256 for r in a)
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    assert torch.equal(a[3].A, b[3].A) and torch.equal(a[3].A, a[3].A.t())


def test_autotune_choice_rules():
    """choose_nb scales each candidate's time by the cube of the padded order
    it needs, so a size just above a multiple of a large nb takes a smaller
    one; without a table the rule applies."""
    from evd4sc2025_b200 import autotune
    table = {"b": 32, "entries": [
        {"n": 1024, "nb": 1024, "ms": {"32": 30.0, "256": 12.0, "1024": 10.0}},
        {"n": 4096, "nb": 256, "ms": {"32": 200.0, "256": 80.0, "1024": 90.0}}]}
    assert autotune.choose_nb(1000, table) == 1024
    assert autotune.choose_nb(1030, table) == 256   # nb 1024 would pad to 2048
    assert autotune.choose_nb(4096, table) == 256
    assert autotune.choose_nb(1, table) in (32, 256, 1024)
    assert autotune.choose_nb(500, {"entries": []}) is None
    # the rule's choice stands unless the table beats it by more than 5 %
    assert autotune.choose_nb(1024, table, default_nb=256) == 1024  # 10 vs 12: tuned wins
    assert autotune.choose_nb(4096, table, default_nb=1024) == 256  # 80 vs 90: tuned wins
    assert autotune.choose_nb(4096, table, default_nb=64) == 64     # no time for 64: rule
    near = {"entries": [{"n": 512, "nb": 256, "ms": {"256": 10.0, "512": 10.3}}]}
    assert autotune.choose_nb(512, near, default_nb=512) == 512     # within 5 %: rule
    assert autotune.padded_order(1, 32) == 64 and autotune.padded_order(1030, 256) == 1280
    sizes = autotune.default_sizes(64, 8192, 3)
    assert sizes[0] == 64 and sizes[-1] == 8192 and len(sizes) == 22


def test_solve_shape_is_a_valid_padding():
    for n in (1, 63, 64, 65, 1000, 1056, 3000, 8192):
        np_, nb = serve.solve_shape(n)
        assert np_ >= n and np_ % nb == 0 and (nb // 32) & (nb // 32 - 1) == 0


def test_autotune_active_table_switch():
    from evd4sc2025_b200 import autotune
    t = {"entries": [{"n": 512, "nb": 64, "ms": {"64": 1.0, "512": 2.0}}]}
    try:
        autotune.use_table(t)
        assert autotune.choose_nb(512) == 64 and serve.solve_shape(512) == (512, 64)
        autotune.use_table(None)
        assert autotune.choose_nb(512) is None and serve.solve_shape(512) == serve.padded_shape(512)
    finally:
        autotune._cached = autotune._cached_path = None


def test_server_runs_twice():
    """A server can serve a second stream after the first (warm-up, then the
    measured stream); results and statistics are per run."""
    srv = serve.Server(nworkers=2, budget_bytes=100, solve_fn=lambda k, A, tol: (A, A),
                       footprint_fn=lambda n, tol: n)
    first = srv.run(_fake_requests([3, 4, 5], gap=0.0))
    assert first["requests"] == 3
    second = srv.run(_fake_requests([6, 7], gap=0.0))
    assert second["requests"] == 2 and len(srv.results) == 2


def test_failed_solve_returns_its_memory():
    """A request whose solve raises is reported as failed and gives its memory
    back, so the requests behind it are still admitted and served."""
    def solve(k, A, tol):
        if A.shape[0] == 5:
            raise RuntimeError("bad input")
        return A, A
    srv = serve.Server(nworkers=1, budget_bytes=6, solve_fn=solve, footprint_fn=lambda n, tol: n)
    stats = srv.run(_fake_requests([5, 6, 4, 6], gap=0.0))
    assert stats["requests"] == 4 and stats["failed"] == 1
    bad = [r for r in srv.results if r.error is not None]
    assert len(bad) == 1 and bad[0].n == 5 and "bad input" in bad[0].error


def test_shipped_tuning_table_is_consistent():
    """The measured B200 table: every entry times every candidate nb that fits
    its order, its best nb is the fastest one, and every order 1..65536 gets a
    valid (n', nb) from solve_shape."""
    import math

    from evd4sc2025_b200 import autotune
    table = autotune.load(autotune.DEFAULT_TABLE)
    assert table and table["b"] == 32 and len(table["entries"]) >= 10
    for e in table["entries"]:
        ms = {int(k): v for k, v in e["ms"].items()}
        assert set(ms) == set(autotune._candidates(e["n"]))
        assert all(v > 0 and math.isfinite(v) for v in ms.values())
        assert e["nb"] == min(ms, key=ms.get)
    for n in list(range(1, 300)) + [1000, 1023, 1025, 4095, 5152, 8191, 16384, 40000, 65536]:
        np_, nb = serve.solve_shape(n)
        assert np_ >= max(n, 64) and np_ % nb == 0 and 32 <= nb <= 1024
        assert (nb // 32) & (nb // 32 - 1) == 0
