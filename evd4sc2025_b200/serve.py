"""Batched uneven-size solves and a continuous-batching serving loop.

Both sit on the solvers of this library (``evd_syevd``, ``evd_syevd_mixed``).
The reference solves one matrix per process (``myEVD n b nb``, src/EVD/myEVD.cu:251-706, n a multiple
of 1024); this layer adds:

* **any n >= 1** through ``evd_syevd`` itself, which pads an order that is
  not a multiple of nb (or below 64) with a diagonal block above the
  spectrum, on the device.  nb comes from the measured table of
  :mod:`evd4sc2025_b200.autotune` (:func:`solve_shape`); without a table it
  is the largest 32 * 2^k dividing n' = 32 * ceil(n / 32) (n' >= 64), at
  most 1024 (:func:`padded_shape`).
* **overlap on the device**: a pool of workers, each with its own CUDA
  stream, one grow-only workspace and padded buffer pair, and a host thread
  (the solver synchronises its own stream a few times per solve; ctypes
  releases the GIL during the call, so the workers' solves overlap on the
  GPU).
* **continuous batching** (:class:`Server`): requests arrive over time; a
  request is admitted when its device footprint fits the memory budget, runs
  as soon as a worker is free, and its memory is returned when it completes,
  so requests that arrive while others are on the GPU are admitted as memory
  frees up.  Latency = completion - arrival; the server reports solves/s and
  p50/p99 latency.

Requests carry an accuracy class (:func:`request_form`): FP64-accurate
requests of order >= ``MIXED_MIN_N`` are solved by the mixed form
(``evd_syevd_mixed``, emulated FP64 products with 14 moduli), FP32-tolerance
requests of that size by the mixed form with 8 moduli (30-bit operands, no
refinement: eigenpairs to about 1e-8), and smaller requests of either class
by the plain FP64 solver, which is faster there.
"""
from __future__ import annotations

import heapq
import math
import threading
import time
from dataclasses import dataclass, field
from typing import Callable

import torch

from . import F64, _cm, _ptr, _stream, autotune, call, empty_cm, lib

MAX_NB = 1024


def padded_shape(n: int) -> tuple[int, int]:
    """(n', nb) for a matrix of order n: n' = 32 * ceil(n/32) (>= 64) and nb
    the largest 32 * 2^k dividing n', at most 1024."""
    if n < 1:
        raise ValueError("matrix order must be >= 1")
    np_ = max(64, 32 * math.ceil(n / 32))
    q = np_ // 32
    nb = 32
    while nb * 2 <= MAX_NB and q % 2 == 0:
        nb *= 2
        q //= 2
    return np_, nb


def solve_shape(n: int) -> tuple[int, int]:
    """(n', nb) the solver uses for order n: nb from the tuned table when one
    is present, else the rule of :func:`padded_shape`; n' the padded order."""
    rule = padded_shape(n)
    nb = autotune.choose_nb(n, default_nb=rule[1])
    if nb is None:
        return rule
    return autotune.padded_order(n, nb), nb


FP64_MODULI = 14   # emulated products with 53-bit operands: FP64-level
FP32_MODULI = 8    # 30-bit operands: the FP32-tolerance class (residual <= 1e-6)
MIXED_MIN_N = 2048  # below it the plain FP64 solver is faster than the mixed form


def request_form(n: int, tol: str = "fp64") -> tuple[str, int]:
    """("plain", 0) or ("mixed", moduli) for a request of order n and
    accuracy class ``tol`` ("fp64": residual <= 1e-13, "fp32": <= 1e-6)."""
    if tol not in ("fp64", "fp32"):
        raise ValueError(f"unknown accuracy class {tol!r}")
    if n < MIXED_MIN_N:
        return "plain", 0
    return "mixed", FP64_MODULI if tol == "fp64" else FP32_MODULI


def work_bytes(n: int, nb: int, tol: str = "fp64") -> int:
    """Workspace bytes of the solve :func:`request_form` picks."""
    form, mod = request_form(n, tol)
    if form == "plain":
        return int(lib().evd_syevd_work_size(n, 32, nb))
    return int(lib().evd_syevd_mixed_work_size(n, 32, nb, mod, 0))


def footprint_bytes(n: int, tol: str = "fp64") -> int:
    """Device bytes one solve of order n holds: workspace (with the padded
    copies when n' > n) + A and X of order n + w."""
    _, nb = solve_shape(n)
    return work_bytes(n, nb, tol) + 2 * n * n * 8 + n * 8


class StreamSolver:
    """One worker: a CUDA stream, one grow-only workspace and one A buffer (a
    smaller problem uses the leading block of the buffer, with its leading
    dimension), so a worker holds at most the footprint of the largest
    problem it has solved.  The solver writes w and X straight into freshly
    allocated result tensors (no copy afterwards)."""

    def __init__(self, device="cuda"):
        self.device = torch.device(device)
        self.stream = torch.cuda.Stream(device=self.device)
        self._ws = None
        self._wsbytes = 0
        self._ld = 0
        self._A = None

    def _ensure(self, n: int, nb: int, tol: str = "fp64"):
        need = work_bytes(n, nb, tol)
        if need <= 0:
            raise ValueError(f"unsupported order {n} (nb {nb})")
        if need > self._wsbytes:
            self._ws = None
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
            self._wsbytes = need
        if n > self._ld:
            self._A = None
            self._A = empty_cm(n, n, device=self.device)
            self._ld = n
        return self._A[:n, :n]

    def release(self):
        """Drop the workspace and buffer (their memory returns to torch)."""
        self._ws = self._A = None
        self._wsbytes = self._ld = 0

    def solve(self, A: torch.Tensor, nb: int | None = None, tol: str = "fp64",
              plain: bool = False):
        """Eigenvalues (ascending, length n) and eigenvectors (n x n,
        column-major) of the symmetric FP64 matrix A on this worker's stream,
        by the form :func:`request_form` picks for the accuracy class ``tol``
        (``plain``: the plain FP64 solver whatever the class).  A may live on
        the host or the device; results are on the device.  The padding runs
        on the device; the solver's own host reads are its only
        synchronisation.  ``nb`` overrides the block size of
        :func:`solve_shape`."""
        n = A.shape[0]
        form, mod = ("plain", 0) if plain else request_form(n, tol)
        if plain:
            tol = "fp64"
            if n >= MIXED_MIN_N:  # work_bytes sizes by the class: ask for the plain size
                need = int(lib().evd_syevd_work_size(n, 32, nb or solve_shape(n)[1]))
                if need > self._wsbytes:
                    self._ws = None
                    self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
                    self._wsbytes = need
        if nb is None:
            _, nb = solve_shape(n)
        # The results belong to the caller's stream; the solve runs on this
        # worker's stream, which first waits for the caller's pending work
        # (A may still be being produced there).  record_stream keeps the
        # caching allocator from handing A, w or X to other work before this
        # stream is done with them.
        caller = torch.cuda.current_stream(self.device)
        w = torch.empty(n, dtype=F64, device=self.device)
        X = empty_cm(n, n, device=self.device)
        self.stream.wait_stream(caller)
        w.record_stream(self.stream)
        X.record_stream(self.stream)
        if A.is_cuda:
            A.record_stream(self.stream)
        with torch.cuda.stream(self.stream):
            Ab = self._ensure(n, nb, tol)
            Ab.copy_(A, non_blocking=True)
            pa, lda = _cm(Ab, "A")
            px, ldx = _cm(X, "X")
            if form == "plain":
                call("evd_syevd", n, 32, nb, pa, lda, _ptr(w), px, ldx, _ptr(self._ws),
                     self._wsbytes, 0, _stream(self.stream))
            else:
                call("evd_syevd_mixed", n, 32, nb, pa, lda, _ptr(w), px, ldx, mod, 0,
                     FP64_MODULI, _ptr(self._ws), self._wsbytes, 0, _stream(self.stream))
        return w, X


def syevd_any(A: torch.Tensor, solver: StreamSolver | None = None):
    """Eigenpairs of a symmetric FP64 matrix of any order (padded as above)."""
    solver = solver or StreamSolver(A.device if A.is_cuda else "cuda")
    w, X = solver.solve(A)
    solver.stream.synchronize()
    return w, X


def syevd_batched(mats: list[torch.Tensor], nstreams: int = 8, device="cuda",
                  solvers: list[StreamSolver] | None = None, nb: int | None = None):
    """Eigenpairs of many symmetric matrices of uneven sizes, solved
    concurrently on ``nstreams`` streams.  Returns a list of (w, X) in input
    order (on the device) and the device time of the whole batch in ms
    (CUDA events: one start event that every stream waits on, one end event
    per stream; the maximum elapsed time)."""
    solvers = solvers or [StreamSolver(device) for _ in range(nstreams)]
    order = sorted(range(len(mats)), key=lambda i: -mats[i].shape[0])  # largest first
    out: list = [None] * len(mats)
    nxt = iter(order)
    lock = threading.Lock()
    errors: list[BaseException] = []
    start = torch.cuda.Event(enable_timing=True)
    start.record(torch.cuda.current_stream(solvers[0].device))
    ends = []

    def worker(sv: StreamSolver):
        sv.stream.wait_event(start)
        try:
            while True:
                with lock:
                    i = next(nxt, None)
                if i is None:
                    break
                out[i] = sv.solve(mats[i], nb)
        except BaseException as e:  # surfaced to the caller below
            errors.append(e)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(sv.stream)
        with lock:
            ends.append(ev)

    threads = [threading.Thread(target=worker, args=(sv,)) for sv in solvers]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    for ev in ends:
        ev.synchronize()
    ms = max(start.elapsed_time(ev) for ev in ends) if ends else 0.0
    return out, ms


def syevd_batched_native(mats: list[torch.Tensor], nstreams: int = 8, device="cuda",
                         stream=None):
    """The same batched solve through the C entry point ``evd_syevd_batched``
    (host threads and streams inside the library, no Python per solve).
    ``mats``: column-major FP64 CUDA matrices.  Returns [(w, X), ...] in input
    order and the device time of the batch in ms."""
    import ctypes as C

    count = len(mats)
    dev = torch.device(device)
    ns = (C.c_long * count)(*[m.shape[0] for m in mats])
    outs = [(torch.empty(m.shape[0], dtype=F64, device=dev), empty_cm(m.shape[0], m.shape[0],
                                                                      device=dev)) for m in mats]
    pa, la, pw, px, lx = [], [], [], [], []
    for m, (w, X) in zip(mats, outs):
        p, ld = _cm(m, "A")
        pa.append(p.value)
        la.append(ld)
        pw.append(w.data_ptr())
        q, ldx = _cm(X, "X")
        px.append(q.value)
        lx.append(ldx)
    nbytes = int(lib().evd_syevd_batched_work_size(count, ns, nstreams))
    if nbytes <= 0:
        raise ValueError("unsupported batch")
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    arr = lambda t, v: (t * count)(*v)  # noqa: E731
    st = stream or torch.cuda.current_stream(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    call("evd_syevd_batched", count, ns, arr(C.c_void_p, pa), arr(C.c_long, la),
         arr(C.c_void_p, pw), arr(C.c_void_p, px), arr(C.c_long, lx), nstreams,
         _ptr(ws), nbytes, _stream(st))
    e1.record(st)
    e1.synchronize()
    return outs, e0.elapsed_time(e1)


# ------------------------------------------------------------------- serving
@dataclass(order=True)
class Request:
    arrival: float                       # seconds from the start of the stream
    rid: int
    A: torch.Tensor = field(compare=False)
    tol: str = field(default="fp64", compare=False)   # "fp64" or "fp32"
    bytes: int = field(default=0, compare=False)


@dataclass
class Result:
    rid: int
    n: int
    arrival: float
    admitted: float
    done: float
    w: torch.Tensor | None
    X: torch.Tensor | None
    error: str | None = None           # set when the solve failed (w, X are None)
    tol: str = "fp64"

    @property
    def latency(self) -> float:
        return self.done - self.arrival


class Server:
    """Continuous-batching request loop over a pool of stream workers.

    ``submit_stream(requests)`` replays requests at their arrival times (seconds
    after start).  A request is admitted when its device footprint fits under
    ``budget_bytes`` next to the requests already admitted, then waits for a
    free worker; its footprint is returned when its solve completes.  Results
    keep the eigenpairs on the host (``to_host``) or the device.

    ``solve_fn(worker_index, A, tol) -> (w, X)`` and ``footprint_fn(n, tol)``
    can be replaced (the tests drive the admission logic without a GPU).
    ``keep(request) -> bool`` selects the requests whose eigenpairs are kept
    in the results (all by default; the others count in the statistics and
    release their memory as soon as they are solved).  The budget
    bounds the sum of the footprints of admitted requests; each worker also
    keeps the buffers of the largest problem it has solved, so the device
    holds at most that sum plus one largest footprint per worker.
    """

    def __init__(self, nworkers: int = 8, budget_bytes: int = 150 * 10**9, device="cuda",
                 solve_fn: Callable | None = None, footprint_fn: Callable | None = None,
                 to_host: bool = True, keep: Callable | None = None):
        self.nworkers = nworkers
        self.budget = budget_bytes
        self.to_host = to_host
        self.keep = keep or (lambda req: True)
        self.footprint_fn = footprint_fn or footprint_bytes
        if solve_fn is None:
            self._solvers = [StreamSolver(device) for _ in range(nworkers)]

            def solve_fn(k, A, tol):
                w, X = self._solvers[k].solve(A, tol=tol)
                if self.to_host:
                    w, X = w.cpu(), X.cpu()  # synchronises the worker's stream
                else:
                    self._solvers[k].stream.synchronize()
                return w, X
        self.solve_fn = solve_fn
        self._cv = threading.Condition()
        self._in_use = 0
        self._ready: list = []          # admitted, waiting for a worker (FIFO by arrival)
        self._results: list[Result] = []
        self._closed = False
        self.max_in_flight_bytes = 0

    def _worker(self, k: int, t0: float):
        while True:
            with self._cv:
                while not self._ready and not self._closed:
                    self._cv.wait()
                if not self._ready:
                    return
                _, _, req, t_adm = heapq.heappop(self._ready)
            err = None
            try:
                w, X = self.solve_fn(k, req.A, req.tol)
            except Exception as e:  # a failed request must still return its memory
                w = X = None
                err = f"{type(e).__name__}: {e}"
            t_done = time.perf_counter() - t0
            if not self.keep(req):
                w = X = None
            with self._cv:
                self._in_use -= req.bytes
                self._results.append(Result(req.rid, req.A.shape[0], req.arrival, t_adm, t_done,
                                            w, X, err, req.tol))
                self._cv.notify_all()

    def run(self, requests: list[Request]) -> dict:
        """Serve the stream; returns throughput and latency statistics.  A
        server can run several streams one after another (the workers keep
        their grown buffers); results and statistics are per run."""
        with self._cv:
            self._closed = False
            self._results = []
            self._ready = []
            self._in_use = 0
            self.max_in_flight_bytes = 0
        reqs = sorted(requests)
        for r in reqs:
            r.bytes = int(self.footprint_fn(r.A.shape[0], r.tol))
            if r.bytes > self.budget:
                raise ValueError(f"request {r.rid} (n={r.A.shape[0]}) needs {r.bytes} bytes, "
                                 f"more than the budget {self.budget}")
        t0 = time.perf_counter()
        workers = [threading.Thread(target=self._worker, args=(k, t0)) for k in range(self.nworkers)]
        for th in workers:
            th.start()
        for r in reqs:
            # replay the arrival time, then wait for memory
            delay = r.arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            with self._cv:
                while self._in_use + r.bytes > self.budget:
                    self._cv.wait()
                self._in_use += r.bytes
                self.max_in_flight_bytes = max(self.max_in_flight_bytes, self._in_use)
                t_adm = time.perf_counter() - t0
                heapq.heappush(self._ready, (r.arrival, r.rid, r, t_adm))
                self._cv.notify_all()
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for th in workers:
            th.join()
        wall = time.perf_counter() - t0
        lat = sorted(res.latency for res in self._results)

        def pct(vals, p):
            if not vals:
                return float("nan")
            return vals[min(len(vals) - 1, int(math.ceil(p / 100.0 * len(vals))) - 1)]
        per_class = {}
        for c in ("fp64", "fp32"):
            lc = sorted(res.latency for res in self._results if res.tol == c)
            if lc:
                per_class[c] = {"requests": len(lc), "p50_s": pct(lc, 50), "p99_s": pct(lc, 99)}
        return {"requests": len(self._results), "wall_s": wall,
                "failed": sum(1 for r in self._results if r.error is not None),
                "solves_per_s": len(self._results) / wall if wall > 0 else float("nan"),
                "p50_s": pct(lat, 50), "p99_s": pct(lat, 99), "per_class": per_class,
                "max_in_flight_bytes": self.max_in_flight_bytes}

    @property
    def results(self) -> list[Result]:
        return sorted(self._results, key=lambda r: r.rid)


def poisson_stream(count: int, rate_per_s: float, n_lo: int, n_hi: int, seed: int = 0,
                   fp64_fraction: float = 0.7) -> list[Request]:
    """Seeded Poisson arrivals; n log-uniform on [n_lo, n_hi]; symmetrised
    Gaussian matrices on the host."""
    g = torch.Generator().manual_seed(seed)
    t = 0.0
    reqs = []
    for i in range(count):
        t += float(-math.log(1.0 - torch.rand(1, generator=g).item()) / rate_per_s)
        u = torch.rand(1, generator=g).item()
        n = int(round(math.exp(math.log(n_lo) + u * (math.log(n_hi) - math.log(n_lo)))))
        G = torch.randn(n, n, generator=g, dtype=F64)
        tol = "fp64" if torch.rand(1, generator=g).item() < fp64_fraction else "fp32"
        reqs.append(Request(t, i, 0.5 * (G + G.t()), tol))
    return reqs
