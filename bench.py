#!/usr/bin/env python3
"""Benchmark: seconds per n=16384 FP64 symmetric EVD (all eigenpairs) on B200.

    python bench.py --gpus N --steps K --warmup W [--impl ours|reference] [--n 16384]

One step = one full eigendecomposition (eigenvalues + eigenvectors) of a seeded
symmetrised Gaussian A = (G + G^T)/2, n = 16384, b = 32, nb = 1024 (the plain
FP64 two-stage configuration of the reference's `myEVD 16384 32 1024`).

* value:   device time per EVD with A already resident in HBM (CUDA events on
           the solver stream, W warm-up steps, K timed steps, max over ranks);
           whole-job seconds per EVD = step time / N GPUs (independent replicas).
* e2e:     the same through the public API with HOST buffers: pinned H2D of A,
           the solve, D2H of eigenvalues and eigenvectors, inside the timed
           region.
* Every matrix is 2 GiB (> 126 MB L2), so no L2 flush is needed between steps.
* cpu_baseline: LAPACK dsyevd (scipy/OpenBLAS, all host cores) on a bounded
  sample (n=4096, or 8192 when fast enough), scaled by n^3 to n=16384.
* --impl reference: the reference's own GPU build (oracle/_ref/ref_driver,
  compiled from the reference sources; host dstedc via scipy's OpenBLAS) on
  the same n/b/nb, timed by its own driver; rank 0 only.
Multi-GPU: replicas only (a single EVD is not sharded; no collectives on the
data path).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "s per n=16384 EVD (resid<=1e-13), plain FP64 two-stage"
UNIT = "s/EVD"


# ------------------------------------------------------------------- clocks
class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# -------------------------------------------------------------- CPU baseline
def cpu_baseline(n_target: int) -> dict:
    """LAPACK dsyevd on the host (the oracle's CPU checker), bounded sample."""
    import numpy as np
    import scipy.linalg as sla
    cores = os.cpu_count() or 1
    sample_n, t = None, None
    for n in (4096, 8192):
        rng = np.random.default_rng(0)
        G = rng.standard_normal((n, n))
        A = 0.5 * (G + G.T)
        t0 = time.perf_counter()
        sla.eigh(A, driver="evd", overwrite_a=True, check_finite=False)
        dt = time.perf_counter() - t0
        sample_n, t = n, dt
        if dt * 8 > 25.0:   # the next size would exceed the ~30 s budget
            break
    scale = (n_target / sample_n) ** 3
    return {"value": t * scale, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"LAPACK dsyevd (scipy OpenBLAS, {cores} threads) n={sample_n}: "
                      f"{t:.3f} s, scaled by (n/{sample_n})^3"}


# ------------------------------------------------------------ reference arm
def run_reference(args) -> int:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    drv = ROOT / "oracle" / "_ref" / "ref_driver"
    base = {"metric": METRIC, "unit": UNIT, "impl": "reference", "higher_is_better": False}
    if not drv.exists():
        print(json.dumps({**base, "unavailable": "oracle/_ref/ref_driver not built "
                                                  "(make -C oracle needs the reference sources)"}))
        return 0
    reps = args.warmup + args.steps
    t0 = time.perf_counter()
    res = subprocess.run([str(drv), str(args.n), "32", str(args.nb), "-", "-", str(reps)],
                         capture_output=True, text=True, timeout=3600)
    wall = time.perf_counter() - t0
    recs = []
    for ln in res.stdout.splitlines():
        ln = ln.strip()
        if ln.startswith("{") and ln.endswith("}"):
            try:
                recs.append(json.loads(ln))
            except json.JSONDecodeError:
                pass
    if res.returncode != 0 or len(recs) < reps:
        print(json.dumps({**base, "unavailable": f"reference driver failed rc={res.returncode}: "
                                                  f"{res.stderr.strip()[-200:]}"}))
        return 0
    timed = recs[args.warmup:]
    ms = max(r["total_ms"] for r in timed)
    mean_ms = sum(r["total_ms"] for r in timed) / len(timed)
    value = mean_ms / 1000.0
    stages = {k: round(sum(r[k] for r in timed) / len(timed), 2)
              for k in ("sy2sb_ms", "chase_ms", "dstedc_host_ms", "back_ms", "dc_back_overlap_ms",
                        "final_gemm_ms")}
    cores = os.cpu_count() or 1
    line = {
        **base, "value": value, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mean_ms, "max_ms_per_step": ms, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (reference cuRAND U(0,1], seed 3000, symmetrised)",
        "config": {"workload": f"plain FP64 two-stage EVD n={args.n} b=32 nb={args.nb}",
                   "n": args.n, "b": 32, "nb": args.nb, "parallelism": "replicas"},
        "stages_ms": stages,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": "reference GPU build (sm_100a compile of its sources) with "
                                   "host dstedc (OpenBLAS) overlapped, full n per step"},
        "wall_s": wall,
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ our arm
def run_ours(args) -> int:
    import torch
    import torch.distributed as dist

    import evd4sc2025_b200 as evd

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n, b, nb = args.n, 32, args.nb
    stream = torch.cuda.Stream(device=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    # FP64 DMMA peak of this GPU (roofline denominator): best of three probes,
    # taken before the solver warms the GPU up
    fp64_peak = max(evd.fp64_peak_tflops() for _ in range(3))
    with torch.cuda.stream(stream):
        A, lam_known = _make_input(args.input, n, dev, 1234 + rank)
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()  # the generator's temporaries (QR of an n x n Gaussian)
    with torch.cuda.stream(stream):
        ws = evd.Workspace(n, b, nb, device=dev)
        w = torch.empty(n, dtype=torch.float64, device=dev)
        X = evd.empty_cm(n, n, device=dev)
        launches0 = evd.lib().evd_launch_count()
        evd.syevd(A, b, nb, ws=ws, w=w, X=X, stream=stream)
        launches_per_step = evd.lib().evd_launch_count() - launches0
        for _ in range(max(0, args.warmup - 1)):
            evd.syevd(A, b, nb, ws=ws, w=w, X=X, stream=stream)
        stream.synchronize()

    # ---- device-timed region: A resident ----
    barrier()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local)
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stage_sum = {}
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            evd.syevd(A, b, nb, ws=ws, w=w, X=X, timed=True, stream=stream)
            for k, v in evd.last_timings().items():
                stage_sum[k] = stage_sum.get(k, 0.0) + v
        e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    stages = {k: v / args.steps for k, v in stage_sum.items()}
    # note: timed=True inserts CUDA events between stages only (no sync inside a stage)

    # ---- accuracy of the last result ----
    with torch.cuda.stream(stream):
        resid, orth = evd.check_eig(A, w, X, stream=stream)
    eig_err = None
    if lam_known is not None:  # against the spectrum the input was built from
        eig_err = float((w - lam_known).abs().max() / lam_known.abs().max())

    # ---- e2e through the public API with host buffers ----
    # every step copies its A from pinned host memory and reads w and X back;
    # the copies run on a second stream with double-buffered A, w, X, so the
    # upload of step i+1 and the download of step i overlap the solves
    A_h = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
    A_h.copy_(A.t())  # column-major bytes of A as a row-major (n, n) host array (A symmetric)
    w_h = torch.empty(n, dtype=torch.float64, pin_memory=True)
    X_h = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
    e2e_steps = max(1, min(args.steps, 3))
    A_d = [evd.empty_cm(n, n, device=dev), A]
    w_d = [w, torch.empty(n, dtype=torch.float64, device=dev)]
    X_d = [X, evd.empty_cm(n, n, device=dev)]
    cs = torch.cuda.Stream(device=dev)
    ev = lambda: torch.cuda.Event()  # noqa: E731
    h2d = [ev(), ev()]
    solved = [ev(), ev()]
    d2h = [ev(), ev()]
    barrier()
    torch.cuda.synchronize(dev)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    cs.wait_stream(stream)
    with torch.cuda.stream(cs):
        A_d[0].t().copy_(A_h, non_blocking=True)
        h2d[0].record(cs)
    for i in range(e2e_steps):
        k = i % 2
        stream.wait_event(h2d[k])
        if i >= 2:
            stream.wait_event(d2h[k])  # X_d[k], w_d[k] read back by step i - 2
        if i + 1 < e2e_steps:
            kn = (i + 1) % 2
            with torch.cuda.stream(cs):
                if i >= 1:
                    cs.wait_event(solved[kn])  # A_d[kn] used by step i - 1
                A_d[kn].t().copy_(A_h, non_blocking=True)
                h2d[kn].record(cs)
        evd.syevd(A_d[k], b, nb, ws=ws, w=w_d[k], X=X_d[k], stream=stream)
        solved[k].record(stream)
        with torch.cuda.stream(cs):
            cs.wait_event(solved[k])
            w_h.copy_(w_d[k], non_blocking=True)
            X_h.copy_(X_d[k].t(), non_blocking=True)
            d2h[k].record(cs)
    stream.wait_stream(cs)
    f1.record(stream)
    f1.synchronize()
    e2e_ms = f0.elapsed_time(f1) / e2e_steps
    te = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_ms = float(te.item())

    # ---- roofline of the dominant kernel ----
    flops_total = 16.0 / 3.0 * n ** 3
    stage_flops = {"sy2sb": 4.0 / 3.0 * n ** 3, "bc_back": 2.0 * n ** 3, "sbr_back": 2.0 * n ** 3}
    dom = max(("sy2sb", "bulge_chasing", "tridiagonal_dc", "bc_back", "sbr_back"),
              key=lambda k: stages.get(k, 0.0))
    # the stage-2 back transformation: q2_tbuild_kernel (T factors, <1 % of the
    # stage) then q2_mma_kernel, timed together by the stage events
    bc_ms = stages.get("bc_back", float("nan"))
    achieved = stage_flops["bc_back"] / (bc_ms * 1e-3) / 1e12
    # DRAM bytes of one q2_mma_kernel launch: 34.33e9 measured by ncu at n=8192
    # (dram__bytes_read.sum + dram__bytes_write.sum), growing as n^3 (each of
    # the n/128 strips streams the rows of X below it once)
    traffic = 34.33e9 * (n / 8192.0) ** 3
    roofline = {"kernel": "q2_mma_kernel (stage-2 back transformation on DMMA)",
                "bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak, "traffic": traffic,
                "traffic_source": "ncu capture at n=8192 scaled by (n/8192)^3",
                "algorithmic_flops": stage_flops["bc_back"],
                "peak_source": "FP64 DMMA peak measured live by evd_fp64_peak_probe, best of "
                               "3 before the run (MEASURED_PEAKS.json has no FP64 figure)",
                "dominant_stage": dom,
                "pipeline": {"flops_per_evd": flops_total,
                             "achieved_tflops": flops_total / (ms * 1e-3) / 1e12,
                             "frac": flops_total / (ms * 1e-3) / 1e12 / fp64_peak}}
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    cpu = cpu_baseline(n) if not args.no_cpu else None
    line = {
        "metric": METRIC, "value": ms_max / 1000.0 / world, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": INPUT_DESC[args.input] + " (torch Philox seed 1234+rank)",
        "config": {"workload": f"plain FP64 two-stage EVD n={n} b={b} nb={nb}", "n": n, "b": b,
                   "input": args.input,
                   "nb": nb, "parallelism": f"replicas x{world}",
                   "l2": "inputs 2 GiB > 126 MB L2 (no flush needed)"},
        "stages_ms": {k: round(v, 3) for k, v in stages.items()},
        "accuracy": {"resid": resid, "orth": orth, "resid_ok": resid <= 1e-13,
                     "orth_ok": orth <= 1e-13, "eig_err_vs_known_rel": eig_err},
        "e2e": {"value": e2e_ms / 1000.0 / world, "unit": UNIT,
                "h2d_bytes_per_step": n * n * 8, "d2h_bytes_per_step": n * 8 + n * n * 8,
                "steps": e2e_steps,
                "overlap": "copies on a second stream, double-buffered A/w/X: the upload "
                           "of step i+1 and the download of step i overlap the solves"},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": roofline,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


INPUT_DESC = {
    "gauss": "synthetic: seeded symmetrised Gaussian A=(G+G^T)/2",
    "geometric": "synthetic: A = Q diag(lambda) Q^T, Q Haar (QR of a seeded Gaussian, sign(diag R) "
                 "fixed), |lambda| geometric over [1e-6, 1] with seeded random signs",
    "geometric1e10": "synthetic: A = Q diag(lambda) Q^T, Q Haar, |lambda| geometric over "
                     "[1e-10, 1] with seeded random signs",
    "uniform": "synthetic: A = Q diag(lambda) Q^T, Q Haar, lambda uniform on [-1, 1]",
    "clustered": "synthetic: A = Q diag(lambda) Q^T, Q Haar, 100 clusters of width 1e-10 centred "
                 "on linspace(-1, 1, 100)",
}


def _make_input(kind: str, n: int, dev, seed: int):
    """(A column-major FP64 on dev, known ascending spectrum or None)."""
    import torch

    import evd4sc2025_b200 as evd

    g = torch.Generator(device=dev).manual_seed(seed)
    A = evd.empty_cm(n, n, device=dev)
    if kind == "gauss":
        G = torch.randn(n, n, generator=g, dtype=torch.float64, device=dev)
        A.copy_(0.5 * (G + G.t()))
        return A, None
    if kind in ("geometric", "geometric1e10"):
        decades = 6.0 if kind == "geometric" else 10.0
        mag = 10.0 ** (-decades * torch.arange(n, dtype=torch.float64, device=dev) / max(n - 1, 1))
        sign = torch.where(torch.rand(n, generator=g, dtype=torch.float64, device=dev) < 0.5,
                           -1.0, 1.0)
        lam = mag * sign
    elif kind == "uniform":
        lam = 2.0 * torch.rand(n, generator=g, dtype=torch.float64, device=dev) - 1.0
    elif kind == "clustered":
        per = -(-n // 100)
        centers = torch.linspace(-1.0, 1.0, 100, dtype=torch.float64, device=dev)
        lam = (centers[:, None] + 1e-10 * torch.rand(100, per, generator=g, dtype=torch.float64,
                                                     device=dev)).reshape(-1)[:n]
    else:
        raise ValueError(kind)
    G = torch.randn(n, n, generator=g, dtype=torch.float64, device=dev)
    Q, R = torch.linalg.qr(G)
    Q *= torch.sign(torch.diagonal(R))[None, :]
    del G, R
    M = (Q * lam[None, :]) @ Q.t()
    A.copy_(0.5 * (M + M.t()))
    del M, Q
    return A, torch.sort(lam).values


def _loguniform_sizes(count: int, lo: int, hi: int, seed: int) -> list[int]:
    import torch
    g = torch.Generator().manual_seed(seed)
    u = torch.rand(count, generator=g, dtype=torch.float64)
    return [int(round(math.exp(math.log(lo) + float(x) * (math.log(hi) - math.log(lo)))))
            for x in u]


def run_batched(args) -> int:
    """Batched uneven sizes: solves/s of the concurrent-stream batch vs the plain
    solver looped over the same matrices (both FP64, device-timed)."""
    import torch

    from evd4sc2025_b200 import serve

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    out = []
    for tag, count, lo, hi, seed in (("fp64 batch", args.batch_count, 64, 1024, 7),
                                     ("fp32-tolerance batch", args.batch_count // 8, 256, 2048,
                                      8)):
        sizes = _loguniform_sizes(count, lo, hi, seed)
        mats = []
        for i, n in enumerate(sizes):
            g = torch.Generator(device=dev).manual_seed(1000 * seed + i)
            G = torch.randn(n, n, generator=g, dtype=torch.float64, device=dev)
            mats.append(0.5 * (G + G.t()))
        solvers = [serve.StreamSolver(dev) for _ in range(args.streams)]
        # warm-up: one full pass, so the grow-only workspaces and the caching
        # allocator have reached their size before the timed pass
        serve.syevd_batched(mats, solvers=solvers)
        _, ms = serve.syevd_batched(mats, solvers=solvers)
        one = [serve.StreamSolver(dev)]
        serve.syevd_batched(sorted(mats, key=lambda m: -m.shape[0])[:4], solvers=one)
        _, ms_loop = serve.syevd_batched(mats, solvers=one)
        # the same batch through the C entry point (threads and streams inside
        # the library; nb by the fixed rule); the matrices are symmetric, so
        # the transposed views are their column-major forms
        cms = [m.t() for m in mats]
        serve.syevd_batched_native(cms, nstreams=args.streams)  # warm-up
        _, ms_native = serve.syevd_batched_native(cms, nstreams=args.streams)
        flops = sum(16.0 / 3.0 * n ** 3 for n in sizes)
        out.append({"batch": tag, "matrices": count, "n_range": [lo, hi],
                    "solves_per_s": count / (ms * 1e-3), "ms": ms,
                    "native_c_api_solves_per_s": count / (ms_native * 1e-3),
                    "looped_plain_solves_per_s": count / (ms_loop * 1e-3), "looped_ms": ms_loop,
                    "speedup_vs_loop": ms_loop / ms, "tflops_fp64_equiv": flops / (ms * 1e-3) / 1e12})
    line = {"metric": "batched solves/s (uneven sizes, FP64 accuracy)", "value": out[0]["solves_per_s"],
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic: seeded symmetrised Gaussian, n log-uniform",
            "config": {"workload": "batched uneven sizes", "streams": args.streams,
                       "nb": "fixed rule" if args.nb_rule or not serve.autotune.active_table()
                       or not serve.autotune.active_table().get("entries") else
                       "tuned table " + str(serve.autotune.DEFAULT_TABLE.name)},
            "batches": out}
    print(json.dumps(line))
    return 0


def run_values(args) -> int:
    """Eigenvalues only at the headline size: device time per solve."""
    import torch

    import evd4sc2025_b200 as evd

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    n, nb = args.n, args.nb
    stream = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        g = torch.Generator(device=dev).manual_seed(1234)
        G = torch.randn(n, n, generator=g, dtype=torch.float64, device=dev)
        A = evd.empty_cm(n, n, device=dev)
        A.copy_(0.5 * (G + G.t()))
        del G
        ws = evd.Workspace(n, 32, nb, device=dev)
        w = torch.empty(n, dtype=torch.float64, device=dev)
        for _ in range(args.warmup):
            evd.syevd_values(A, 32, nb, ws=ws, w=w, stream=stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stage_sum = {}
        e0.record(stream)
        for _ in range(args.steps):
            evd.syevd_values(A, 32, nb, ws=ws, w=w, timed=True, stream=stream)
            for k, v in evd.last_timings().items():
                stage_sum[k] = stage_sum.get(k, 0.0) + v
        e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    st = {k: round(v / args.steps, 3) for k, v in stage_sum.items()
          if k in ("sy2sb", "bulge_chasing", "tridiagonal_dc", "total")}
    st["tridiagonal_eigenvalues"] = st.pop("tridiagonal_dc")
    line = {"metric": f"s per n={n} eigenvalues-only solve (FP64)", "value": ms / 1000.0,
            "unit": "s/solve", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": False, "dtype": "f64",
            "data": "synthetic: seeded symmetrised Gaussian",
            "config": {"workload": f"eigenvalues only n={n} b=32 nb={nb}"}, "stages_ms": st}
    print(json.dumps(line))
    return 0


def run_refine(args) -> int:
    """Ogita-Aishima refinement at the headline size: device time per
    iteration, from eigenvectors of the FP64 solve perturbed by 1e-7
    (seeded), and the residual / orthogonality after the iterations."""
    import torch

    import evd4sc2025_b200 as evd

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    n, iters = args.n, 2
    A, _ = _make_input(args.input, n, dev, 1234)
    w, X = evd.syevd(A, 32, args.nb)
    g = torch.Generator(device=dev).manual_seed(99)
    X0 = evd.to_cm(X + 1e-7 * torch.randn(n, n, generator=g, dtype=torch.float64, device=dev),
                   device=dev)
    del X
    torch.cuda.empty_cache()
    Xw = X0.clone()
    evd.refine_syev(A, Xw, 1)  # warm-up
    torch.cuda.synchronize(dev)
    Xr = X0.clone()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    wr, Xr = evd.refine_syev(A, Xr, iters)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / iters
    res, orth = evd.check_eig(A, wr, Xr)
    line = {"metric": f"ms per Ogita-Aishima refinement iteration, n={n} (FP64 DMMA GEMMs)",
            "value": ms, "unit": "ms/iteration", "n_gpus": 1, "higher_is_better": False,
            "dtype": "f64", "data": INPUT_DESC[args.input] + "; start X = FP64 eigenvectors "
            "+ 1e-7 N(0,1) (seed 99)",
            "config": {"workload": f"refinement n={n}", "iterations": iters},
            "tflops": 8.0 * n ** 3 / (ms * 1e-3) / 1e12,
            "accuracy_after": {"resid": res, "orth": orth}}
    print(json.dumps(line))
    return 0


def run_serving(args) -> int:
    """Continuous-batching serving loop on a seeded Poisson stream."""
    import torch

    from evd4sc2025_b200 import serve

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    reqs = serve.poisson_stream(args.requests, args.rate, 128, 8192, seed=2024)
    srv = serve.Server(nworkers=args.streams, budget_bytes=150 * 10**9, device=dev)
    # warm-up (not counted): every worker grows its buffers to the largest
    # order of the stream and every kernel is loaded once
    g = torch.Generator().manual_seed(5)
    warm = []
    for i, n in enumerate([8192] * args.streams + [128, 512, 2048] * 2):
        G = torch.randn(n, n, generator=g, dtype=torch.float64)
        warm.append(serve.Request(0.0, i, 0.5 * (G + G.t())))
    srv.run(warm)
    stats = srv.run(reqs)
    lat = [r.latency for r in srv.results]
    line = {"metric": "serving solves/s with p50/p99 latency (FP64 accuracy)",
            "value": stats["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f64",
            "data": "synthetic: seeded Poisson arrivals, n log-uniform [128, 8192], "
                    "symmetrised Gaussian; every request served in FP64",
            "config": {"workload": "serving loop", "requests": len(reqs),
                       "rate_per_s": args.rate, "workers": args.streams,
                       "hbm_budget_bytes": 150 * 10**9},
            "p50_s": stats["p50_s"], "p99_s": stats["p99_s"], "mean_latency_s": sum(lat) / len(lat),
            "wall_s": stats["wall_s"], "max_in_flight_bytes": stats["max_in_flight_bytes"]}
    print(json.dumps(line))
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--nb", type=int, default=1024)
    ap.add_argument("--input", choices=tuple(INPUT_DESC), default="gauss",
                    help="evd workload input: gauss (default) or a known spectrum")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU LAPACK baseline")
    ap.add_argument("--workload", choices=("evd", "values", "batched", "serving", "refine"),
                    default="evd",
                    help="evd (default): the n=16384 solve; batched / serving: the uneven-size "
                         "batch and the serving loop (one GPU)")
    ap.add_argument("--streams", type=int, default=8, help="worker streams (batched/serving)")
    ap.add_argument("--nb-rule", action="store_true",
                    help="batched/serving: nb by the fixed rule instead of the tuned table")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--requests", type=int, default=1000)
    ap.add_argument("--rate", type=float, default=12.0, help="serving arrivals per second")
    args = ap.parse_args(argv)
    # at least three untimed warm-up solves, whatever was asked for
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.nb_rule:  # batched / serving: the fixed nb rule instead of the tuned table
        from evd4sc2025_b200 import autotune
        autotune.use_table(None)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "refine":
        return run_refine(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "values":
        return run_values(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
