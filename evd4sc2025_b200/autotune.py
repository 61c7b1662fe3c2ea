"""Per-size choice of the block size nb, measured on the device.

The reference fixes b = 32 and nb = 1024 and needs n % nb == 0
(src/EVD/myEVD.cu:251-266, api/zy_zy_sy2sb.cu:51-55).  Here ``evd_syevd``
takes any n (padding to a multiple of nb) and any nb = 32 * 2^k, and the best
nb depends on n: a small nb means more, thinner panels; a large nb means
fewer panel merges in the back transformation but more padding when n is not
a multiple of it.  b stays 32: the chase keeps a 32-row reflector per lane
pair and the panel kernels are built for 32-wide panels.

:func:`tune` times every candidate nb for a list of sizes (device time per
solve with the batched path's concurrent streams, best of ``reps``) and
returns a table; :func:`save` /
:func:`load` keep it as JSON.  :func:`choose_nb` answers for any n from the
nearest tuned size (in log n), scaling each candidate's time by the cube of
the padded order it would need at n, so a size just above a multiple of a
large nb is steered to a smaller one.  The table measured on a B200 ships in
``tuning/nb_b200.json``; without a table the rule of
:func:`evd4sc2025_b200.serve.padded_shape` applies.

Run ``python -m evd4sc2025_b200.autotune --out tuning/nb_b200.json`` on the
target GPU to rebuild it.
"""
from __future__ import annotations

import argparse
import json
import math
import pathlib

CANDIDATES = (32, 64, 128, 256, 512, 1024)
DEFAULT_TABLE = pathlib.Path(__file__).resolve().parent / "tuning" / "nb_b200.json"

_cached: dict | None = None
_cached_path: pathlib.Path | None = None


def padded_order(n: int, nb: int) -> int:
    """Order the solver pads n to for block size nb (as evd_syevd does)."""
    return max(-(-n // nb) * nb, 64)


def default_sizes(lo: int = 64, hi: int = 8192, per_octave: int = 3) -> list[int]:
    k = int(round(math.log2(hi / lo) * per_octave))
    return sorted({int(round(lo * 2 ** (i / per_octave))) for i in range(k + 1)})


def _candidates(n: int) -> list[int]:
    # a block wider than the padded order only adds padding
    return [nb for nb in CANDIDATES if nb <= max(64, padded_order(n, 32))]


def tune(sizes=None, reps: int = 2, device="cuda", seed: int = 5, streams: int = 8,
         log=None) -> dict:
    """Time evd_syevd for every (n, nb candidate) and return the table.

    The figure per candidate is device time per solve with ``streams``
    workers solving 2 * streams copies of one matrix concurrently (the way
    the batched and serving paths run them), best of ``reps`` batches after
    one warm-up batch; ``streams=1`` times solves one at a time."""
    import torch

    from . import F64, empty_cm
    from . import serve

    sizes = list(sizes or default_sizes())
    dev = torch.device(device)
    solvers = [serve.StreamSolver(dev) for _ in range(max(1, streams))]
    count = 2 * len(solvers) if streams > 1 else 1
    entries = []
    for n in sizes:
        g = torch.Generator(device=dev).manual_seed(seed + n)
        G = torch.randn(n, n, generator=g, dtype=F64, device=dev)
        A = empty_cm(n, n, device=dev)
        A.copy_(0.5 * (G + G.t()))
        mats = [A] * count
        times = {}
        for nb in _candidates(n):
            best = float("inf")
            for r in range(reps + 1):  # first batch is a warm-up
                _, ms = serve.syevd_batched(mats, solvers=solvers, nb=nb)
                if r > 0:
                    best = min(best, ms / count)
            times[nb] = best
        nb_best = min(times, key=times.get)
        entries.append({"n": n, "nb": nb_best, "ms": {str(k): v for k, v in times.items()}})
        if log:
            log(f"n={n}: nb={nb_best} " + " ".join(f"{k}:{v:.3f}" for k, v in times.items()))
    for sv in solvers:
        sv.release()
    return {"b": 32, "device": torch.cuda.get_device_name(dev), "streams": streams, "reps": reps,
            "figure": "device ms per solve, concurrent streams", "entries": entries}


def save(table: dict, path) -> None:
    path = pathlib.Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps(table, indent=1) + "\n")


def load(path=None) -> dict | None:
    """The table at ``path`` (default: the shipped B200 table), or None."""
    global _cached, _cached_path
    path = pathlib.Path(path) if path else DEFAULT_TABLE
    if _cached_path == path:
        return _cached
    table = json.loads(path.read_text()) if path.exists() else None
    _cached, _cached_path = table, path
    return table


def use_table(table: dict | None) -> None:
    """Make ``table`` the active one (None: no table, the fixed rule applies)."""
    global _cached, _cached_path
    _cached, _cached_path = table, pathlib.Path("<active>")
    if table is None:
        _cached = {"entries": []}


def active_table() -> dict | None:
    return _cached if _cached_path is not None else load()


def _estimate(ent: dict, n: int, nb: int) -> float | None:
    t = ent["ms"].get(str(nb))
    if t is None:
        return None
    return t * (padded_order(n, nb) / padded_order(ent["n"], nb)) ** 3


def choose_nb(n: int, table: dict | None = None, default_nb: int | None = None,
              margin: float = 0.05) -> int | None:
    """Block size for order n from the table (None without a table).

    With ``default_nb`` (the fixed rule's choice) the tuned candidate replaces
    it only when its estimated time is lower by more than ``margin``: at
    small n the candidates differ by less than run-to-run noise."""
    if n < 1:
        raise ValueError("matrix order must be >= 1")
    table = table if table is not None else active_table()
    if not table or not table.get("entries"):
        return None
    ent = min(table["entries"], key=lambda e: abs(math.log(e["n"]) - math.log(n)))
    best, best_t = None, float("inf")
    for k in ent["ms"]:
        est = _estimate(ent, n, int(k))
        if est < best_t:
            best, best_t = int(k), est
    if default_nb is not None:
        d = _estimate(ent, n, default_nb)
        if d is None or best_t >= (1.0 - margin) * d:
            return default_nb
    return best


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", default=str(DEFAULT_TABLE))
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--streams", type=int, default=8)
    ap.add_argument("--lo", type=int, default=64)
    ap.add_argument("--hi", type=int, default=8192)
    ap.add_argument("--per-octave", type=int, default=3)
    a = ap.parse_args(argv)
    table = tune(default_sizes(a.lo, a.hi, a.per_octave), reps=a.reps, streams=a.streams,
                 log=print)
    save(table, a.out)
    print(f"wrote {a.out}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
