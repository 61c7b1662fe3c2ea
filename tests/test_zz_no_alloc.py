"""The allocation-free bulge chasing entry point (evd_bulge_chase_noalloc).

It exists for callers that cannot allocate device memory where they run the
chase (no cudaMalloc allowed at that point: a fixed memory footprint, or a
host framework that owns the allocator); its scratch is a device array inside
the library.  Checked through the C ABI against the regular entry point
(evd_bulge_chase, caller-provided scratch) on the same band, twice in a row,
so that a second call sees a correctly cleared scratch.  This file runs last
so that an earlier failure elsewhere has already been reported.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _band(n, b, seed, dev, evd):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    A = np.tril(np.triu(0.5 * (G + G.T), -b), b)
    return evd.band_pack(evd.to_cm(torch.from_numpy(A), device=dev), b)


def _run(evd, name, sub, n, b, iwork=None):
    dev = sub.device
    U = evd.zeros_cm(n, n, device=dev)
    d = torch.empty(n, dtype=torch.float64, device=dev)
    e = torch.empty(n, dtype=torch.float64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = [n, b, C.c_void_p(sub.data_ptr()), sub.stride(1), C.c_void_p(U.data_ptr()),
            U.stride(1), C.c_void_p(d.data_ptr()), C.c_void_p(e.data_ptr())]
    if iwork is not None:
        args.append(C.c_void_p(iwork.data_ptr()))
    rc = getattr(evd.lib(), name)(*args, stream)
    assert rc == 0, f"{name} returned {rc}"
    torch.cuda.synchronize()
    return d.cpu().numpy(), e[: n - 1].cpu().numpy(), U.cpu().numpy()


@pytest.mark.parametrize("n", [300, 1500])
def test_noalloc_chase_matches_regular_entry_point(cuda, evdlib, n):
    b = 32
    iw = torch.zeros(evdlib.lib().evd_bulge_chase_iwork_size(n) // 4 + 1, dtype=torch.int32,
                     device=cuda)
    ref = _run(evdlib, "evd_bulge_chase", _band(n, b, n, cuda, evdlib), n, b, iw)
    # two calls in a row: the shared scratch must be cleared between them
    for _ in range(2):
        out = _run(evdlib, "evd_bulge_chase_noalloc", _band(n, b, n, cuda, evdlib), n, b)
        for x, y in zip(out, ref):
            assert np.abs(x - y).max() <= 1e-12 * max(1.0, np.abs(y).max())


def test_noalloc_chase_rejects_oversized_band(cuda, evdlib):
    n = 65537  # above the scratch array's capacity; rejected before any launch
    rc = evdlib.lib().evd_bulge_chase_noalloc(n, 32, None, 64, None, n, None, None, None)
    assert rc == -1
