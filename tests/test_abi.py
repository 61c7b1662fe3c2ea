"""C ABI: the shared library loads and exports every entry point declared in
include/*.h; argument validation and workspace queries work without a GPU."""
import ctypes as C
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(evd_[a-z0-9_]+)\s*\(", text):
            names.append(m.group(1))
    return sorted(set(names))


def test_every_declared_symbol_is_exported(evdlib):
    lib = evdlib.lib()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_header(evdlib):
    from evd4sc2025_b200._native import SIGNATURES
    assert set(declared_functions()) <= set(SIGNATURES)


def test_status_strings_and_version(evdlib):
    lib = evdlib.lib()
    assert lib.evd_status_string(0) == b"success"
    assert b"workspace" in lib.evd_status_string(-5)
    assert lib.evd_version().startswith(b"evd_b200")


def test_workspace_queries(evdlib):
    lib = evdlib.lib()
    assert lib.evd_panel_qr_work_size(16384, 32) > 16384 * 10
    assert lib.evd_panel_qr_work_size(100, 32) == 0      # m % 32 != 0: unsupported
    assert lib.evd_sy2sb_work_size(4096, 32, 1024) > 0
    assert lib.evd_sy2sb_work_size(4096, 16, 1024) == 0  # b must be 32
    assert lib.evd_syevd_work_size(4096, 32, 1024) > 8 * 4096 * 4096 * 5
    # n % nb != 0: padded internally to 4096, workspace holds the padded copies
    assert lib.evd_syevd_work_size(4000, 32, 1024) > lib.evd_syevd_work_size(4096, 32, 1024)
    assert lib.evd_syevd_work_size(4096, 32, 96) == 0    # nb must be 32 * 2^k
    assert lib.evd_syevd_work_size(0, 32, 64) == 0
    assert lib.evd_stedc_work_size(1000) > 1000 * 1000
    assert lib.evd_bulge_chase_iwork_size(1000) >= 4 * 1000


@pytest.mark.parametrize("call,args", [
    ("evd_sy2sb", (96, 96, 32, 64) + (None, 96) * 6 + (None, 0, None)),          # M % nb != 0
    ("evd_sy2sb", (128, 128, 16, 64) + (None, 128) * 6 + (None, 0, None)),        # b != 32
    ("evd_bulge_chase", (100, 16, None, 64, None, 100, None, None, None, None)),
    ("evd_panel_qr", (100, 32, None, 100, None, 100, None, 32, None, 0, None)),
    ("evd_tsqr", (64, 16, None, 64, None, 32, None, 0, None)),
    ("evd_bc_back", (None, 10, None, 10, 10, 16, None)),
    ("evd_syevd", (1000, 32, 1024, None, 1000, None, None, 1000, None, 0, 0, None)),
    ("evd_dgemm", (b"n", b"n", 10, 10, 10, 1.0, None, 5, None, 10, 0.0, None, 10, None)),
    ("evd_syevd_values", (1000, 32, 1024, None, 1000, None, None, 0, 0, None)),
    ("evd_refine_syev", (10, None, 10, None, None, 10, 2, None, 0, None)),
    ("evd_refine_syev", (70000, 256, 70000, 256, 256, 70000, 1, 256, 1 << 40, None)),
    ("evd_tc_syr2k", (10, 4, 1.0, 256, 5, 256, 10, 0.0, 256, 10, None, 0, None)),   # lda < n
    ("evd_syr2k_lower_s", (10, 4, 1.0, 256, 10, 256, 10, 0.0, 256, 5, 0, None)),    # ldc < n
    ("evd_syr2k_lower_h", (10, 4, 1.0, None, 10, 256, 10, 0.0, 256, 10, 0, None)),  # A missing
    ("evd_panel_qr_s", (100, 32, None, 100, None, 100, None, 32, None, 0, None)),
    ("evd_tsqr_h", (64, 16, None, 64, None, 32, None, 0, None)),
    ("evd_stebz", (-1, None, None, None, None, 100, None)),
    ("evd_write_matrix_bin", (None, 0, 2, 2, None, 2)),
])
def test_invalid_arguments_rejected_without_gpu(evdlib, call, args):
    # every check happens on the host before any CUDA call
    rc = getattr(evdlib.lib(), call)(*args)
    assert rc == -1


def test_oracle_not_imported_by_product():
    src = "\n".join(p.read_text() for p in (ROOT / "evd4sc2025_b200").rglob("*.py"))
    assert "oracle" not in src.replace("no fallback", "")  # the product never touches oracle/


def test_workspace_too_small_reported_without_gpu(evdlib):
    lib = evdlib.lib()
    # non-null placeholders are never dereferenced: the size check comes first
    assert lib.evd_refine_syev(8, 256, 8, 256, 256, 8, 1, 256, 10, None) == -5
    assert lib.evd_refine_syev_work_size(8) > 3 * 64
    assert lib.evd_refine_syev_work_size(70000) == 0
    assert lib.evd_panel_qr_lp_work_size(4096, 32) > 8 * 2 * 4096 * 32
    assert lib.evd_panel_qr_lp_work_size(4096, 16) == 0
    assert lib.evd_panel_qr_s(128, 32, 256, 128, 256, 128, 256, 32, 256, 10, None) == -5


def test_fp32_solve_queries_without_gpu(evdlib):
    lib = evdlib.lib()
    for n, nb in ((1, 64), (100, 64), (4096, 1024)):
        need = lib.evd_syevd_s_work_size(n, 32, nb)
        # FP64 copies of A, X and w on top of the 8-moduli mixed workspace
        assert need >= lib.evd_syevd_mixed_work_size(n, 32, nb, 8, 0) + 16 * n * n + 8 * n
    assert lib.evd_syevd_s_work_size(100, 16, 64) == 0           # b = 32 only
    assert lib.evd_syevd_s_work_size(0, 32, 64) == 0
    assert lib.evd_syevd_s_work_size(100, 32, 96) == 0           # nb = 32 * 2^k
    # argument errors are reported before any device work
    assert lib.evd_syevd_s(100, 32, 64, None, 100, None, None, 100, None, 0, None) == -1
    assert lib.evd_syevd_s(100, 32, 64, 8, 99, 8, 8, 100, 8, 1 << 30, None) == -1


def test_batched_queries_without_gpu(evdlib):
    lib = evdlib.lib()
    n = (C.c_long * 3)(100, 1000, 64)
    assert lib.evd_syevd_batched_work_size(3, n, 2) >= 2 * lib.evd_syevd_work_size(1024, 32, 1024)
    assert lib.evd_syevd_batched_work_size(0, None, 8) > 0
    assert lib.evd_syevd_batched_work_size(3, n, 0) == 0          # nstreams >= 1
    bad = (C.c_long * 2)(10, 0)
    assert lib.evd_syevd_batched_work_size(2, bad, 2) == 0        # order 0
    assert lib.evd_syevd_batched(2, bad, None, None, None, None, None, 2, None, 0, None) == -1
