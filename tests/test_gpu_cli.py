"""The myEVD command line: the reference's positional form, and the
eigenvalues-only and refinement modes."""
import pathlib
import subprocess

import pytest

pytestmark = pytest.mark.gpu

BIN = pathlib.Path(__file__).resolve().parent.parent / "evd4sc2025_b200" / "bin" / "myEVD"


def _run(*args):
    if not BIN.exists():
        pytest.fail(f"{BIN} is missing: build with python -m evd4sc2025_b200.build")
    r = subprocess.run([str(BIN), *map(str, args)], capture_output=True, text=True, timeout=300)
    return r.returncode, r.stdout + r.stderr


def test_usage_without_arguments(evdlib):
    rc, out = _run()
    assert rc == 0 and "Usage" in out  # the reference prints the usage and returns 0


def test_full_solve_prints_stages_and_metrics(cuda, evdlib):
    rc, out = _run(1024, 32, 256, "--dist", "gauss")
    assert rc == 0, out
    for key in ("sy2sb", "Bugle chasing", "DC (device)", "BC back", "SBR back", "total EVD",
                "Orthogonality"):
        assert key in out
    orth = float(out.split("Orthogonality metrix is")[1].split()[0])
    assert orth <= 1e-13


def test_values_mode(cuda, evdlib):
    rc, out = _run(512, 32, 128, "--values")
    assert rc == 0 and "eigenvalues only" in out, out


def test_refine_mode(cuda, evdlib):
    rc, out = _run(512, 32, 128, "--dist", "gauss", "--refine", "1")
    assert rc == 0 and "refinement 1 iteration" in out, out
    res = float(out.split("Residual ||AX - XW||_F / (n ||A||_F) is")[1].split()[0])
    assert res <= 1e-13
