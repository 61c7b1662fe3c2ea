"""Generate golden fixtures from the reference's own GPU build.

Runs on a machine with a B200 (needs oracle/_ref/ref_driver, built by `make -C oracle`
from the reference sources).  For each (n, seed) it writes the seeded
symmetrised Gaussian A = (G + G^T)/2 (numpy default_rng(seed)) to a raw
column-major file, runs the reference pipeline on it (my_ZY_ZY_SBR_Vector ->
chasing kernel -> host dstedc -> my_SBRBack_BCBack -> final Dgemm) and stores,
compressed:
  w   eigenvalues (ascending, from the reference's dstedc)
  d,e the tridiagonal the reference's sy2sb + bulge chasing produced
  X8  the first 8 eigenvector columns of the reference's X = Q^T Z
  resid, orth  the reference result's residual / orthogonality (computed here)

usage: python tests/golden/make_golden.py OUT_DIR [n ...]   (default: every case)
Fixtures are small (n <= 4096; vectors: 8 columns); A itself is regenerated
from the seed.
"""
from __future__ import annotations

import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import algos as O  # noqa: E402

CASES = [(1024, 11), (2048, 12), (4096, 13)]


def main(out_dir: str, only: list[int] | None = None) -> int:
    out = pathlib.Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    drv = ROOT / "oracle" / "_ref" / "ref_driver"
    for n, seed in CASES:
        if only and n not in only:
            continue
        A = O.sym_gaussian(n, seed)
        fin = out / f"A_{n}_{seed}.bin"
        np.asfortranarray(A).T.tofile(fin)  # column-major bytes
        prefix = out / f"ref_{n}_{seed}"
        res = subprocess.run([str(drv), str(n), "32", "1024", str(fin), str(prefix), "1"],
                             capture_output=True, text=True, timeout=600)
        if res.returncode != 0:
            print(res.stdout[-2000:], res.stderr[-2000:])
            return 1
        w = np.fromfile(f"{prefix}_w.bin", dtype=np.float64)
        X = np.fromfile(f"{prefix}_X.bin", dtype=np.float64).reshape(n, n).T
        d = np.fromfile(f"{prefix}_d.bin", dtype=np.float64)
        e = np.fromfile(f"{prefix}_e.bin", dtype=np.float64)
        resid = O.residual(A, w, X)
        orth = O.orthogonality(X)
        np.savez_compressed(out / f"ref_n{n}_s{seed}.npz", w=w, d=d, e=e, X8=X[:, :8],
                            resid=resid, orth=orth, n=n, seed=seed)
        for suffix in ("_w.bin", "_X.bin", "_d.bin", "_e.bin"):
            pathlib.Path(f"{prefix}{suffix}").unlink()
        fin.unlink()
        print(f"n={n} seed={seed} resid={resid:.3e} orth={orth:.3e}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1] if len(sys.argv) > 1 else str(HERE),
                  [int(a) for a in sys.argv[2:]] or None))
