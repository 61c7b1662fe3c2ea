"""The C++ shims with the reference's signatures compile against the headers
(every template specialisation the reference instantiates, host compile only:
no GPU needed)."""
import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]

USAGE = r'''
#include "evd_b200_compat.hpp"

void use_all(cublasHandle_t h, cusolverDnHandle_t s, double* d, float* f, __half* hp, int* info) {
  my_ZY_ZY_SBR_Vector<double>(s, h, 4096, 4096, 32, 1024, d, 4096, d, 4096, d, 4096, d, 4096, d,
                              4096, d, 4096, d, info);
  panelQR<double>(s, h, 4096, 32, d, 4096, d, 4096, d, 32, d, info);
  panelQR<float>(s, h, 4096, 32, f, 4096, f, 4096, f, 32, f, info);
  panelQR<__half>(s, h, 4096, 32, hp, 4096, hp, 4096, hp, 32, hp, info);
  hou_tsqr_panel<double, 128, 32>(h, 4096, 32, d, 4096, d, 32, d);
  hou_tsqr_panel<float, 128, 32>(h, 4096, 32, f, 4096, f, 32, f);
  hou_tsqr_panel<__half, 128, 32>(h, 4096, 32, hp, 4096, hp, 32, hp);
  tc_ozimmu_syr2k<double>(h, 1024, 256, -1.0, d, 1024, d, 1024, 1.0, d, 1024, 256);
  tc_ozimmu_syr2k<float>(h, 1024, 256, -1.0f, f, 1024, f, 1024, 1.0f, f, 1024, 256);
  tc_ozimmu_syr2k<__half>(h, 1024, 256, __float2half(-1.0f), hp, 1024, hp, 1024,
                          __float2half(1.0f), hp, 1024, 256);
  tc_syr2k(h, 1024, 256, -1.0f, f, 1024, f, 1024, 1.0f, f, 1024, hp, 256);
  (void)my_BC_back_trans_v8_10_noBandU(d, 4096, d, 4096, 4096, 32);
  computerWYFromSlide(h, 4096, 1024, 32, d, 4096, d, 4096, d);
  computerQFromWY(h, 4096, 1024, d, 4096, d, 4096, d, 4096);
  checkOrthogonality(h, 4096, 4096, d, 4096, d, 4096, d);
}
'''


def test_compat_shims_compile(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not pathlib.Path(nvcc).exists():
        pytest.fail("nvcc is required to build this project")
    src = tmp_path / "use.cu"
    src.write_text(USAGE)
    r = subprocess.run([nvcc, "-std=c++17", "-c", "-I", str(ROOT / "include"), str(src), "-o",
                        str(tmp_path / "use.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
