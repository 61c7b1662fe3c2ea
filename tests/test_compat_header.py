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


C_USAGE = r'''
#include <stdio.h>
#include <cuda_runtime.h>
#include "evd_b200.h"

int use_c_api(long n, double* dA, double* dw, double* dX, long count, const long* orders,
              double** A_ptrs, const long* ldas, double** w_ptrs, double** X_ptrs,
              const long* ldXs, cudaStream_t stream) {
  long nb = 256, wbytes = evd_syevd_work_size(n, 32, nb);
  void* work = 0;
  cudaMalloc(&work, wbytes);
  int rc = evd_syevd(n, 32, nb, dA, n, dw, dX, n, work, wbytes, 0, stream);
  if (rc != EVD_SUCCESS) fprintf(stderr, "%s\n", evd_status_string(rc));
  long rn = evd_refine_syev_work_size(n);
  double* rw = 0;
  cudaMalloc((void**)&rw, rn * sizeof(double));
  rc = evd_refine_syev(n, dA, n, dw, dX, n, 2, rw, rn, stream);
  long bw = evd_syevd_batched_work_size(count, orders, 8);
  void* bwork = 0;
  cudaMalloc(&bwork, bw);
  rc = evd_syevd_batched(count, orders, (const double* const*)A_ptrs, ldas, w_ptrs, X_ptrs,
                         ldXs, 8, bwork, bw, stream);
  evd_write_eigenpairs_bin("eig.bin", n, dw, dX, n);
  evd_read_eigenpairs_bin("eig.bin", n, dw, dX, n);
  return rc;
}
'''


def test_c_header_compiles_as_c(tmp_path):
    """include/evd_b200.h is plain C: the usage shown in the integration notes
    compiles with the host C compiler."""
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no host C compiler")
    src = tmp_path / "use.c"
    src.write_text(C_USAGE)
    r = subprocess.run([gcc, "-std=c11", "-Wall", "-Werror", "-c", "-I", str(ROOT / "include"),
                        "-I", "/usr/local/cuda/include", str(src), "-o", str(tmp_path / "use.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
