"""ctypes binding of ``libevd_b200.so`` (the C ABI declared in include/evd_b200.h).

The library is the product: there is no fallback.  If the shared library is
missing, :func:`lib` raises with the build command instead of silently doing
the work another way.
"""
from __future__ import annotations

import ctypes as C
import pathlib

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libevd_b200.so"

_p = C.c_void_p
_l = C.c_long
_d = C.c_double
_i = C.c_int
_c = C.c_char

# name -> (restype, argtypes); mirrors include/evd_b200.h one to one.
SIGNATURES = {
    "evd_status_string": (C.c_char_p, [_i]),
    "evd_version": (C.c_char_p, []),
    "evd_launch_count": (_l, []),
    "evd_fp64_peak_probe": (_i, [_p, _p]),
    "evd_dgemm": (_i, [_c, _c, _l, _l, _l, _d, _p, _l, _p, _l, _d, _p, _l, _p]),
    "evd_dgemm_strided_batched": (_i, [_c, _c, _l, _l, _l, _d, _p, _l, _l, _p, _l, _l, _d,
                                       _p, _l, _l, _l, _p]),
    "evd_syr2k_lower_mirror": (_i, [_l, _l, _d, _p, _l, _p, _l, _d, _p, _l, _l, _p]),
    "evd_panel_qr_work_size": (_l, [_l, _l]),
    "evd_tsqr": (_i, [_l, _l, _p, _l, _p, _l, _p, _l, _p]),
    "evd_panel_qr": (_i, [_l, _l, _p, _l, _p, _l, _p, _l, _p, _l, _p]),
    "evd_sy2sb_work_size": (_l, [_l, _l, _l]),
    "evd_sy2sb": (_i, [_l, _l, _l, _l, _p, _l, _p, _l, _p, _l, _p, _l, _p, _l, _p, _l, _p,
                       _l, _p]),
    "evd_band_pack": (_i, [_l, _l, _p, _l, _p, _l, _p]),
    "evd_bulge_chase_iwork_size": (_l, [_l]),
    "evd_bulge_chase": (_i, [_l, _l, _p, _l, _p, _l, _p, _p, _p, _p]),
    "evd_bulge_chase_noalloc": (_i, [_l, _l, _p, _l, _p, _l, _p, _p, _p]),
    "evd_stedc_work_size": (_l, [_l]),
    "evd_stedc_iwork_size": (_l, [_l]),
    "evd_stedc": (_i, [_l, _p, _p, _p, _l, _p, _l, _p, _l, _p]),
    "evd_bc_back": (_i, [_p, _l, _p, _l, _l, _i, _p]),
    "evd_bc_back_work_size": (_l, [_l]),
    "evd_bc_back_apply": (_i, [_l, _l, _p, _l, _p, _l, _i, _p, _l, _p]),
    "evd_wy_from_slide": (_i, [_l, _l, _l, _p, _l, _p, _l, _p, _p]),
    "evd_q_from_wy": (_i, [_l, _l, _p, _l, _p, _l, _p, _l, _p]),
    "evd_sbr_back_work_size": (_l, [_l, _l, _l]),
    "evd_sbr_back": (_i, [_l, _l, _l, _p, _l, _p, _l, _p, _l, _l, _p, _l, _p]),
    "evd_check_orthogonality": (_i, [_l, _l, _p, _l, _p, _l, _p, _p, _p]),
    "evd_check_eig": (_i, [_l, _p, _l, _p, _p, _l, _p, _p, _p]),
    "evd_syevd_work_size": (_l, [_l, _l, _l]),
    "evd_syevd_last_timings": (None, [_p]),
    "evd_stebz_work_size": (_l, [_l]),
    "evd_stebz": (_i, [_l, _p, _p, _p, _p, _l, _p]),
    "evd_syevd_values": (_i, [_l, _l, _l, _p, _l, _p, _p, _l, _i, _p]),
    "evd_syevd": (_i, [_l, _l, _l, _p, _l, _p, _p, _l, _p, _l, _i, _p]),
    "evd_syevd_mixed_work_size": (_l, [_l, _l, _l, _i, _i]),
    "evd_syevd_s_work_size": (_l, [_l, _l, _l]),
    "evd_syevd_s": (_i, [_l, _l, _l, _p, _l, _p, _p, _l, _p, _l, _p]),
    "evd_syevd_mixed_work_size_min": (_l, [_l, _l, _l, _i, _i]),
    "evd_syevd_mixed": (_i, [_l, _l, _l, _p, _l, _p, _p, _l, _i, _i, _i, _p, _l, _i, _p]),
    "evd_syevd_last_refine_ms": (_d, []),
    "evd_syevd_mixed_last_timings": (None, [_p]),
    "evd_syevd_batched_work_size": (_l, [_l, _p, _i]),
    "evd_syevd_batched": (_i, [_l, _p, _p, _p, _p, _p, _p, _i, _p, _l, _p]),
    "evd_refine_syev_work_size": (_l, [_l]),
    "evd_refine_syev": (_i, [_l, _p, _l, _p, _p, _l, _i, _p, _l, _p]),
    "evd_refine_syev_ozaki_work_size": (_l, [_l, _i]),
    "evd_refine_syev_ozaki": (_i, [_l, _p, _l, _p, _p, _l, _i, _i, _i, _p, _l, _p]),
    "evd_dgemm_ozaki_work_size": (_l, [_c, _c, _l, _l, _l, _i]),
    "evd_dgemm_ozaki": (_i, [_c, _c, _l, _l, _l, _d, _p, _l, _p, _l, _d, _p, _l, _i, _p, _l, _p]),
    "evd_ozaki_bits": (_i, [_i, _l]),
    "evd_panel_qr_lp_work_size": (_l, [_l, _l]),
    "evd_panel_qr_s": (_i, [_l, _l, _p, _l, _p, _l, _p, _l, _p, _l, _p]),
    "evd_panel_qr_h": (_i, [_l, _l, _p, _l, _p, _l, _p, _l, _p, _l, _p]),
    "evd_tsqr_s": (_i, [_l, _l, _p, _l, _p, _l, _p, _l, _p]),
    "evd_tsqr_h": (_i, [_l, _l, _p, _l, _p, _l, _p, _l, _p]),
    "evd_syr2k_lower_s": (_i, [_l, _l, C.c_float, _p, _l, _p, _l, C.c_float, _p, _l, _l, _p]),
    "evd_tc_syr2k": (_i, [_l, _l, C.c_float, _p, _l, _p, _l, C.c_float, _p, _l, _p, _l, _p]),
    "evd_syr2k_lower_h": (_i, [_l, _l, C.c_float, _p, _l, _p, _l, C.c_float, _p, _l, _l, _p]),
    "evd_write_matrix_bin": (_i, [C.c_char_p, _i, _l, _l, _p, _l]),
    "evd_matrix_bin_count": (_l, [C.c_char_p]),
    "evd_matrix_bin_shape": (_i, [C.c_char_p, _l, C.POINTER(_l), C.POINTER(_l)]),
    "evd_read_matrix_bin": (_i, [C.c_char_p, _l, _l, _l, _p, _l]),
    "evd_write_eigenpairs_bin": (_i, [C.c_char_p, _l, _p, _p, _l]),
    "evd_read_eigenpairs_bin": (_i, [C.c_char_p, _l, _p, _p, _l]),
    "evd_write_matrix_csv": (_i, [C.c_char_p, _l, _l, _p, _l]),
    "evd_read_matrix_csv": (_i, [C.c_char_p, C.POINTER(_l), C.POINTER(_l), _p, _l]),
}

_LIB = None


class EvdError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, fn: str, status: int):
        self.status = status
        msg = "?"
        try:
            msg = lib().evd_status_string(status).decode()
        except Exception:  # pragma: no cover - message lookup only
            pass
        super().__init__(f"{fn} failed with status {status} ({msg})")


def lib() -> C.CDLL:
    """Load the shared library once and attach the argument types."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m evd4sc2025_b200.build` "
                "(the CUDA extension is required; there is no CPU fallback)")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _LIB = handle
    return _LIB


def call(name: str, *args) -> int:
    """Call a status-returning entry point; raise EvdError on failure."""
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise EvdError(name, rc)
    return rc
