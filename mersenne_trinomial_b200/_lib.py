"""ctypes binding of libgf2e.so (the C ABI declared in include/gf2e.h).

The shared library is built in-tree by `python -m mersenne_trinomial_b200.build`.
There is no fallback: if the library is missing or fails to load, every
entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libgf2e.so")

GF2E_OK = 0
STATUS = {
    0: "GF2E_OK",
    -1: "GF2E_ERR_INVALID",
    -2: "GF2E_ERR_CUDA",
    -3: "GF2E_ERR_NOMEM",
    -4: "GF2E_ERR_UNSUPPORTED_R",
    -5: "GF2E_ERR_TIMEOUT",
    -6: "GF2E_ERR_OVERFLOW",
    -7: "GF2E_ERR_INTERNAL",
}


class Gf2eError(RuntimeError):
    def __init__(self, status: int, detail: str):
        super().__init__(f"{STATUS.get(status, status)}: {detail}")
        self.status = status
        self.detail = detail


class GcdJob(C.Structure):
    _fields_ = [("a_dev", C.c_void_p), ("abits", C.c_uint64), ("b_dev", C.c_void_p),
                ("bbits", C.c_uint64), ("g_dev", C.c_void_p), ("g_cap_words", C.c_size_t)]


class ScanResult(C.Structure):
    _fields_ = [("s", C.c_uint64), ("status", C.c_int), ("d", C.c_uint64),
                ("mask_words", C.c_uint64), ("rlo", C.c_uint64), ("rhi", C.c_uint64)]


class MulJob(C.Structure):
    _fields_ = [("a_dev", C.c_void_p), ("abits", C.c_uint64), ("b_dev", C.c_void_p),
                ("bbits", C.c_uint64), ("out_dev", C.c_void_p)]


class HgcdStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("nodes", "base_cases", "base_rounds", "fft_products",
                                        "school_products", "division_steps", "probes", "us_base",
                                        "us_products", "us_division", "us_small_gcd",
                                        "base_cycles_serial", "base_cycles_total")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tune(C.Structure):
    _fields_ = [("fft_tile_log", C.c_int), ("fft_cmin", C.c_int), ("fft_taylor_lv", C.c_int),
                ("fft_bfly_lv", C.c_int), ("sieve_strip_log", C.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Sched(C.Structure):
    _fields_ = [("mode", C.c_int), ("q0", C.c_uint64), ("G", C.c_uint64), ("rho", C.c_double),
                ("qcap", C.c_uint64)]


SCHED_MODES = {"doubling": 0, "linear": 1, "opt": 2}

_lib = None
_lock = threading.Lock()

_u64, _i32, _vp, _sz = C.c_uint64, C.c_int, C.c_void_p, C.c_size_t
_P = C.POINTER

# name -> (restype, argtypes); every symbol of include/gf2e.h
SIGNATURES = {
    "gf2e_abi_version": (_i32, []),
    "gf2e_status_string": (C.c_char_p, [_i32]),
    "gf2e_last_error": (C.c_char_p, []),
    "gf2e_stream_sync": (_i32, [_vp]),
    "gf2e_device_alloc": (_i32, [_P(_vp), _sz]),
    "gf2e_device_free": (_i32, [_vp]),
    "gf2e_copy_to_host": (_i32, [_vp, _vp, _sz, _vp]),
    "gf2e_copy_to_device": (_i32, [_vp, _vp, _sz, _vp]),
    "gf2e_sieve_workspace_size": (_i32, [_i32, _P(_sz)]),
    "gf2e_sieve_fill": (_i32, [_vp, _u64, _vp]),
    "gf2e_sieve_run": (_i32, [_u64, _i32, _i32, _u64, _vp, _vp, _sz, _vp]),
    "gf2e_sieve_stats": (_i32, [_vp, _i32, _vp, _vp, _vp]),
    "gf2e_primitive_poly": (_u64, [_i32]),
    "gf2e_trin_square": (_i32, [_vp, _vp, _u64, _u64, _vp]),
    "gf2e_trin_square_batch": (_i32, [_vp, _vp, _sz, _i32, _u64, _vp, C.c_uint32, _vp]),
    "gf2e_trin_frobenius_host": (_i32, [_u64, _vp, _i32, C.c_uint32, _vp, _sz, _vp]),
    "gf2e_trin_squarings_per_pass": (_i32, [_u64, _sz, _i32]),
    "gf2e_trin_set_x": (_i32, [_vp, _sz, _i32, _u64, _vp]),
    "gf2e_trin_set_one": (_i32, [_vp, _sz, _i32, _u64, _vp]),
    "gf2e_trin_reduce": (_i32, [_vp, _u64, _vp, _u64, _u64, _vp]),
    "gf2e_cantor_basis": (_i32, [_vp, _P(_i32)]),
    "gf2e_fft_plan_create": (_i32, [_i32, _P(_vp)]),
    "gf2e_fft_plan_destroy": (_i32, [_vp]),
    "gf2e_fft_plan_m": (_i32, [_vp]),
    "gf2e_fft_fwd": (_i32, [_vp, _vp, _vp]),
    "gf2e_fft_inv": (_i32, [_vp, _vp, _vp]),
    "gf2e_fft_twiddles": (_i32, [_vp, _vp]),
    "gf2e_fft_pack": (_i32, [_vp, _sz, _vp, _sz, _sz, _vp]),
    "gf2e_fft_pointwise": (_i32, [_vp, _vp, _sz, _vp]),
    "gf2e_fft_overlap_add": (_i32, [_vp, _sz, _vp, _sz, _vp]),
    "gf2e_mul_fft_m": (_i32, [_u64, _u64]),
    "gf2e_mul_out_words": (_sz, [_u64, _u64]),
    "gf2e_mul": (_i32, [_vp, _vp, _u64, _vp, _u64, _vp, _vp, _vp, _vp]),
    "gf2e_mul_noalloc": (_i32, [_vp, _u64, _vp, _u64, _vp, _vp]),
    "gf2e_mul_batch_workspace_size": (_i32, [_P(MulJob), _i32, _P(_sz)]),
    "gf2e_mul_batch": (_i32, [_P(MulJob), _i32, _vp, _sz, _vp]),
    "gf2e_gcd_workspace_size": (_i32, [_P(GcdJob), _i32, _P(_sz)]),
    "gf2e_gcd_batch": (_i32, [_P(GcdJob), _i32, _vp, _vp, _sz, _vp]),
    "gf2e_scan": (_i32, [_u64, _vp, _i32, _u64, _u64, _u64, _u64, _i32, _P(ScanResult), _vp,
                         _sz, _vp]),
    "gf2e_resolve_factor": (_i32, [_vp, _sz, _u64, _u64, _P(_u64), _vp, _sz, _P(_sz)]),
    "gf2e_server_create": (_i32, [_sz, _i32, _P(_vp)]),
    "gf2e_server_create_blocked": (_i32, [_sz, _i32, _i32, _P(_vp)]),
    "gf2e_server_destroy": (_i32, [_vp]),
    "gf2e_server_submit": (_i32, [_vp, _u64, _u64, _vp, _i32, _u64, _u64, _u64]),
    "gf2e_server_step": (_i32, [_vp, _i32, _vp]),
    "gf2e_server_status": (_i32, [_vp, _P(_i32), _P(_i32), _P(_i32), _P(_sz)]),
    "gf2e_server_poll": (_i32, [_vp, _vp, _vp, _i32, _P(_i32)]),
    "gf2e_server_pairs": (_i32, [_vp, _P(_u64), _P(_u64)]),
    "gf2e_server_job_lines": (_i32, [_vp, _u64, C.c_char_p, _sz, _P(_sz)]),
    "gf2e_server_release": (_i32, [_vp, _u64]),
    "gf2e_scanner_footprint": (_i32, [_u64, _i32, _P(_sz)]),
    "gf2e_scanner_create": (_i32, [_u64, _i32, _P(_vp)]),
    "gf2e_scanner_footprint_blocked": (_i32, [_u64, _i32, _i32, _P(_sz)]),
    "gf2e_scanner_create_blocked": (_i32, [_u64, _i32, _i32, _P(_vp)]),
    "gf2e_scan_blocked": (_i32, [_u64, _vp, _i32, _u64, _u64, _u64, _u64, _i32, _i32,
                                 _P(ScanResult), _vp, _sz, _vp]),
    "gf2e_scanner_destroy": (_i32, [_vp]),
    "gf2e_scanner_set_schedule": (_i32, [_vp, _P(Sched)]),
    "gf2e_sched_widths": (_i32, [_P(Sched), _i32, _u64, _u64, _u64, _i32, _vp]),
    "gf2e_scan_sched": (_i32, [_u64, _vp, _i32, _u64, _u64, _P(Sched), _u64, _u64, _i32, _i32,
                               _P(ScanResult), _vp, _sz, _vp]),
    "gf2e_scanner_submit": (_i32, [_vp, _vp, _i32, _u64, _u64, _u64, _u64, _u64]),
    "gf2e_scanner_step": (_i32, [_vp, _i32, _vp]),
    "gf2e_scanner_status": (_i32, [_vp, _P(_i32), _P(_i32), _P(_i32), _P(_u64)]),
    "gf2e_scanner_poll": (_i32, [_vp, _P(ScanResult), _vp, _vp, _sz, _i32, _P(_i32)]),
    "gf2e_scanner_frontiers": (_i32, [_vp, _vp, _vp, _vp, _i32, _P(_i32)]),
    "gf2e_scanner_gcd_time": (_i32, [_vp, _P(_u64), _P(C.c_double)]),
    "gf2e_trin_create": (_i32, [_u64, _P(_vp)]),
    "gf2e_trin_destroy": (_i32, [_vp]),
    "gf2e_trin_set_s": (_i32, [_vp, _u64]),
    "gf2e_trin_buffers": (_i32, [_vp, _P(_vp), _P(_vp), _P(_vp), _P(_sz), _P(_i32)]),
    "gf2e_trin_scratch": (_i32, [_vp, _P(_vp), _P(_vp), _P(_vp), _P(_i32)]),
    "gf2e_trin_reset_A": (_i32, [_vp, _vp]),
    "gf2e_trin_reset_acc": (_i32, [_vp, _vp]),
    "gf2e_trin_square_A": (_i32, [_vp, _vp]),
    "gf2e_trin_square_A_k": (_i32, [_vp, _u64, _vp]),
    "gf2e_trin_mul_dev": (_i32, [_vp, _vp, _vp, _vp]),
    "gf2e_trin_reduce_T0": (_i32, [_vp, _vp, _u64, _vp]),
    "gf2e_trin_accumulate": (_i32, [_vp, _vp]),
    "gf2e_gcd_large": (_i32, [_vp, _i32, _vp, _i32, _P(HgcdStats), _vp]),
    "gf2e_fft_plan_passes": (_i32, [_vp, _P(_i32), _P(_i32)]),
    "gf2e_tune_default": (_i32, [_P(Tune)]),
    "gf2e_tune_get": (_i32, [_P(Tune)]),
    "gf2e_tune_set": (_i32, [_P(Tune)]),
    "gf2e_fft_autotune": (_i32, [_i32, _i32, _P(Tune), _P(C.c_double), C.c_char_p, _sz]),
    "gf2e_sieve_autotune": (_i32, [_u64, _i32, _u64, _i32, _P(Tune), _P(C.c_double),
                                   C.c_char_p, _sz]),
    "gf2e_scan_choose_block": (_i32, [C.c_double, C.c_double, _P(_i32)]),
    "gf2e_scan_choose_interval": (_i32, [_u64, _u64, C.c_double, C.c_double, _P(_u64),
                                         _P(_u64), _P(C.c_double)]),
}


def lib():
    """Load libgf2e.so once; raise if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m mersenne_trinomial_b200.build`")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def check(status: int) -> None:
    if status != GF2E_OK:
        detail = lib().gf2e_last_error()
        raise Gf2eError(status, detail.decode() if detail else "")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
