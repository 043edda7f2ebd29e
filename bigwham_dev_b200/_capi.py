"""ctypes binding of the C ABI in include/bigwham_b200.h (libbigwham_b200.so).

The shared library is built in-tree by ``bigwham_dev_b200.build`` (or
``__graft_entry__.build()``).  There is no fallback: if the library is missing
every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libbigwham_b200.so")

BW_OK, BW_ERR_ARG, BW_ERR_STATE, BW_ERR_OOM, BW_ERR_CUDA, BW_ERR_DEVICE, BW_ERR_UNSUPPORTED, BW_ERR_IO = range(8)
BW_FP64, BW_FP32, BW_BF16 = 1, 2, 4
BW_STORE_TRANSPOSE, BW_NO_FINITE_CHECK, BW_PLAN_ONLY, BW_STORE_MATMAT = 16, 32, 64, 128
BW_PERMUTED, BW_TRANSPOSE = 256, 512

STATUS_NAMES = {BW_ERR_ARG: "BW_ERR_ARG", BW_ERR_STATE: "BW_ERR_STATE", BW_ERR_OOM: "BW_ERR_OOM",
                BW_ERR_CUDA: "BW_ERR_CUDA", BW_ERR_DEVICE: "BW_ERR_DEVICE", BW_ERR_UNSUPPORTED: "BW_ERR_UNSUPPORTED",
                BW_ERR_IO: "BW_ERR_IO"}

PRECISIONS = {"fp64": BW_FP64, "fp32": BW_FP32, "bf16": BW_BF16}

# Exported symbols and their signatures: (restype, argtypes)
_P = C.c_void_p
_I64 = C.c_int64
_SIGS = {
    "bw_create": (C.c_int, [C.c_int, _I64, _I64, _P, _P, C.c_int, C.POINTER(_P)]),
    "bw_create_batch": (C.c_int, [C.c_int, C.c_int, _P, _P, _P, _P, C.c_int, C.POINTER(_P)]),
    "bw_batch_offsets": (C.c_int, [_P, C.c_int, _P, _P]),
    "bw_batch_count": (C.c_int, [_P]),
    "bw_set_tuning": (C.c_int, [_P, C.c_char_p, _I64]),
    "bw_set_wait_limit": (C.c_int, [_P, _I64]),
    "bw_test_withhold_chunk": (C.c_int, [_P, C.c_int]),
    "bw_add_full": (C.c_int, [_P, _I64, _I64, _I64, _I64, _P, _I64]),
    "bw_add_lowrank": (C.c_int, [_P, _I64, _I64, _I64, _I64, _I64, _P, _I64, _P, _I64]),
    "bw_add_flat_device": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _I64, _P, _I64]),
    "bw_finalize": (C.c_int, [_P, C.c_int]),
    "bw_matvec": (C.c_int, [_P, _P, _P, C.c_int, _P]),
    "bw_matvec_host": (C.c_int, [_P, _P, _P, C.c_int]),
    "bw_matvec_static_scratch": (C.c_int, [_P, _P, _P, C.c_int, _P]),
    "bw_matmat": (C.c_int, [_P, _P, _I64, _P, _I64, C.c_int, C.c_int, _P]),
    "bw_diagonal": (C.c_int, [_P, _P, C.c_int]),
    "bw_sync": (C.c_int, [_P, _P]),
    "bw_info": (C.c_int, [_P, _P, C.c_int]),
    "bw_algorithmic_bytes": (C.c_int, [_P, C.c_int, _P]),
    "bw_last_error": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "bw_set_device_limit": (C.c_int, [_P, _I64]),
    "bw_plan_export": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P]),
    "bw_plan_split": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _P, _P]),
    "bw_matvec_launches": (C.c_int, [_P, C.c_int, C.c_int, _P]),
    "bw_set_timing": (C.c_int, [_P, C.c_int]),
    "bw_timing_read": (C.c_int, [_P, _P, _P]),
    "bw_timing_read_launches": (C.c_int, [_P, _P, _P]),
    "bw_phase_bytes": (C.c_int, [_P, C.c_int, C.c_int, _P, _P]),
    "bw_plan_tscale": (C.c_int, [_P, C.c_int, _P, _P]),
    "bw_mm_plan_export": (C.c_int, [_P, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P, _P]),
    "bw_plan_gather": (C.c_int, [_P, C.c_int, C.c_int, _P, _P]),
    "bw_file_write": (C.c_int, [C.c_char_p, C.c_int, _I64, _I64, _P, _P, _I64, _P, _P, _I64, _P, _P, _P]),
    "bw_file_write_blocks": (C.c_int, [C.c_char_p, C.c_int, _I64, _I64, _P, _P, _I64, _P, _P, _P, _I64, _P, _P, _P,
                                       _P, _P, _P]),
    "bw_file_info": (C.c_int, [C.c_char_p, _P]),
    "bw_file_read": (C.c_int, [C.c_char_p, C.c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "bw_create_from_file": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.POINTER(_P)]),
    "bw_r0_assemble_fr": (C.c_int, [C.c_int, _I64, _P, C.c_double, C.c_double, _I64, _P, _P, _I64, _P, _I64, _P]),
    "bw_r0_aca": (C.c_int, [C.c_int, _I64, _P, C.c_double, C.c_double, _I64, _P, _P, _I64, C.c_double, C.c_int,
                            _P, _I64, _P, _I64, _P, _P, _P]),
    "bw_s0_fields": (C.c_int, [C.c_int, _I64, _P, _P, C.c_double, C.c_double, _I64, _P, _P, _P, _P]),
    "bw_r0_fields": (C.c_int, [C.c_int, _I64, _P, _P, C.c_double, C.c_double, _I64, _P, _P, _P, _P]),
    "bw_destroy": (C.c_int, [_P]),
    "bw_version": (C.c_char_p, []),
}

_lib = None


class BigWhamError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA backend not built: {LIB_PATH} is missing "
                               f"(run python -m bigwham_dev_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error(h) -> str:
    buf = C.create_string_buffer(1024)
    lib().bw_last_error(h, buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, h=None) -> None:
    if status != BW_OK:
        raise BigWhamError(status, last_error(h))
