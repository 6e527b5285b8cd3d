"""ctypes binding of libmsa_b200.so (declared in include/msa_b200.h).

The shared library is the product; this module only declares its C entry
points. Loading fails loudly when the library has not been built: there is no
Python or CPU fallback behind these calls.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libmsa_b200.so"

c_u8p = ctypes.POINTER(ctypes.c_uint8)
c_u16p = ctypes.POINTER(ctypes.c_uint16)
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_i32p = ctypes.POINTER(ctypes.c_int32)

MSA_OK = 0
MSA_ERR_INVALID = 1
MSA_ERR_CUDA = 2
MSA_ERR_NOMEM = 3
MSA_ERR_UNKNOWN_TABLE = 4
MSA_ERR_UNKNOWN_ALGORITHM = 5
MSA_ERR_HANDLE = 6
MSA_ERR_DEVICE_TIMEOUT = 7
MSA_ERR_UNDEFINED = 8
MSA_ERR_NO_DEVICE = 9
MSA_ERR_QUEUE = 10
MSA_ERR_TOO_LARGE = 11

MSA_NW_AUTO = 0
MSA_NW_PLAIN = 1
MSA_NW_PERSISTENT = 2
MSA_NW_VARIANT_INT32 = 1
MSA_NW_VARIANT_NO_PACKED = 2

MSA_TRI_F32_HOST = 0
MSA_TRI_F32_DEVICE = 1
MSA_TRI_I32_HOST = 2
MSA_TRI_I32_DEVICE = 3
MSA_NJ_SYMMETRIC = 0
MSA_NJ_LINEAR = 1

UNIT_END = 0x18
UNIT_GAP = 0x19
UNDEFINED_REF = 0xFFFFFFFF


class MsaTable(ctypes.Structure):
    _fields_ = [("score", ctypes.c_int32 * 625), ("penalty", ctypes.c_int32), ("index", ctypes.c_int32)]


class MsaNwStats(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("total_ms", ctypes.c_double), ("cells", ctypes.c_uint64),
                ("pairs", ctypes.c_uint64), ("launches", ctypes.c_uint32), ("narrow_tasks", ctypes.c_uint32),
                ("graph", ctypes.c_uint32)]


class MsaOtu(ctypes.Structure):
    _fields_ = [("parent", ctypes.c_uint32), ("child", ctypes.c_uint32 * 2), ("distance", ctypes.c_float),
                ("level", ctypes.c_uint32)]


class MsaNjStats(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("total_ms", ctypes.c_double), ("n", ctypes.c_uint32),
                ("cluster", ctypes.c_uint32), ("cycles_scan", ctypes.c_uint64), ("cycles_wait", ctypes.c_uint64),
                ("cycles_join", ctypes.c_uint64), ("cycles_join_wait", ctypes.c_uint64), ("cycles_write", ctypes.c_uint64),
                ("cycles_fold", ctypes.c_uint64), ("cycles_fold_row", ctypes.c_uint64),
                ("cycles_fold_wait", ctypes.c_uint64), ("helper_clusters", ctypes.c_uint32)]


class MsaServeConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_uint64), ("max_jobs", ctypes.c_uint32),
                ("quantum_mcells", ctypes.c_uint32), ("batch_window_us", ctypes.c_uint32),
                ("age_weight_us", ctypes.c_uint32)]


class MsaJobStats(ctypes.Structure):
    _fields_ = [("submit_ms", ctypes.c_double), ("admit_ms", ctypes.c_double), ("done_ms", ctypes.c_double),
                ("cells", ctypes.c_uint64), ("n", ctypes.c_uint32), ("launches", ctypes.c_uint32)]


class MsaOpProbe(ctypes.Structure):
    _fields_ = [("ops_per_clk_sm", ctypes.c_double), ("ms", ctypes.c_double), ("lane_ops", ctypes.c_uint64),
                ("sm_clock_mhz", ctypes.c_double)]


class MsaError(RuntimeError):
    """A non-zero msa_status from the library."""

    def __init__(self, status: int, detail: str = ""):
        self.status = status
        msg = lib().msa_strerror(status).decode()
        super().__init__(f"{msg}: {detail}" if detail else msg)


# (name, restype, argtypes); every declaration of include/msa_b200.h.
_PROTOS = [
    ("msa_strerror", ctypes.c_char_p, [ctypes.c_int]),
    ("msa_table_make", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(MsaTable)]),
    ("msa_table_has", ctypes.c_int, [ctypes.c_char_p]),
    ("msa_table_list", ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int]),
    ("msa_encode", ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint64, c_u8p]),
    ("msa_decode", ctypes.c_int, [c_u8p, ctypes.c_uint64, ctypes.c_char_p]),
    ("msa_encode_blocks", ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint64, c_u16p]),
    ("msa_unpack_blocks", ctypes.c_int, [c_u16p, ctypes.c_uint64, c_u8p]),
    ("msa_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("msa_destroy", None, [ctypes.c_void_p]),
    ("msa_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("msa_set_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("msa_get_stream", ctypes.c_void_p, [ctypes.c_void_p]),
    ("msa_launch_count", ctypes.c_uint64, [ctypes.c_void_p]),
    ("msa_seqs_upload", ctypes.c_int, [ctypes.c_void_p, c_u8p, c_u64p, c_u64p, ctypes.c_uint32,
                                       ctypes.POINTER(ctypes.c_uint64)]),
    ("msa_seqs_release", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    ("msa_seqs_count", ctypes.c_int64, [ctypes.c_void_p, ctypes.c_uint64]),
    ("msa_nw_all_pairs", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(MsaTable), ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_int]),
    ("msa_nw_all_pairs_part", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(MsaTable), ctypes.c_int,
                                             ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int]),
    ("msa_nw_part_of_pairs", ctypes.c_int, [ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64),
                                            ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint32, ctypes.POINTER(MsaTable),
                                            ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]),
    ("msa_nw_set_tiles", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    ("msa_nw_set_variant", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32]),
    ("msa_seqs_load_fasta", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_uint32,
                                           ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint32)]),
    ("msa_seqs_description", ctypes.c_char_p, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32]),
    ("msa_fasta_count", ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.c_uint32,
                                       ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)]),
    ("msa_fasta_encode", ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.c_uint32,
                                        ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64),
                                        ctypes.POINTER(ctypes.c_uint64)]),
    ("msa_nw_all_pairs_noalloc", ctypes.c_int, [ctypes.c_void_p, c_u64p, c_u64p, ctypes.c_uint32,
                                                ctypes.POINTER(MsaTable), ctypes.c_void_p, ctypes.c_void_p]),
    ("msa_noalloc_last_error", ctypes.c_char_p, []),
    ("msa_nw_last_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(MsaNwStats)]),
    ("msa_nj", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32,
                              ctypes.POINTER(MsaOtu)]),
    ("msa_nj_order", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_int,
                                    ctypes.POINTER(MsaOtu)]),
    ("msa_nj_last_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(MsaNjStats)]),
    ("msa_nj_set_clusters", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.c_int]),
    ("msa_probe_op", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(MsaOpProbe)]),
    ("msa_serve_start", ctypes.c_int, [ctypes.POINTER(MsaServeConfig), ctypes.POINTER(ctypes.c_void_p)]),
    ("msa_serve_submit", ctypes.c_int, [ctypes.c_void_p, c_u8p, c_u64p, c_u64p, ctypes.c_uint32,
                                        ctypes.POINTER(MsaTable), ctypes.POINTER(ctypes.c_uint64)]),
    ("msa_serve_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.POINTER(MsaJobStats)]),
    ("msa_serve_stop", ctypes.c_int, [ctypes.c_void_p]),
]

EXPORTED = [p[0] for p in _PROTOS]

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library; raises if it is missing (build it with msa_b200.build)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m msa_b200.build`")
        handle = ctypes.CDLL(str(LIB_PATH), mode=os.RTLD_NOW)
        for name, res, args in _PROTOS:
            fn = getattr(handle, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int, ctx=None) -> None:
    if status != MSA_OK:
        detail = ""
        if ctx:
            detail = (lib().msa_last_error(ctx) or b"").decode()
        raise MsaError(status, detail)
