"""ctypes view of include/cspb.h and the loader of libcspb.so.

The library is loaded from this package's directory only (it is built in-tree by ``python -m cospanmdao_b200.build``).
There is no fallback: if the library is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcspb.so"

# status codes (include/cspb.h)
OK = 0
ERR_ARGUMENT = 1
ERR_WORKSPACE = 2
ERR_LAUNCH = 3
ERR_TIMEOUT = 4
ERR_NEGATIVE = 5
ERR_EXCEEDS32 = 6
ERR_UNSUPPORTED = 7
ERR_CUDA = 8
ERR_CAPACITY = 9
ERR_TOO_LARGE = 10

DEV_TIMEOUT = 1
DEV_NEGATIVE = 2
DEV_EXCEEDS32 = 4
DEV_CAPACITY = 8
DEV_ARGUMENT = 16

# the flag word of a ragged-column build (total_flag[1])
COLUMN_NEGATIVE = 1
COLUMN_EXCEEDS32 = 2
COLUMN_TIMEOUT = 4

F32 = 0
BF16 = 1
GEMVER_PANEL = 1
GEMVER_BULK = 2
GEMVER_LOWRANK = 4
BATCH_LOWRANK = 1 << 16
BATCH_NO_B = 1 << 17
NS_REFERENCE_ROUNDING = 1
I32, U32, I64, U64 = 0, 1, 2, 3

vp = C.c_void_p
fp = C.c_void_p  # float* / const void* as raw addresses
i64 = C.c_int64
i32 = C.c_int32
u32 = C.c_uint32
u64 = C.c_uint64
sz = C.c_size_t


class GemverDesc(C.Structure):
    _fields_ = [("n", i64), ("lda", i64), ("ldb", i64), ("a_dtype", i32), ("flags", i32),
                ("A", vp), ("u1", vp), ("v1", vp), ("u2", vp), ("v2", vp), ("y", vp), ("z", vp),
                ("alpha", C.c_float), ("beta", C.c_float), ("B", vp), ("x", vp), ("w", vp),
                ("workspace", vp), ("workspace_bytes", sz)]


class GemverRowsDesc(C.Structure):
    _fields_ = [("n", i64), ("rows", i64), ("lda", i64), ("ldb", i64), ("a_dtype", i32), ("flags", i32),
                ("A", vp), ("u1", vp), ("v1", vp), ("u2", vp), ("v2", vp), ("y", vp), ("z", vp),
                ("alpha", C.c_float), ("beta", C.c_float), ("B", vp), ("x", vp), ("w", vp),
                ("workspace", vp), ("workspace_bytes", sz)]


class NsIncompSlabDesc(C.Structure):
    _fields_ = [("nx", i32), ("rows", i32), ("dtype", i32), ("flags", i32), ("h", C.c_double), ("nu", C.c_double),
                ("u", vp), ("v", vp), ("p", vp), ("up", vp * 3), ("dn", vp * 3), ("ru", vp), ("rv", vp), ("rc", vp),
                ("sums", vp), ("workspace", vp), ("workspace_bytes", sz)]


class BicgkDesc(C.Structure):
    _fields_ = [("n", i64), ("ldb", i64), ("b_dtype", i32), ("flags", i32), ("B", vp), ("p", vp), ("r", vp),
                ("q", vp), ("s", vp), ("workspace", vp), ("workspace_bytes", sz)]


class ChainDesc(C.Structure):
    _fields_ = [("n", i64), ("A0", vp), ("u1a", vp), ("v1a", vp), ("u2a", vp), ("v2a", vp), ("ya", vp), ("za", vp),
                ("u1b", vp), ("v1b", vp), ("u2b", vp), ("v2b", vp), ("alpha", C.c_float), ("beta", C.c_float),
                ("B1", vp), ("x1", vp), ("w1", vp), ("q", vp), ("s", vp), ("B2", vp), ("x2", vp), ("w2", vp),
                ("workspace", vp), ("workspace_bytes", sz)]


class BatchedDesc(C.Structure):
    _fields_ = [("count", i64), ("max_elems", i64), ("max_vec", i64), ("a_dtype", i32), ("tune", i32),
                ("n", vp), ("A", vp), ("u1", vp), ("v1", vp), ("u2", vp), ("v2", vp), ("y", vp), ("z", vp),
                ("alpha", vp), ("beta", vp), ("B", vp), ("x", vp), ("w", vp), ("a_off", vp), ("v_off", vp),
                ("workspace", vp), ("workspace_bytes", sz)]


class GemverTask(C.Structure):
    _fields_ = [("n", i64), ("lda", i64), ("ldb", i64), ("A", vp), ("B", vp), ("u1", vp), ("v1", vp), ("u2", vp),
                ("v2", vp), ("y", vp), ("z", vp), ("x", vp), ("w", vp), ("alpha", C.c_float), ("beta", C.c_float)]


class NsIncompTask(C.Structure):
    _fields_ = [("nx", i32), ("ny", i32), ("h", C.c_double), ("nu", C.c_double), ("u", vp), ("v", vp), ("p", vp),
                ("ru", vp), ("rv", vp), ("rc", vp), ("norms", vp)]


class NsCompDesc(C.Structure):
    _fields_ = [("nx", i32), ("ny", i32), ("limiter", i32), ("walls", i32), ("flags", i32), ("reserved", i32),
                ("U", vp), ("R", vp), ("diag", vp),
                ("det_sq64", vp), ("workspace", vp), ("workspace_bytes", sz)]


class NsCompSlabDesc(C.Structure):
    _fields_ = [("nx", i32), ("rows", i32), ("limiter", i32), ("walls", i32), ("flags", i32), ("edges", i32),
                ("U", vp), ("halo_lo", vp), ("halo_hi", vp), ("R", vp), ("diag", vp), ("det_sq64", vp),
                ("workspace", vp), ("workspace_bytes", sz)]


class NsIncompDesc(C.Structure):
    _fields_ = [("nx", i32), ("ny", i32), ("dtype", i32), ("flags", i32), ("h", C.c_double), ("nu", C.c_double),
                ("u", vp), ("v", vp), ("p", vp), ("ru", vp), ("rv", vp), ("rc", vp), ("norms", vp),
                ("workspace", vp), ("workspace_bytes", sz)]


# name -> (restype, argtypes); every function include/cspb.h declares
PROTOTYPES = {
    "cspb_status_string": (C.c_char_p, [C.c_int]),
    "cspb_version": (C.c_char_p, []),
    "cspb_read_status": (C.c_int, [vp, C.POINTER(u32), vp]),
    "cspb_gemver_workspace_bytes": (sz, [i64]),
    "cspb_gemver_fused": (C.c_int, [C.POINTER(GemverDesc), vp]),
    "cspb_ns_incomp_slab_workspace_bytes": (sz, [i32, i32]),
    "cspb_ns_incomp_slab": (C.c_int, [C.POINTER(NsIncompSlabDesc), vp]),
    "cspb_gemver_rows_workspace_bytes": (sz, [i64, i64]),
    "cspb_gemver_rows_partial": (C.c_int, [C.POINTER(GemverRowsDesc), vp, vp]),
    "cspb_gemver_rows_finish": (C.c_int, [C.POINTER(GemverRowsDesc), vp, vp]),
    "cspb_bicgk_workspace_bytes": (sz, [i64]),
    "cspb_bicgk_fused": (C.c_int, [C.POINTER(BicgkDesc), vp]),
    "cspb_chain_workspace_bytes": (sz, [i64]),
    "cspb_gemver_chain": (C.c_int, [C.POINTER(ChainDesc), vp]),
    "cspb_gemver_batched_workspace_bytes": (sz, [i64, i64, i64]),
    "cspb_gemver_batched": (C.c_int, [C.POINTER(BatchedDesc), vp]),
    "cspb_gemver_batched_tunings": (C.c_int, []),
    "cspb_gemver_tasks": (C.c_int, [vp, i64, i64, i64, i32, i32, vp, sz, vp]),
    "cspb_ns_incomp_tasks_workspace_bytes": (sz, [i64, i64]),
    "cspb_ns_incomp_tasks": (C.c_int, [vp, i64, i64, i32, vp, sz, vp]),
    "cspb_ns_comp_workspace_bytes": (sz, [i32, i32]),
    "cspb_ns_compressible": (C.c_int, [C.POINTER(NsCompDesc), vp]),
    "cspb_ns_comp_slab_workspace_bytes": (sz, [i32, i32]),
    "cspb_ns_comp_slab": (C.c_int, [C.POINTER(NsCompSlabDesc), vp]),
    "cspb_ns_init_cons": (C.c_int, [vp, i32, i32, C.c_float, vp]),
    "cspb_ns_incomp_workspace_bytes": (sz, [i32, i32]),
    "cspb_ns_incompressible": (C.c_int, [C.POINTER(NsIncompDesc), vp]),
    "cspb_scan_workspace_bytes": (sz, [i64]),
    "cspb_exclusive_scan_u32": (C.c_int, [vp, vp, i64, vp, sz, vp]),
    "cspb_exclusive_scan_u64": (C.c_int, [vp, vp, i64, vp, sz, vp]),
    "cspb_build_column": (C.c_int, [vp, i32, i64, i64, i32, vp, vp, vp, vp, sz, vp]),
    "cspb_build_column_static": (C.c_int, [vp, i32, i64, i64, i32, vp, vp, vp, vp]),
    "cspb_build_column64": (C.c_int, [vp, i32, i64, i64, i32, vp, vp, vp, vp, sz, vp]),
    "cspb_fill_hash": (C.c_int, [vp, i32, i64, u64, u32, i32, vp]),
}

_lock = threading.Lock()
_lib = None


class LibraryMissing(RuntimeError):
    pass


def lib() -> C.CDLL:
    """The loaded libcspb.so with every prototype set. Raises LibraryMissing when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise LibraryMissing(f"{LIB_PATH} is not built; run `python -m cospanmdao_b200.build` "
                                 "(there is no non-CUDA fallback)")
        h = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(h, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = h
        return h


def missing_symbols() -> list[str]:
    h = lib()
    return [n for n in PROTOTYPES if not hasattr(h, n)]
