"""ctypes binding of libtspg.so (the C ABI declared in include/tspg.h).

The shared library is built in-tree (``trident_b200/libtspg.so``) by
``__graft_entry__.build()`` or ``make -C trident_b200/csrc``.  There is no
fallback: importing this module without the library raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtspg.so")

TSPG_OK, TSPG_EINVAL, TSPG_ENOMEM, TSPG_EOVERFLOW, TSPG_ETIMEOUT, TSPG_ECUDA, TSPG_EUNSORTED, TSPG_ESCRATCH = range(8)
TSPG_PACK_NOALLOC_MAX_SEGMENTS = 262144
TSPG_ROWS, TSPG_COLS = 0, 1
TSPG_F_B_SORTED = 1
TSPG_F_ACC_FUSE, TSPG_F_ACC_SPLIT = 2, 4


class TspgCsr(C.Structure):
    _fields_ = [
        ("nrows", C.c_int64),
        ("ncols", C.c_int64),
        ("nnz", C.c_int64),
        ("rowptr", C.c_void_p),
        ("rowptr_bits", C.c_int32),
        ("val_bits", C.c_int32),
        ("col", C.c_void_p),
        ("val", C.c_void_p),
    ]


ALLOC_FN = C.CFUNCTYPE(C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)


class TspgCsrOut(C.Structure):
    _fields_ = [
        ("nrows", C.c_int64),
        ("ncols", C.c_int64),
        ("nnz", C.c_int64),
        ("rowptr", C.c_void_p),
        ("rowptr_bits", C.c_int32),
        ("val_bits", C.c_int32),
        ("col", C.c_void_p),
        ("val", C.c_void_p),
        ("capacity", C.c_int64),
        ("alloc", ALLOC_FN),
        ("alloc_user", C.c_void_p),
    ]


class TspgTuning(C.Structure):
    """Row binning (tspg_tuning): group-class bounds and hash slots per key."""
    _fields_ = [
        ("sym_lim", C.c_int32 * 4),
        ("num_lim", C.c_int32 * 4),
        ("hash_load", C.c_int32),
        ("dense_win_log2", C.c_int32),
        ("dense_win_fill_log2", C.c_int32),
        ("dense_win_cluster", C.c_int32),
    ]


class TspgServerConfig(C.Structure):
    _fields_ = [("mem_budget", C.c_size_t), ("lanes", C.c_int), ("max_batch", C.c_int)]


TSPG_REQ_AB, TSPG_REQ_RAP = 0, 1


class TspgError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {strerror(status)} (status {status})")


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `make -C trident_b200/csrc`; there is no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    vp, i32, i64, sz = C.c_void_p, C.c_int, C.c_int64, C.c_size_t
    P = C.POINTER
    sigs = {
        "tspg_abi_version": (i32, []),
        "tspg_strerror": (C.c_char_p, [i32]),
        "tspg_last_cuda_error": (i32, [vp]),
        "tspg_ctx_create": (i32, [i32, sz, P(vp)]),
        "tspg_ctx_destroy": (i32, [vp]),
        "tspg_ctx_mem": (i32, [vp, P(sz), P(sz)]),
        "tspg_ctx_stats": (i32, [vp, P(i64)]),
        "tspg_ctx_phase_timing": (i32, [vp, i32]),
        "tspg_ctx_phase_ms": (i32, [vp, P(C.c_float), P(C.c_float)]),
        "tspg_ctx_set_tuning": (i32, [vp, P(TspgTuning)]),
        "tspg_ctx_get_tuning": (i32, [vp, P(TspgTuning)]),
        "tspg_ctx_class_profile": (i32, [vp, i32]),
        "tspg_ctx_class_cycles": (i32, [vp, P(C.c_uint64)]),
        "tspg_batch_create": (i32, [vp, P(vp)]),
        "tspg_batch_destroy": (i32, [vp]),
        "tspg_batch_clear": (i32, [vp]),
        "tspg_batch_add": (i32, [vp, P(TspgCsr), P(TspgCsr), P(C.c_int)]),
        "tspg_batch_run": (i32, [vp, vp, i32, P(i64)]),
        "tspg_batch_count": (i32, [vp, vp, P(i64), P(i64)]),
        "tspg_batch_result": (i32, [vp, i32, P(TspgCsr)]),
        "tspg_spgemm_count": (i32, [vp, vp, P(TspgCsr), P(TspgCsr), P(i64), P(i64)]),
        "tspg_spgemm_row_products": (i32, [vp, vp, P(TspgCsr), P(TspgCsr), vp]),
        "tspg_spgemm_count_mask": (i32, [vp, vp, P(TspgCsr), P(TspgCsr), vp, P(i64), P(i64)]),
        "tspg_spgemm": (i32, [vp, vp, P(TspgCsr), P(TspgCsr), P(TspgCsrOut), i32]),
        "tspg_spgemm_symbolic": (i32, [vp, vp, P(TspgCsr), P(TspgCsr), i32, P(vp), P(i64)]),
        "tspg_spgemm_numeric": (i32, [vp, vp, vp, P(TspgCsr), P(TspgCsr), P(TspgCsrOut)]),
        "tspg_plan_destroy": (i32, [vp]),
        "tspg_spgemm_acc": (i32, [vp, vp, P(TspgCsr), P(TspgCsr), P(TspgCsr), P(TspgCsrOut), i32]),
        "tspg_spadd": (i32, [vp, vp, P(TspgCsr), P(TspgCsr), P(TspgCsrOut)]),
        "tspg_transpose": (i32, [vp, vp, P(TspgCsr), P(TspgCsrOut)]),
        "tspg_coo_to_csx": (i32, [vp, vp, i64, i64, i64, vp, vp, vp, i32, i32, P(TspgCsrOut)]),
        "tspg_mcl_normalize": (i32, [vp, vp, P(TspgCsr), vp]),
        "tspg_mcl_inflate": (i32, [vp, vp, P(TspgCsr), C.c_double, vp]),
        "tspg_mcl_prune": (i32, [vp, vp, P(TspgCsr), C.c_double, P(TspgCsrOut)]),
        "tspg_bitmask_gen": (i32, [vp, vp, vp, i32, i64, vp]),
        "tspg_bitmask_and": (i32, [vp, vp, vp, vp, i64, vp]),
        "tspg_pack": (i32, [vp, vp, P(TspgCsr), i32, vp, vp, sz, vp, P(i64)]),
        "tspg_packed_bytes": (sz, [i64, i64, i32, i32]),
        "tspg_select_ptrs": (i32, [vp, vp, vp, i32, i64, vp]),
        "tspg_rowptrs_to_rownnz": (i32, [vp, vp, vp, i32, i64]),
        "tspg_rownnz_to_rowptrs": (i32, [vp, vp, vp, i32, i64]),
        "tspg_pack_noalloc": (i32, [vp, P(TspgCsr), i32, vp, vp, sz, vp]),
        "tspg_unpack": (i32, [vp, i64, i64, i32, i64, i32, i32, P(TspgCsr)]),
        "tspg_server_create": (i32, [vp, P(TspgServerConfig), P(vp)]),
        "tspg_server_destroy": (i32, [vp]),
        "tspg_server_submit": (i32, [vp, i32, P(TspgCsr), P(TspgCsr), P(TspgCsr), P(i64)]),
        "tspg_server_wait": (i32, [vp, i64, i32, P(TspgCsr), P(C.c_double)]),
        "tspg_server_release": (i32, [vp, i64]),
        "tspg_server_stats": (i32, [vp, P(i64), P(i64), P(i64), P(sz)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def strerror(status: int) -> str:
    return lib.tspg_strerror(status).decode()


def check(status: int, what: str) -> None:
    if status != TSPG_OK:
        raise TspgError(status, what)
