"""Host CSR container and the ctypes binding of libtspg_synth.so (the seeded
workload generators, the .bmtx reader and a host transpose declared in
include/tspg_synth.h).

This module loads only the host-only generator library, never the device
library libtspg.so, so the benchmark's CPU legs (the timed CPU baseline and the
reference arm) build exactly the same matrices as the GPU arm without mapping
the GPU product.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
SYNTH_PATH = os.path.join(_HERE, "libtspg_synth.so")


class TspgHostCsr(C.Structure):
    _fields_ = [
        ("nrows", C.c_int64),
        ("ncols", C.c_int64),
        ("nnz", C.c_int64),
        ("rowptr", C.POINTER(C.c_int64)),
        ("col", C.POINTER(C.c_int32)),
        ("val", C.POINTER(C.c_double)),
    ]


def _load() -> C.CDLL:
    if not os.path.exists(SYNTH_PATH):
        raise ImportError(f"{SYNTH_PATH} is missing: build it with `make -C trident_b200/csrc`")
    lib = C.CDLL(SYNTH_PATH)
    i32, i64 = C.c_int, C.c_int64
    P = C.POINTER
    sigs = {
        "tspg_host_free": (None, [P(TspgHostCsr)]),
        "tspg_gen_uniform_rows": (i32, [i64, i32, i32, C.c_uint64, P(TspgHostCsr)]),
        "tspg_gen_rmat": (i32, [i32, i32, C.c_double, C.c_double, C.c_double, C.c_uint64, P(TspgHostCsr)]),
        "tspg_gen_laplacian": (i32, [i64, i64, i64, i32, P(TspgHostCsr)]),
        "tspg_gen_sa_prolongator": (i32, [i64, i64, i64, i32, i32, C.c_double, P(TspgHostCsr)]),
        "tspg_host_transpose": (i32, [P(TspgHostCsr), P(TspgHostCsr)]),
        "tspg_gen_poisson_rows": (i32, [i64, C.c_double, C.c_uint64, P(TspgHostCsr)]),
        "tspg_read_bmtx": (i32, [C.c_char_p, P(TspgHostCsr)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what}: status {status}")


@dataclass
class HostCSR:
    nrows: int
    ncols: int
    rowptr: np.ndarray  # int64 (or int32), nrows + 1
    col: np.ndarray  # int32
    val: np.ndarray  # float64 / float32

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1]) if len(self.rowptr) else 0

    @staticmethod
    def from_abi(h: TspgHostCsr) -> "HostCSR":
        """Copy a library-allocated host CSR into numpy and free the original."""
        n, nnz = int(h.nrows), int(h.nnz)
        rp = np.ctypeslib.as_array(h.rowptr, shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(h.col, shape=(max(nnz, 1),))[:nnz].copy()
        val = np.ctypeslib.as_array(h.val, shape=(max(nnz, 1),))[:nnz].copy()
        out = HostCSR(n, int(h.ncols), rp, col, val)
        lib.tspg_host_free(C.byref(h))
        return out

    def abi_host(self) -> TspgHostCsr:
        """Borrowed ABI view (int64 rowptr, float64 values) of this matrix."""
        self._keep = (np.ascontiguousarray(self.rowptr, dtype=np.int64),
                      np.ascontiguousarray(self.col, dtype=np.int32),
                      np.ascontiguousarray(self.val, dtype=np.float64))
        rp, col, val = self._keep
        return TspgHostCsr(self.nrows, self.ncols, int(rp[-1]),
                           rp.ctypes.data_as(C.POINTER(C.c_int64)),
                           col.ctypes.data_as(C.POINTER(C.c_int32)),
                           val.ctypes.data_as(C.POINTER(C.c_double)))

    def rows(self, rows: np.ndarray) -> "HostCSR":
        """The sub-matrix of the listed rows (in the given order)."""
        rows = np.asarray(rows, dtype=np.int64)
        lens = self.rowptr[rows + 1] - self.rowptr[rows]
        rp = np.zeros(rows.size + 1, dtype=np.int64)
        np.cumsum(lens, out=rp[1:])
        if rows.size and rp[-1]:
            starts = np.repeat(self.rowptr[rows] - rp[:-1], lens)
            idx = np.arange(rp[-1], dtype=np.int64) + starts
        else:
            idx = np.zeros(0, np.int64)
        return HostCSR(rows.size, self.ncols, rp, self.col[idx], self.val[idx])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.rowptr), shape=(self.nrows, self.ncols))

    def astype(self, rowptr=np.int64, val=np.float64) -> "HostCSR":
        return HostCSR(self.nrows, self.ncols, self.rowptr.astype(rowptr),
                       self.col.astype(np.int32), self.val.astype(val))

    def to_device(self, device="cuda", rowptr_bits: int = 32, val_bits: int = 64,
                  pinned_from=None):
        """Copy to the GPU as a DeviceCSR (loads the device library)."""
        import torch

        from .csr import DeviceCSR
        rdt = torch.int32 if rowptr_bits == 32 else torch.int64
        vdt = torch.float64 if val_bits == 64 else torch.float32
        rp = torch.from_numpy(np.ascontiguousarray(self.rowptr)).to(device=device, dtype=rdt)
        col = torch.from_numpy(np.ascontiguousarray(self.col, dtype=np.int32)).to(device)
        val = torch.from_numpy(np.ascontiguousarray(self.val)).to(device=device, dtype=vdt)
        return DeviceCSR(self.nrows, self.ncols, rp, col, val)
