"""Sparse containers: host CSR (numpy) and device CSR (torch tensors on CUDA).

Both carry the C ABI view (``abi()``) used by every call into libtspg.  The
device container only borrows torch for memory and streams; all arithmetic is
in the library's CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import TspgCsr, TspgHostCsr, lib


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

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.rowptr), shape=(self.nrows, self.ncols))

    def astype(self, rowptr=np.int64, val=np.float64) -> "HostCSR":
        return HostCSR(self.nrows, self.ncols, self.rowptr.astype(rowptr),
                       self.col.astype(np.int32), self.val.astype(val))

    def to_device(self, device="cuda", rowptr_bits: int = 32, val_bits: int = 64,
                  pinned_from=None) -> "DeviceCSR":
        import torch
        rdt = torch.int32 if rowptr_bits == 32 else torch.int64
        vdt = torch.float64 if val_bits == 64 else torch.float32
        rp = torch.from_numpy(np.ascontiguousarray(self.rowptr)).to(device=device, dtype=rdt)
        col = torch.from_numpy(np.ascontiguousarray(self.col, dtype=np.int32)).to(device)
        val = torch.from_numpy(np.ascontiguousarray(self.val)).to(device=device, dtype=vdt)
        return DeviceCSR(self.nrows, self.ncols, rp, col, val)


class DeviceCSR:
    """CSR whose arrays are CUDA torch tensors (borrowed by the ABI views)."""

    def __init__(self, nrows, ncols, rowptr, col, val, nnz=None):
        self.nrows = int(nrows)
        self.ncols = int(ncols)
        self.rowptr = rowptr
        self.col = col
        self.val = val
        self._nnz = nnz

    @property
    def nnz(self) -> int:
        if self._nnz is None:
            self._nnz = int(self.rowptr[-1].item()) if self.rowptr.numel() else 0
        return self._nnz

    @property
    def rowptr_bits(self) -> int:
        return 32 if self.rowptr.element_size() == 4 else 64

    @property
    def val_bits(self) -> int:
        return 64 if self.val.element_size() == 8 else 32

    def abi(self) -> TspgCsr:
        return TspgCsr(self.nrows, self.ncols, self.nnz, self.rowptr.data_ptr(),
                       self.rowptr_bits, self.val_bits,
                       self.col.data_ptr() if self.nnz else None,
                       self.val.data_ptr() if self.nnz else None)

    def to_host(self) -> HostCSR:
        return HostCSR(self.nrows, self.ncols,
                       self.rowptr.cpu().numpy().astype(np.int64),
                       self.col[: self.nnz].cpu().numpy(),
                       self.val[: self.nnz].cpu().numpy())
