"""Sparse containers: host CSR (numpy, defined in synth.py and re-exported
here) and device CSR (torch tensors on CUDA).

Both carry the C ABI view (``abi()``) used by every call into libtspg.  The
device container only borrows torch for memory and streams; all arithmetic is
in the library's CUDA kernels.
"""
from __future__ import annotations

import numpy as np

from ._lib import TspgCsr
from .synth import HostCSR  # noqa: F401  (re-exported: the host container)


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
