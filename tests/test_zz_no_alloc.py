"""GPU: tspg_pack_noalloc, the allocation-free tile pack.

Some callers cannot allocate device memory while they pack: a communication
thread that packs the next tile while the compute stream and network transfers
run would be stalled by cudaMalloc's implicit device synchronisation.  For
them the library has one entry point whose scratch is a static device array.
This test calls it through the C ABI and checks its output byte for byte
against tspg_pack (the allocating entry point) on two calls in a row, so the
second call runs on the scratch contents the first one left behind.  It sits
in a file of its own that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import random_csr
from trident_b200 import ops
from trident_b200._lib import (TSPG_ESCRATCH, TSPG_OK, TSPG_PACK_NOALLOC_MAX_SEGMENTS, TSPG_ROWS,
                               TspgCsr, lib)

pytestmark = pytest.mark.gpu


def _pack_noalloc(M, mask, major=TSPG_ROWS):
    length = M.nrows if major == TSPG_ROWS else M.ncols
    cap = ops.packed_bytes(M.nnz, length, M.val_bits, M.rowptr_bits)
    out = torch.zeros(max(cap, 16), dtype=torch.uint8, device="cuda")
    kept = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    m = M.abi()
    st = lib.tspg_pack_noalloc(torch.cuda.current_stream().cuda_stream, C.byref(m), major,
                               mask.data_ptr(), out.data_ptr(), out.numel(), kept.data_ptr())
    assert st == TSPG_OK, st
    return out, kept


def _pack_reference(ctx, M, mask, major=TSPG_ROWS):
    length = M.nrows if major == TSPG_ROWS else M.ncols
    cap = ops.packed_bytes(M.nnz, length, M.val_bits, M.rowptr_bits)
    out = torch.zeros(max(cap, 16), dtype=torch.uint8, device="cuda")
    buf, kept = ops.compress(ctx, M, mask, major, out=out)
    return buf, kept


@pytest.mark.parametrize("ptr_bits,val_bits", [(32, 64), (64, 32)])
def test_noalloc_matches_pack_twice(ctx, ptr_bits, val_bits):
    rng = np.random.default_rng(ptr_bits + val_bits)
    M = random_csr(70000, 9000, density=0.0015, seed=3).to_device(rowptr_bits=ptr_bits, val_bits=val_bits)
    for call in range(2):  # second call reuses the scratch the first one left
        mask = torch.tensor(rng.integers(0, 256, size=(M.nrows + 7) // 8, dtype=np.uint8), device="cuda")
        got, kept_dev = _pack_noalloc(M, mask)
        want, kept = _pack_reference(ctx, M, mask)
        torch.cuda.synchronize()
        assert int(kept_dev.item()) == kept, f"call {call}"
        n = ops.packed_bytes(kept, M.nrows, val_bits, ptr_bits)
        assert torch.equal(got[:n], want[:n]), f"call {call}: packed bytes differ"


def test_noalloc_rejects_oversize_tile():
    big = TSPG_PACK_NOALLOC_MAX_SEGMENTS + 1
    m = TspgCsr(big, 4, 0, 1 << 20, 32, 64, None, None)  # rejected before any device work
    st = lib.tspg_pack_noalloc(None, C.byref(m), TSPG_ROWS, 1 << 20, 1 << 20, 1 << 30, None)
    assert st == TSPG_ESCRATCH
    assert "static scratch" in lib.tspg_strerror(st).decode()
