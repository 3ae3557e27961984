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

import oracle
from helpers import random_csr
from trident_b200 import ops
from trident_b200._lib import (TSPG_COLS, TSPG_ESCRATCH, TSPG_OK, TSPG_PACK_NOALLOC_MAX_SEGMENTS, TSPG_ROWS,
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


def _unpacked(buf, kept, length, val_bits, ptr_bits):
    """(ptr, idx, val) of a packed tile in the [val | idx | ptr] wire layout."""
    b = buf.cpu().numpy()
    vdt = np.float64 if val_bits == 64 else np.float32
    vb = val_bits // 8
    val = b[:kept * vb].view(vdt)
    idx = b[kept * vb:kept * (vb + 4)].view(np.int32)
    po = (kept * (vb + 4) + ptr_bits // 8 - 1) // (ptr_bits // 8) * (ptr_bits // 8)
    ptr = b[po:po + (length + 1) * ptr_bits // 8].view(np.int32 if ptr_bits == 32 else np.int64)
    return ptr.astype(np.int64), idx, val


def test_noalloc_cols_major_matches_pack_and_oracle(ctx):
    """A CSC tile (the A operand of a stage, packed by column) through the
    allocation-free entry point, twice: byte for byte tspg_pack's output, and
    the oracle's pack of the same segments."""
    rng = np.random.default_rng(17)
    H = random_csr(5000, 30000, density=0.002, seed=8)  # the CSR of the transpose of a 30000 x 5000 CSC tile
    M = H.to_device(rowptr_bits=32, val_bits=64)
    m = M.abi()
    m.nrows, m.ncols = H.ncols, H.nrows  # CSC view: the pointer array runs over the 5000 columns
    for call in range(2):
        mask_h = rng.integers(0, 256, size=(H.nrows + 7) // 8, dtype=np.uint8)
        mask = torch.tensor(mask_h, device="cuda")
        cap = ops.packed_bytes(H.nnz, H.nrows, 64, 32)
        got = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        kept_dev = torch.full((1,), -1, dtype=torch.int64, device="cuda")
        st = lib.tspg_pack_noalloc(torch.cuda.current_stream().cuda_stream, C.byref(m), TSPG_COLS,
                                   mask.data_ptr(), got.data_ptr(), got.numel(), kept_dev.data_ptr())
        assert st == TSPG_OK, st
        want = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        kept_want = C.c_int64()
        st = lib.tspg_pack(ctx.h, torch.cuda.current_stream().cuda_stream, C.byref(m), TSPG_COLS,
                           mask.data_ptr(), want.data_ptr(), want.numel(), None, C.byref(kept_want))
        assert st == TSPG_OK, st
        torch.cuda.synchronize()
        kept = int(kept_dev.item())
        assert kept == kept_want.value, f"call {call}"
        n = ops.packed_bytes(kept, H.nrows, 64, 32)
        assert torch.equal(got[:n], want[:n]), f"call {call}: packed bytes differ"
        optr, oidx, oval = oracle.pack(H.rowptr, H.col, H.val, mask_h)
        ptr, idx, val = _unpacked(got, kept, H.nrows, 64, 32)
        np.testing.assert_array_equal(ptr, optr)
        np.testing.assert_array_equal(idx, oidx)
        np.testing.assert_array_equal(val, oval)


def test_noalloc_empty_tile():
    """A tile with no segments: nothing kept, the pointer array is [0] — also
    after a call that left other counts in the scratch."""
    H = random_csr(300, 200, density=0.05, seed=2).to_device()
    mask = torch.full(((300 + 7) // 8,), 255, dtype=torch.uint8, device="cuda")
    _pack_noalloc(H, mask)  # leaves a non-zero first count in the scratch
    rp = torch.zeros(1, dtype=torch.int32, device="cuda")
    E = TspgCsr(0, 7, 0, rp.data_ptr(), 32, 64, None, None)
    out = torch.full((16,), 0xAB, dtype=torch.uint8, device="cuda")
    kept = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    st = lib.tspg_pack_noalloc(torch.cuda.current_stream().cuda_stream, C.byref(E), TSPG_ROWS, None,
                               out.data_ptr(), out.numel(), kept.data_ptr())
    assert st == TSPG_OK, st
    torch.cuda.synchronize()
    assert int(kept.item()) == 0
    assert out[:4].view(torch.int32).item() == 0


def test_noalloc_rejects_oversize_tile():
    big = TSPG_PACK_NOALLOC_MAX_SEGMENTS + 1
    m = TspgCsr(big, 4, 0, 1 << 20, 32, 64, None, None)  # rejected before any device work
    st = lib.tspg_pack_noalloc(None, C.byref(m), TSPG_ROWS, 1 << 20, 1 << 20, 1 << 30, None)
    assert st == TSPG_ESCRATCH
    assert "static scratch" in lib.tspg_strerror(st).decode()
