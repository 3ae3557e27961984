"""GPU parity at sizes where C's row offsets pass INT32_MAX.

The benchmark's product (R-MAT scale 20, nnz(C) = 9.7e9) needs int64 row
offsets; this test crosses 2^31 output entries on a shape that fits in about
30 GB: C = A·B with B 16 x 2^20 (each row a random 75 % of the columns) and A
2300 x 16 with two entries per row, so every row of C is the union of two rows
of B (about 983k columns, 1.6M products).  The whole row-offset array is
checked against the union sizes computed on the host, and sampled rows —
including the last ones, whose offsets lie beyond 2^31 — against the oracle.
"""
import numpy as np
import pytest
import torch

import oracle
from helpers import TOL64
from trident_b200 import ops
from trident_b200.csr import HostCSR

pytestmark = pytest.mark.gpu


def _operands():
    n, kb, m = 1 << 20, 16, 2300
    rng = np.random.default_rng(11)
    brows = [np.nonzero(rng.random(n) < 0.75)[0].astype(np.int32) for _ in range(kb)]
    brp = np.zeros(kb + 1, np.int64)
    brp[1:] = np.cumsum([r.size for r in brows])
    bcol = np.concatenate(brows)
    B = HostCSR(kb, n, brp, bcol, rng.uniform(-1, 1, bcol.size))
    pairs = np.stack([np.arange(m) % kb, (np.arange(m) + 5) % kb], axis=1)
    pairs.sort(axis=1)
    A = HostCSR(m, kb, np.arange(0, 2 * m + 1, 2, dtype=np.int64), pairs.ravel().astype(np.int32),
                rng.uniform(-1, 1, 2 * m))
    union = {}
    for a, b in {tuple(p) for p in pairs.tolist()}:
        union[(a, b)] = int(np.union1d(brows[a], brows[b]).size)
    lens = np.array([union[tuple(p)] for p in pairs.tolist()], np.int64)
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    return A, B, rp


def test_int64_offsets_beyond_int32(ctx):
    A, B, rp_expect = _operands()
    assert rp_expect[-1] > 2**31 - 1
    dA, dB = A.to_device(), B.to_device()
    mults, _ = ops.spgemm_count(ctx, dA, dB)
    assert mults == int(np.diff(B.rowptr)[A.col].sum())
    C = ops.spgemm(ctx, dA, dB, rowptr_bits=64)
    assert C.rowptr.dtype == torch.int64
    rp = C.rowptr.cpu().numpy()
    np.testing.assert_array_equal(rp, rp_expect)
    for r in [0, 1, 1150, A.nrows - 2, A.nrows - 1]:
        lo, hi = int(rp[r]), int(rp[r + 1])
        cols = C.col[lo:hi].cpu().numpy()
        vals = C.val[lo:hi].cpu().numpy()
        orp, cj, cx, ca = oracle.spgemm(A.rows(np.array([r])), B)
        np.testing.assert_array_equal(cols, cj)
        assert np.all(np.abs(vals - cx) <= TOL64 * np.maximum(np.abs(cx), ca))
    assert rp[A.nrows - 1] > 2**31  # the last rows were addressed past int32
    del C, dA, dB
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
