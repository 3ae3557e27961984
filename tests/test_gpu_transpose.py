"""GPU parity: device transpose (CSC <-> CSR) against the oracle's transpose."""
import numpy as np
import pytest

import oracle
from helpers import random_csr
from trident_b200 import ops, workloads

pytestmark = pytest.mark.gpu


def _check(ctx, M, rowptr_bits=64):
    T = ops.transpose(ctx, M.to_device(), rowptr_bits=rowptr_bits).to_host()
    rp, col, val = oracle.transpose(M)
    np.testing.assert_array_equal(T.rowptr.astype(np.int64), rp)
    np.testing.assert_array_equal(T.col, col)
    np.testing.assert_array_equal(T.val, val)


@pytest.mark.parametrize("seed", [0, 1])
def test_transpose_random(ctx, seed):
    _check(ctx, random_csr(3000, 2000, density=0.01, seed=seed))


def test_transpose_long_columns(ctx):
    # R-MAT hub columns exceed one CTA segment (4096): sorted runs + merges
    A = workloads.rmat(scale=16, edge_factor=16, seed=2)
    assert np.bincount(A.col, minlength=A.ncols).max() > 4096
    _check(ctx, A, rowptr_bits=32)


def test_prolongator_restriction(ctx):
    P = workloads.sa_prolongator(12, pts=27, agg=3)
    _check(ctx, P)


def test_transpose_empty_and_roundtrip(ctx):
    from trident_b200.csr import HostCSR
    Z = HostCSR(5, 7, np.zeros(6, np.int64), np.zeros(0, np.int32), np.zeros(0))
    T = ops.transpose(ctx, Z.to_device())
    assert T.nrows == 7 and T.nnz == 0 and T.rowptr.cpu().tolist() == [0] * 8
    M = random_csr(400, 300, density=0.05, seed=4)
    TT = ops.transpose(ctx, ops.transpose(ctx, M.to_device())).to_host()
    np.testing.assert_array_equal(TT.col, M.col)
    np.testing.assert_array_equal(TT.val, M.val)
