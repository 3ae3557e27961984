"""GPU: the Markov-clustering updates (tspg_mcl_normalize / _inflate / _prune)
against the oracle's restatement of the reference's host loops: prune
bit-exact (no arithmetic), normalize and inflation within a relative 1e-12
(FP64; the row sum is added in another order) or 1e-5 (FP32)."""
import numpy as np
import pytest
import torch

import oracle
from helpers import random_csr
from trident_b200 import ops, workloads
from trident_b200.csr import HostCSR

pytestmark = pytest.mark.gpu


def _mcl_matrix(seed, val_bits=64):
    # an expansion result of a column-stochastic-like matrix: nonnegative
    # values, R-MAT rows (hub rows of thousands of entries), some empty rows,
    # one row that sums to 0
    A = workloads.rmat(scale=12, edge_factor=8, seed=seed)
    rng = np.random.default_rng(seed)
    val = rng.uniform(0, 1, A.nnz) ** 3
    if A.rowptr[8] > A.rowptr[7]:
        val[A.rowptr[7]:A.rowptr[8]] = 0.0
    dt = np.float64 if val_bits == 64 else np.float32
    return HostCSR(A.nrows, A.ncols, A.rowptr, A.col, val.astype(dt).astype(np.float64))


@pytest.mark.parametrize("val_bits,rowptr_bits", [(64, 64), (64, 32), (32, 32)])
def test_inflate_normalize(ctx, val_bits, rowptr_bits):
    H = _mcl_matrix(1, val_bits)
    dt = np.float64 if val_bits == 64 else np.float32
    tol = 1e-12 if val_bits == 64 else 1e-5
    for power in (2.0, 1.5):
        D = H.to_device(rowptr_bits=rowptr_bits, val_bits=val_bits)
        ops.mcl_inflate(ctx, D, power)
        want = oracle.mcl_inflate(H.rowptr, H.val.astype(dt), power)
        got = D.val.cpu().numpy()
        assert np.all(np.abs(got - want) <= tol * np.abs(want) + 1e-300)
    D = H.to_device(rowptr_bits=rowptr_bits, val_bits=val_bits)
    ops.mcl_normalize(ctx, D)
    want = oracle.mcl_normalize(H.rowptr, H.val.astype(dt))
    got = D.val.cpu().numpy()
    assert np.all(np.abs(got - want) <= tol * np.abs(want) + 1e-300)
    # rows sum to 1 except the zero row and empty rows
    rows = np.repeat(np.arange(H.nrows), np.diff(H.rowptr))
    rs = np.bincount(rows, weights=got.astype(np.float64), minlength=H.nrows)
    nz = np.diff(H.rowptr) > 0
    assert np.allclose(rs[nz & (np.arange(H.nrows) != 7)], 1.0, rtol=1e-4)


@pytest.mark.parametrize("val_bits,rowptr_bits", [(64, 64), (64, 32), (32, 64)])
def test_prune(ctx, val_bits, rowptr_bits):
    H = _mcl_matrix(2, val_bits)
    D = H.to_device(val_bits=val_bits)
    dt = np.float64 if val_bits == 64 else np.float32
    for tol in (1e-3, 0.1, 0.5, 2.0):
        P = ops.mcl_prune(ctx, D, tol, rowptr_bits=rowptr_bits).to_host()
        rp, cj, cx = oracle.mcl_prune(H.rowptr, H.col, H.val.astype(dt), tol)
        np.testing.assert_array_equal(P.rowptr.astype(np.int64), rp)
        np.testing.assert_array_equal(P.col, cj)
        np.testing.assert_array_equal(P.val.astype(dt), cx)


def test_mcl_iteration_and_empty(ctx):
    # one iteration (expansion A·A, inflation, prune) against the oracle; and
    # an empty matrix through every step
    H = _mcl_matrix(3)
    D = H.to_device()
    ops.mcl_normalize(ctx, D)
    Hn = HostCSR(H.nrows, H.ncols, H.rowptr, H.col, D.val.cpu().numpy())
    E = ops.spgemm(ctx, D, D)
    ops.mcl_inflate(ctx, E, 2.0)
    P = ops.mcl_prune(ctx, E, 1e-4).to_host()
    rp, cj, cx, _ = oracle.spgemm(Hn, Hn)
    cx = oracle.mcl_inflate(rp, cx, 2.0)
    prp, pcj, pcx = oracle.mcl_prune(rp, cj, cx, 1e-4)
    # entries near the threshold may fall either side: compare away from it
    got = dict(zip(zip(np.repeat(np.arange(P.nrows), np.diff(P.rowptr)), P.col), P.val))
    want = dict(zip(zip(np.repeat(np.arange(H.nrows), np.diff(prp)), pcj), pcx))
    far = {k: v for k, v in want.items() if v > 1.001e-4}
    assert all(abs(got[k] - v) <= 1e-12 * v for k, v in far.items())
    assert all(v > 0.999e-4 for v in got.values())
    Z = random_csr(5, 5, density=0.0, seed=1).to_device()
    ops.mcl_inflate(ctx, Z, 2.0)
    ops.mcl_normalize(ctx, Z)
    assert ops.mcl_prune(ctx, Z, 0.5).nnz == 0
