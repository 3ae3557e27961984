"""GPU: the device COO -> CSR / CSC builder (tspg_coo_to_csx) against the
oracle's restatement of the reference's host builders: pointer arrays and
minor indices bit-exact, values moved bit-exact (no arithmetic)."""
import numpy as np
import pytest
import torch

import oracle
from trident_b200 import ops, workloads
from trident_b200._lib import TSPG_COLS, TSPG_EINVAL, TSPG_ROWS, TspgError

pytestmark = pytest.mark.gpu


def _coo(nrows, ncols, nnz, seed, dup=0.0):
    rng = np.random.default_rng(seed)
    r = rng.integers(0, nrows, nnz).astype(np.int32)
    c = rng.integers(0, ncols, nnz).astype(np.int32)
    if dup and nnz:  # repeat some triples' coordinates with other values
        k = int(nnz * dup)
        src = rng.integers(0, nnz, k)
        dst = rng.integers(0, nnz, k)
        r[dst], c[dst] = r[src], c[src]
    v = rng.uniform(-1, 1, nnz)
    return r, c, v


def _check(ctx, nrows, ncols, r, c, v, major, rowptr_bits=64, val_bits=64):
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    vv = v.astype(np.float64 if val_bits == 64 else np.float32)
    M = ops.coo_to_csx(ctx, nrows, ncols, dev(r), dev(c), dev(vv), major=major, rowptr_bits=rowptr_bits)
    maj, mnr, nmaj = (r, c, nrows) if major == TSPG_ROWS else (c, r, ncols)
    ptr, idx, val = oracle.coo_to_csx(nmaj, maj, mnr, vv)
    H = M.to_host()
    np.testing.assert_array_equal(H.rowptr.astype(np.int64), ptr)
    np.testing.assert_array_equal(H.col, idx)
    np.testing.assert_array_equal(H.val.astype(vv.dtype), val)
    return M


@pytest.mark.parametrize("major", [TSPG_ROWS, TSPG_COLS])
@pytest.mark.parametrize("rowptr_bits,val_bits", [(64, 64), (32, 64), (32, 32)])
def test_random_coo_with_duplicates(ctx, major, rowptr_bits, val_bits):
    r, c, v = _coo(3000, 5000, 60000, seed=1, dup=0.2)
    _check(ctx, 3000, 5000, r, c, v, major, rowptr_bits, val_bits)


def test_rmat_coo_long_segments(ctx):
    # R-MAT draws: hub rows / columns of > 4096 entries take the multi-run
    # merge of the segment sort; 5000 coordinates repeated with other values
    A = workloads.rmat(scale=14, edge_factor=16, seed=4)
    rows = np.repeat(np.arange(A.nrows, dtype=np.int32), np.diff(A.rowptr))
    perm = np.random.default_rng(5).permutation(A.nnz)
    r, c, v = rows[perm], A.col[perm], A.val[perm]
    # coordinates unique: the shuffled generator output comes back as it was
    M = _check(ctx, A.nrows, A.ncols, r, c, v, TSPG_ROWS).to_host()
    np.testing.assert_array_equal(M.rowptr.astype(np.int64), A.rowptr.astype(np.int64))
    np.testing.assert_array_equal(M.col, A.col)
    np.testing.assert_array_equal(M.val, A.val)
    # plus 10000 entries in row 3 (two merge passes of the segment sort) and
    # 7000 in column 5 (one pass, then the copy back), repeats among them
    rng = np.random.default_rng(6)
    ex_c = rng.integers(0, A.ncols, 10000).astype(np.int32)
    ex_r = rng.integers(0, A.nrows, 7000).astype(np.int32)
    r2 = np.concatenate([r, r[:5000], np.full(10000, 3, np.int32), ex_r])
    c2 = np.concatenate([c, c[:5000], ex_c, np.full(7000, 5, np.int32)])
    v2 = np.concatenate([v, -v[:5000], rng.uniform(-1, 1, 17000)])
    assert np.bincount(r2).max() > 8192 and 4096 < np.bincount(c2).max() <= 8192
    for major in (TSPG_ROWS, TSPG_COLS):
        _check(ctx, A.nrows, A.ncols, r2, c2, v2, major)


def test_empty_and_edge_shapes(ctx):
    e = np.zeros(0, np.int32)
    M = ops.coo_to_csx(ctx, 5, 7, torch.from_numpy(e).cuda(), torch.from_numpy(e).cuda(),
                       torch.zeros(0, dtype=torch.float64, device="cuda"))
    assert M.nnz == 0 and M.rowptr.cpu().tolist() == [0] * 6
    r, c, v = _coo(1, 1, 100, seed=3)  # every entry at (0, 0)
    _check(ctx, 1, 1, r, c, v, TSPG_ROWS)
    r, c, v = _coo(50000, 3, 20000, seed=4)  # mostly empty rows
    _check(ctx, 50000, 3, r, c, v, TSPG_ROWS)
    _check(ctx, 50000, 3, r, c, v, TSPG_COLS)


def test_out_of_range_index_rejected(ctx):
    r, c, v = _coo(100, 100, 1000, seed=6)
    c[500] = 100
    dev = lambda a: torch.from_numpy(a).cuda()
    with pytest.raises(TspgError) as e:
        ops.coo_to_csx(ctx, 100, 100, dev(r), dev(c), dev(v))
    assert e.value.status == TSPG_EINVAL
    c[500] = 0
    r[7] = -1
    with pytest.raises(TspgError) as e:
        ops.coo_to_csx(ctx, 100, 100, dev(r), dev(c), dev(v), major=TSPG_COLS)
    assert e.value.status == TSPG_EINVAL
