"""GPU: single-GPU 4x4 SUMMA with bitmask-packed tiles equals the plain product."""
import numpy as np
import pytest

import oracle
from trident_b200 import summa, workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("use_masks,batched", [(True, False), (False, False), (True, True)])
def test_summa_4x4_rmat(ctx, use_masks, batched):
    A = workloads.rmat(scale=11, edge_factor=8, seed=3)
    tiles, rb, cb = summa.cut_tiles(A, 4)
    dt = [[t.to_device() for t in row] for row in tiles]
    st = summa.StageStats()
    C = summa.summa(ctx, dt, dt, 4, use_masks=use_masks, stats=st, batched=batched)
    H = summa.assemble(C, rb, cb)
    rp, cj, cx, ca = oracle.spgemm(A, A)
    np.testing.assert_array_equal(H.rowptr, rp)
    np.testing.assert_array_equal(H.col, cj)
    assert np.all(np.abs(H.val - cx) <= 1e-12 * np.maximum(np.abs(cx), ca) + 1e-15)
    if use_masks:
        # R-MAT tiles have empty rows/columns: the masks drop some entries
        assert st.a_kept + st.b_kept < st.a_nnz + st.b_nnz
        assert st.packed_bytes < st.full_bytes


def test_mod_pattern_filters(ctx):
    # The reference's synthetic-pattern check (test/test_compression.cu:452-518):
    # tiles whose non-empty rows / columns follow i % m == k give filters whose
    # bits follow the intersection of those patterns.
    import torch
    from trident_b200 import ops
    from trident_b200.csr import HostCSR

    def pattern_csr(n, keep):
        rp = np.zeros(n + 1, np.int64)
        cols = []
        for i in range(n):
            if keep(i):
                cols.append(i)
            rp[i + 1] = len(cols)
        return HostCSR(n, n, rp, np.array(cols, np.int32), np.ones(len(cols)))

    n = 96
    for (ma, ka), (mb, kb) in [((2, 0), (3, 2)), ((2, 1), (3, 1)), ((6, 5), (2, 1))]:
        A = pattern_csr(n, lambda i: i % ma == ka)   # A's non-empty columns (diagonal)
        B = pattern_csr(n, lambda i: i % mb == kb)   # B's non-empty rows
        dA, dB = A.to_device(), B.to_device()
        fa = summa.col_mask(ctx, dA)
        fb = ops.gen_bitmask(ctx, dB.rowptr, n)
        f = ops.intersect_bitmasks(ctx, fa, fb).cpu().numpy()
        want = np.zeros(n // 8, np.uint8)
        for i in range(n):
            if i % ma == ka and i % mb == kb:
                want[i // 8] |= 1 << (i % 8)
        np.testing.assert_array_equal(f, want)
        fused, _, _ = ops.spgemm_count_mask(ctx, dA, dB)
        np.testing.assert_array_equal(fused.cpu().numpy(), want)


@pytest.mark.parametrize("bits", [(32, 32), (64, 32), (32, 64)])
def test_count_mask_matches_separate_masks(ctx, bits):
    # the fused flop count + stage mask against the oracle's gen / and of the
    # column mask of A and the row mask of B, and against the plain count
    from trident_b200 import ops
    A = workloads.rmat(scale=11, edge_factor=8, seed=5)
    tiles, _, _ = summa.cut_tiles(A, 4)
    for i, s_, j in [(0, 1, 2), (3, 3, 0), (2, 0, 3), (1, 2, 1)]:
        Ah, Bh = tiles[i][s_], tiles[s_][j]
        dA, dB = Ah.to_device(rowptr_bits=bits[0]), Bh.to_device(rowptr_bits=bits[1])
        mask, mults, upper = ops.spgemm_count_mask(ctx, dA, dB)
        colptr = np.zeros(Ah.ncols + 1, np.int64)
        np.add.at(colptr, Ah.col.astype(np.int64) + 1, 1)
        want = oracle.bitmask_and(oracle.bitmask_gen(np.cumsum(colptr), Ah.ncols),
                                  oracle.bitmask_gen(Bh.rowptr, Bh.nrows))
        np.testing.assert_array_equal(mask.cpu().numpy(), want)
        rm = oracle.row_mults(Ah, Bh)
        assert mults == int(rm.sum()) and upper == int(np.minimum(rm, Bh.ncols).sum())
        assert (mults, upper) == ops.spgemm_count(ctx, dA, dB)
