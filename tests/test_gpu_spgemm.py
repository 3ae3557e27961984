"""GPU parity: SpGEMM through the C ABI against the oracle on the same inputs.

Structure (rowptr, sorted columns) must be bit-exact; FP64 values within
|x - y| <= 1e-12 * max(|y|, sum |a_ik b_kj|) per entry (summation order only).
"""
import os

import numpy as np
import pytest
import torch

import oracle
from helpers import TOL32, check_product, random_csr, spgemm_poisoned
from trident_b200 import ops, workloads
from trident_b200._lib import TSPG_EINVAL, TSPG_F_B_SORTED, TspgError
from trident_b200.csr import HostCSR

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("rp_in,rp_out", [(32, 64), (64, 32), (32, 32), (64, 64)])
def test_uniform_rows_1024(ctx, rp_in, rp_out):
    A = workloads.uniform_rows(1024, 16, True, seed=1)
    dA = A.to_device(rowptr_bits=rp_in)
    C = ops.spgemm(ctx, dA, dA, rowptr_bits=rp_out)
    assert C.rowptr.dtype == (torch.int32 if rp_out == 32 else torch.int64)
    check_product(C, A, A)


@pytest.mark.parametrize("name", ["n16_full.bmtx", "n1024.bmtx"])
def test_bmtx_fixtures(ctx, name):
    A = workloads.read_bmtx(os.path.join(GOLD, name))
    dA = A.to_device()
    check_product(ops.spgemm(ctx, dA, dA), A, A)


@pytest.mark.parametrize("scale", [8, 11, 13])
def test_rmat(ctx, scale):
    A = workloads.rmat(scale=scale, edge_factor=16, seed=1)
    dA = A.to_device()
    check_product(ops.spgemm(ctx, dA, dA), A, A)


def test_rmat_scale15_all_classes(ctx):
    # scale 15 R-MAT squared has rows in every class, DENSE symbolic included
    A = workloads.rmat(scale=15, edge_factor=16, seed=2)
    dA = A.to_device()
    mults = oracle.row_mults(A, A)
    assert mults.max() > 24576
    check_product(ops.spgemm(ctx, dA, dA), A, A)


def test_dense_numeric_rows_multiwindow(ctx):
    # a few rows whose products hit > 8192 distinct columns over 3 windows of
    # 16384 columns: the DENSE numeric class with cursors
    rng = np.random.default_rng(4)
    n = 40000
    B = random_csr(3000, n, per_row=40, seed=5)
    A = random_csr(64, 3000, per_row=4, seed=6)
    heavy = random_csr(3, 3000, per_row=800, seed=7)
    Ah = HostCSR(67, 3000, np.concatenate([A.rowptr, A.rowptr[-1] + heavy.rowptr[1:]]),
                 np.concatenate([A.col, heavy.col]), np.concatenate([A.val, heavy.val]))
    C = ops.spgemm(ctx, Ah.to_device(), B.to_device())
    H = check_product(C, Ah, B)
    assert np.diff(H.rowptr).max() > 8192


def test_dense_numeric_long_a_row_global_cursors(ctx):
    # one A row with > 8192 entries: cursors live in the global scratch
    B = random_csr(20000, 30000, per_row=3, seed=8)
    A = random_csr(2, 20000, per_row=9000, seed=9)
    check_product(ops.spgemm(ctx, A.to_device(), B.to_device()), A, B)


def test_unsorted_and_duplicate_b_rows(ctx):
    B = random_csr(500, 20000, per_row=60, seed=10, sort=False)
    A = random_csr(300, 500, per_row=200, seed=11)  # several DENSE numeric rows
    check_product(ops.spgemm(ctx, A.to_device(), B.to_device()), A, B)
    Bd = random_csr(400, 300, per_row=30, seed=12, sort=False, dup=True)
    Ad = random_csr(200, 400, per_row=10, seed=13, dup=True)
    check_product(ops.spgemm(ctx, Ad.to_device(), Bd.to_device()), Ad, Bd)


def test_galerkin_rap_small(ctx):
    R, A, P = workloads.galerkin_operands(n=18, pts=27, agg=3)
    dR, dA, dP = R.to_device(), A.to_device(), P.to_device()
    AP = ops.spgemm(ctx, dA, dP, rowptr_bits=32)
    hAP = check_product(AP, A, P)
    RAP = ops.spgemm(ctx, dR, AP)
    check_product(RAP, R, hAP)


def test_poisson_rows(ctx):
    A = workloads.poisson_rows(5000, 24.0, seed=3)
    B = workloads.poisson_rows(5000, 24.0, seed=4)
    check_product(ops.spgemm(ctx, A.to_device(), B.to_device()), A, B)


def test_empty_cases(ctx):
    E = HostCSR(0, 5, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0))
    B = random_csr(5, 7, density=0.5, seed=1)
    C = ops.spgemm(ctx, E.to_device(), B.to_device())
    assert C.nrows == 0 and C.nnz == 0 and C.rowptr.cpu().tolist() == [0]
    Z = HostCSR(6, 5, np.zeros(7, np.int64), np.zeros(0, np.int32), np.zeros(0))
    C = ops.spgemm(ctx, Z.to_device(), B.to_device())
    assert C.nnz == 0 and C.rowptr.cpu().tolist() == [0] * 7
    A = random_csr(6, 5, density=0.5, seed=2)
    BZ = HostCSR(5, 7, np.zeros(6, np.int64), np.zeros(0, np.int32), np.zeros(0))
    C = ops.spgemm(ctx, A.to_device(), BZ.to_device())
    assert C.nnz == 0
    # some empty rows mixed in
    A2 = random_csr(100, 50, density=0.05, seed=3)
    B2 = random_csr(50, 80, density=0.05, seed=4)
    check_product(ops.spgemm(ctx, A2.to_device(), B2.to_device()), A2, B2)


def test_structural_zero_kept(ctx):
    A = HostCSR(1, 2, np.array([0, 2]), np.array([0, 1], np.int32), np.array([1.0, 1.0]))
    B = HostCSR(2, 1, np.array([0, 1, 2]), np.array([0, 0], np.int32), np.array([1.0, -1.0]))
    C = ops.spgemm(ctx, A.to_device(), B.to_device()).to_host()
    assert C.rowptr.tolist() == [0, 1] and C.col.tolist() == [0] and C.val[0] == 0.0


def test_fp32_twin(ctx):
    A = workloads.rmat(scale=11, edge_factor=8, seed=3)
    dA = A.to_device(val_bits=32)
    A32 = HostCSR(A.nrows, A.ncols, A.rowptr, A.col, A.val.astype(np.float32).astype(np.float64))
    check_product(ops.spgemm(ctx, dA, dA), A32, A32, tol=TOL32)


def test_plan_reuse_new_values(ctx):
    A = workloads.rmat(scale=10, edge_factor=16, seed=5)
    dA = A.to_device()
    plan = ops.Plan(ctx, dA, dA)
    C1 = plan.numeric(dA, dA)
    check_product(C1, A, A)
    A2 = HostCSR(A.nrows, A.ncols, A.rowptr, A.col, -2.0 * A.val)
    dA2 = A2.to_device()
    C2 = plan.numeric(dA2, dA2)
    check_product(C2, A2, A2)
    plan.close()


def test_count_pass(ctx):
    A = workloads.rmat(scale=11, edge_factor=16, seed=6)
    dA = A.to_device()
    mults, upper = ops.spgemm_count(ctx, dA, dA)
    rm = oracle.row_mults(A, A)
    assert mults == int(rm.sum())
    assert upper == int(np.minimum(rm, A.ncols).sum())


@pytest.mark.parametrize("bits", [32, 64])
def test_count_pass_row_lengths(ctx, bits):
    # The count pass walks rows of at most 64 A entries with one lane and
    # longer ones with the whole warp, 32 rows per warp: rows of 0, 1, 63, 64,
    # 65 and 700 entries side by side in one 32-row tile, the tile boundary
    # crossed, and the product against the oracle (per-row products, totals,
    # the product itself)
    from trident_b200 import panels
    rng = np.random.default_rng(17)
    lens = [0, 64, 65, 63, 1, 700, 0, 64] * 5 + [65] * 7
    n = 2000
    rp = np.zeros(len(lens) + 1, dtype=np.int64)
    rp[1:] = np.cumsum(lens)
    col = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens]).astype(np.int32)
    A = HostCSR(len(lens), n, rp, col, rng.uniform(-1, 1, size=col.size))
    B = random_csr(n, 300, density=0.02, seed=18)
    dA, dB = A.to_device(rowptr_bits=bits), B.to_device(rowptr_bits=bits)
    rm = oracle.row_mults(A, B)
    np.testing.assert_array_equal(panels.row_products(ctx, dA, dB).cpu().numpy(), rm)
    mults, upper = ops.spgemm_count(ctx, dA, dB)
    assert mults == int(rm.sum())
    assert upper == int(np.minimum(rm, B.ncols).sum())
    check_product(ops.spgemm(ctx, dA, dB), A, B)


def _launches(ctx):
    import ctypes as C

    from trident_b200._lib import lib
    n = C.c_int64()
    lib.tspg_ctx_stats(ctx.h, C.byref(n))
    return n.value


@pytest.mark.parametrize("bits,vbits", [(32, 64), (64, 64), (32, 32)])
def test_onepass_warp_rows(ctx, bits, vbits):
    # A one-shot product of at least 65536 rows multiplies its warp rows whole
    # in the symbolic launch (into a scratch), and the numeric launch copies
    # them into C: Galerkin A·P on 42^3 (74,088 rows of ~119 products) into
    # poisoned outputs, against the oracle.  The launch counts show the
    # one-pass kernels ran: the one-shot call has 3 scan launches, the
    # one-pass kernel, 3 launches for the rows sent back to the two-pass path
    # and the copy more than a plan's symbolic + numeric calls, which have
    # one operand-setting launch more
    R, A, P = workloads.galerkin_operands(n=42, pts=27, agg=3)
    assert A.nrows >= 1 << 16
    dA, dP = A.to_device(rowptr_bits=bits, val_bits=vbits), P.to_device(rowptr_bits=bits, val_bits=vbits)
    n0 = _launches(ctx)
    ops.spgemm(ctx, dA, dP)
    n1 = _launches(ctx)
    plan = ops.Plan(ctx, dA, dP)
    plan.numeric(dA, dP)
    plan.close()
    n2 = _launches(ctx)
    assert (n1 - n0) - (n2 - n1) == 7
    C1 = spgemm_poisoned(ctx, dA, dP)
    r32 = (lambda M: HostCSR(M.nrows, M.ncols, M.rowptr, M.col, M.val.astype(np.float32).astype(np.float64)))
    if vbits == 32:
        check_product(C1, r32(A), r32(P), tol=TOL32)
    else:
        check_product(C1, A, P)


def _vstack(*Ms):
    rp = [np.zeros(1, np.int64)]
    for M in Ms:
        rp.append(M.rowptr[1:].astype(np.int64) + rp[-1][-1])
    return HostCSR(sum(M.nrows for M in Ms), Ms[0].ncols, np.concatenate(rp),
                   np.concatenate([M.col for M in Ms]), np.concatenate([M.val for M in Ms]))


def test_onepass_mixed_row_classes(ctx):
    # Most rows one-pass (Galerkin A·P on 42^3, ~12 columns each) beside rows
    # of random entries that stay two-pass (40 entries: ~150 columns; 300 and
    # 700 entries: 128-, 256- and CTA-thread rows) and short ones, into
    # poisoned outputs
    R, A, P = workloads.galerkin_operands(n=42, pts=27, agg=3)
    rows = [A, random_csr(1500, A.ncols, per_row=40, seed=41), random_csr(300, A.ncols, per_row=300, seed=42),
            random_csr(100, A.ncols, per_row=700, seed=43), random_csr(500, A.ncols, per_row=2, seed=44)]
    Am = _vstack(*rows)
    check_product(spgemm_poisoned(ctx, Am.to_device(), P.to_device()), Am, P)


def test_onepass_rows_sent_back(ctx):
    # One-pass rows too large for a warp's full table (600 products each,
    # every B row starting on column 0, so all are candidates): those with
    # fewer than 32 columns finish in their 64-slot attempt, the others
    # (~500 columns) go back to the two-pass path within the same symbolic
    # launch sequence; 80,000 rows, half of each kind, into poisoned outputs
    rng = np.random.default_rng(51)
    rows_b = []
    for k in range(2000):
        span = 24 if k < 1000 else 2000
        rows_b.append(np.concatenate([[0], np.sort(rng.choice(np.arange(1, span), size=19, replace=False))]))
    rpb = np.concatenate([[0], np.cumsum([len(r) for r in rows_b])]).astype(np.int64)
    B = HostCSR(2000, 2000, rpb, np.concatenate(rows_b).astype(np.int32), rng.uniform(-1, 1, size=rpb[-1]))
    rows_a = [np.sort(rng.choice(1000, size=30, replace=False)) + (0 if i % 2 == 0 else 1000) for i in range(80000)]
    rpa = np.concatenate([[0], np.cumsum([30] * 80000)]).astype(np.int64)
    A = HostCSR(80000, 2000, rpa, np.concatenate(rows_a).astype(np.int32), rng.uniform(-1, 1, size=rpa[-1]))
    H = check_product(spgemm_poisoned(ctx, A.to_device(), B.to_device()), A, B)
    c = np.diff(H.rowptr)
    assert c[0::2].max() < 32 and c[1::2].min() >= 32


def test_onepass_skips_rows_without_repeats(ctx):
    # 80,000 uniform-random rows of 600 products (~590 columns): too large for
    # a warp's full table, and their B rows do not start on shared columns,
    # so they are no one-pass candidates and the product keeps the two-pass
    # path (no launch beyond the count-pass scan and the fold)
    A = random_csr(80000, 2000, per_row=30, seed=61)
    B = random_csr(2000, 20000, per_row=20, seed=62)
    dA, dB = A.to_device(), B.to_device()
    n0 = _launches(ctx)
    ops.spgemm(ctx, dA, dB)
    n1 = _launches(ctx)
    plan = ops.Plan(ctx, dA, dB)
    plan.numeric(dA, dB)
    plan.close()
    n2 = _launches(ctx)
    # 3 scan launches and the fold more; one operand-setting launch less
    assert (n1 - n0) - (n2 - n1) == 3
    check_product(spgemm_poisoned(ctx, dA, dB), A, B)


def test_onepass_without_workspace_budget():
    # A context whose workspace budget (16 MB) holds the product's row arrays
    # but not the one-pass workspace (~28 MB for the Galerkin A·P on 42^3):
    # the product takes the two-pass path, same result
    R, A, P = workloads.galerkin_operands(n=42, pts=27, agg=3)
    c = ops.Context(0, budget=16 << 20)
    try:
        dA, dP = A.to_device(), P.to_device()
        n0 = _launches(c)
        C1 = ops.spgemm(c, dA, dP)
        n1 = _launches(c)
        plan = ops.Plan(c, dA, dP)
        plan.numeric(dA, dP)
        plan.close()
        n2 = _launches(c)
        assert (n1 - n0) - (n2 - n1) == 3  # the scan and the fold only
        check_product(C1, A, P)
    finally:
        torch.cuda.synchronize()
        c.close()


def test_onepass_minority_folds_back(ctx):
    # R-MAT 17 A·A (131,072 rows): a tenth of the rows qualify for the
    # one-pass path, too few, so they go back to the warp class after their
    # bounds were written (the count pass's bounds cleared again)
    A = workloads.rmat(scale=17, edge_factor=16, seed=4)
    dA = A.to_device()
    check_product(spgemm_poisoned(ctx, dA, dA, flags=TSPG_F_B_SORTED), A, A)


def test_onepass_without_eligible_rows(ctx):
    # 70,000 rows of 600 products each (above the warp-row bound of the
    # symbolic phase): no one-pass row, so the count pass runs again with
    # every row two-pass
    A = random_csr(70000, 2000, per_row=30, seed=31)
    B = random_csr(2000, 1000, per_row=20, seed=32)
    check_product(spgemm_poisoned(ctx, A.to_device(), B.to_device()), A, B)


def test_shape_mismatch_rejected(ctx):
    A = random_csr(4, 5, density=0.5, seed=1).to_device()
    B = random_csr(6, 7, density=0.5, seed=2).to_device()
    with pytest.raises(TspgError) as e:
        ops.spgemm(ctx, A, B)
    assert e.value.status == TSPG_EINVAL


def test_sorted_flag_skips_check(ctx):
    A = workloads.uniform_rows(2048, 16, True, seed=7)
    dA = A.to_device()
    check_product(ops.spgemm(ctx, dA, dA, flags=TSPG_F_B_SORTED), A, A)


def test_dense_rows_wide_b_windowed(ctx):
    # ncols above the whole-row bitmap limit: DENSE rows take the windowed
    # sweep (sorted B with cursors, then unsorted B with rescans)
    n = 1_300_000
    B = random_csr(3000, n, per_row=40, seed=21)
    A = random_csr(6, 3000, per_row=600, seed=22)
    check_product(ops.spgemm(ctx, A.to_device(), B.to_device()), A, B)
    Bu = random_csr(3000, n, per_row=40, seed=23, sort=False)
    check_product(ops.spgemm(ctx, A.to_device(), Bu.to_device()), A, Bu)


def test_dense_rows_wide_b_long_rows_global_cursors(ctx):
    # windowed sweep with A rows longer than the shared cursor array (cursors
    # in global scratch) and a few hub rows of B (walked by one warp each)
    n = 1_200_000
    rng = np.random.default_rng(24)
    B = random_csr(12000, n, per_row=12, seed=25)
    hub_rows = [3, 777, 5000, 11999]
    rows = [np.sort(rng.choice(n, 6000, replace=False)) if i in hub_rows else
            B.col[B.rowptr[i]:B.rowptr[i + 1]] for i in range(B.nrows)]
    rp = np.zeros(B.nrows + 1, dtype=np.int64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate(rows).astype(np.int32)
    B = HostCSR(B.nrows, n, rp, col, rng.uniform(-1, 1, col.size))
    A = random_csr(3, B.nrows, per_row=9000, seed=26)
    check_product(ops.spgemm(ctx, A.to_device(), B.to_device()), A, B)


def test_mixed_rowptr_widths(ctx):
    A = random_csr(300, 200, density=0.05, seed=30)
    B = random_csr(200, 250, density=0.05, seed=31)
    check_product(ops.spgemm(ctx, A.to_device(rowptr_bits=32), B.to_device(rowptr_bits=64)), A, B)
    check_product(ops.spgemm(ctx, A.to_device(rowptr_bits=64), B.to_device(rowptr_bits=32)), A, B)
    p = ops.Plan(ctx, A.to_device(rowptr_bits=32), B.to_device(rowptr_bits=64))
    check_product(p.numeric(A.to_device(rowptr_bits=32), B.to_device(rowptr_bits=64)), A, B)
    p.close()


@pytest.mark.parametrize("lam", [6.0, 20.0, 40.0])
def test_uniform_rows_expand_sort_compress(ctx, lam):
    # Poisson rows of uniform-random columns have almost no repeated columns,
    # so warp, 128- and 256-thread rows take the expand-sort-compress form
    # (lam 40: ~1600 outputs per row, 256-thread rows)
    A, B = workloads.batched_product((3000, lam, 71, 72))
    check_product(ops.spgemm(ctx, A.to_device(), B.to_device()), A, B)
    r32 = lambda M: HostCSR(M.nrows, M.ncols, M.rowptr, M.col,
                            M.val.astype(np.float32).astype(np.float64))
    C32 = ops.spgemm(ctx, A.to_device(val_bits=32), B.to_device(val_bits=32))
    check_product(C32, r32(A), r32(B), tol=TOL32)


def test_row_panels_concatenate_to_the_product(ctx):
    """The row-panel split of the multi-GPU benchmark on one GPU: A's rows cut
    by equal products (tspg_spgemm_row_products), each panel multiplied as a
    view whose row offsets do not start at 0; the panels concatenate to the
    oracle's product."""
    from trident_b200 import panels
    from trident_b200.csr import DeviceCSR
    A = workloads.rmat(scale=12, edge_factor=16, seed=7)
    dA = A.to_device()
    rowf = panels.row_products(ctx, dA, dA).cpu().numpy()
    np.testing.assert_array_equal(rowf, oracle.row_mults(A, A))
    cuts = panels.panel_cuts(rowf, 3)
    parts = []
    for r in range(3):
        r0, r1 = panels.panel_rows(cuts, r)
        dP = DeviceCSR(r1 - r0, A.ncols, dA.rowptr[r0:r1 + 1], dA.col, dA.val,
                       nnz=int(A.rowptr[r1] - A.rowptr[r0]))
        H = ops.spgemm(ctx, dP, dA).to_host()
        parts.append((H.rowptr, H.col, H.val))
    rp, cj, cx = panels.assemble(parts, A.ncols)
    check_product(HostCSR(A.nrows, A.ncols, rp, cj, cx), A, A)


def _window_operands(val_dtype=np.float64):
    """Operands whose heavy rows take the column-window DENSE form (with the
    window threshold at 2^10 products): B has 40000 columns (windows of 16384:
    two full, one partial), 20 hub rows of 12000 sorted columns (segments
    longer than one thread's 8 loads: the warp pass), 4000 short rows, and
    5000 rows of 12 columns inside the first window (one A row takes all of
    them: more long segments than the queue holds); one A row has 9020 entries
    (cursors in global memory); in the last A row one pair of products
    cancels exactly and one product is -0.0 (both stay in the pattern)."""
    rng = np.random.default_rng(21)
    n = 40000
    rows = [np.sort(rng.choice(n, 12000, replace=False)) for _ in range(20)]
    rows += [np.sort(rng.choice(n, 10, replace=False)) for _ in range(4000)]
    rows += [np.sort(rng.choice(16384, 12, replace=False)) for _ in range(5000)]
    p0 = len(rows)
    rows += [np.array([7, 20000, 39999]), np.array([7, 39998])]
    brp = np.zeros(len(rows) + 1, np.int64)
    brp[1:] = np.cumsum([r.size for r in rows])
    bcol = np.concatenate(rows).astype(np.int32)
    bval = rng.uniform(-1, 1, bcol.size)
    bval[brp[p0]] = 0.5       # B[p0, 7]
    bval[brp[p0] + 1] = 0.0   # B[p0, 20000]
    bval[brp[p0 + 1]] = 0.5   # B[p0 + 1, 7]
    B = HostCSR(len(rows), n, brp, bcol, bval.astype(val_dtype).astype(np.float64))
    arows = [np.sort(np.concatenate([rng.choice(20, 3, replace=False), 20 + rng.choice(4000, 300, replace=False)]))
             for _ in range(12)]                    # hubs + short rows
    arows.append(np.arange(4020, 9020))             # 5000 long segments in window 0
    arows.append(np.arange(0, 9020))                # 9020 entries: cursors in global memory
    hub = next(h for h in range(20) if 7 not in rows[h] and 20000 not in rows[h])
    arows.append(np.array([hub, p0, p0 + 1]))      # -1 * 0.5 + 1 * 0.5 = 0 at column 7; -1 * 0.0 = -0.0
    arp = np.zeros(len(arows) + 1, np.int64)
    arp[1:] = np.cumsum([r.size for r in arows])
    acol = np.concatenate(arows).astype(np.int32)
    aval = rng.uniform(-1, 1, acol.size)
    aval[arp[-2] + 1], aval[arp[-2] + 2] = -1.0, 1.0
    A = HostCSR(len(arows), B.nrows, arp, acol, aval.astype(val_dtype).astype(np.float64))
    return A, B


@pytest.mark.parametrize("win,cluster", [(10, 0), (10, 2), (10, 4), (0, 0)])
def test_dense_window_form(win, cluster):
    """The column-window form (win = 10) in one CTA per row and on clusters of
    2 and 4 CTAs (the window in their distributed shared memory), and the rank
    form (win = 0), on the same heavy rows: all equal the oracle (structure
    bit-exact, values within 1e-12), including the exact cancellation and the
    -0.0 product."""
    c = ops.Context(0)
    c.set_tuning({"dense_win_log2": win, "dense_win_cluster": cluster, "num_lim": [1, 1, 1, 1],
                  "sym_lim": [1, 1, 1, 1]})
    A, B = _window_operands()
    H = check_product(spgemm_poisoned(c, A.to_device(), B.to_device(), flags=TSPG_F_B_SORTED), A, B)
    r = A.nrows - 1
    row = H.col[H.rowptr[r]:H.rowptr[r + 1]]
    assert 7 in row and H.val[H.rowptr[r] + int(np.searchsorted(row, 7))] == 0.0
    assert 20000 in row
    torch.cuda.synchronize()
    c.close()


@pytest.mark.parametrize("cluster", [0, 2])
def test_dense_window_form_fp32_and_addend(cluster):
    """FP32 twin, and the fused accumulate (the addend's entries join every
    window), in one CTA and on a cluster."""
    from trident_b200._lib import TSPG_F_ACC_FUSE
    c = ops.Context(0)
    c.set_tuning({"dense_win_log2": 10, "dense_win_cluster": cluster, "num_lim": [1, 1, 1, 1],
                  "sym_lim": [1, 1, 1, 1]})
    A, B = _window_operands(np.float32)
    C32 = spgemm_poisoned(c, A.to_device(val_bits=32), B.to_device(val_bits=32), flags=TSPG_F_B_SORTED)
    check_product(C32, A, B, tol=TOL32)
    E = random_csr(A.nrows, B.ncols, per_row=3000, seed=31)
    junk = torch.full((8 << 20,), -7, dtype=torch.int64, device="cuda")  # blocks the allocator hands back
    del junk
    D = ops.sp_mma(c, A.to_device(), B.to_device(), E.to_device(), flags=TSPG_F_ACC_FUSE)
    rp, cj, cx, ca = oracle.spgemm(A, B)
    S = oracle.spadd(HostCSR(A.nrows, B.ncols, rp, cj, cx), E)
    H = D.to_host()
    np.testing.assert_array_equal(H.rowptr, S[0])
    np.testing.assert_array_equal(H.col, S[1])
    assert np.all(np.abs(H.val - S[2]) <= 1e-12 * np.maximum(1.0, np.abs(S[2])) * 8)
    torch.cuda.synchronize()
    c.close()
