"""GPU parity: merge (spadd, sp_mma) and the bitmask pack/unpack."""
import json
import os

import numpy as np
import pytest
import torch

import oracle
from helpers import check_product, check_sum, random_csr
from trident_b200 import ops, workloads
from trident_b200._lib import TSPG_COLS, TSPG_F_ACC_FUSE, TSPG_F_ACC_SPLIT, TSPG_ROWS
from trident_b200.csr import HostCSR

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _kat():
    with open(os.path.join(GOLD, "kat_bitmask.json")) as fh:
        return json.load(fh)


@pytest.mark.parametrize("seed", [0, 1])
def test_spadd(ctx, seed):
    A = random_csr(3000, 5000, density=0.01, seed=seed)
    B = random_csr(3000, 5000, density=0.01, seed=seed + 10)
    check_sum(ops.spadd(ctx, A.to_device(), B.to_device()), A, B)


def test_spadd_mixed_rowptr_and_empty(ctx):
    A = random_csr(200, 300, density=0.05, seed=2)
    B = random_csr(200, 300, density=0.0, seed=3)
    check_sum(ops.spadd(ctx, A.to_device(rowptr_bits=32), B.to_device(rowptr_bits=64), rowptr_bits=32), A, B)
    check_sum(ops.spadd(ctx, B.to_device(), A.to_device()), B, A)


def test_spadd_long_rows(ctx):
    A = random_csr(4, 200000, per_row=50000, seed=4)
    B = random_csr(4, 200000, per_row=60000, seed=5)
    check_sum(ops.spadd(ctx, A.to_device(), B.to_device()), A, B)


def test_spadd_heavy_and_light_rows(ctx):
    # rows merged by a CTA (above 4096 entries together) next to warp rows:
    # full overlap, one side empty, disjoint interleaved, partial overlap
    n = 50000
    rng = np.random.default_rng(6)
    light = random_csr(300, n, density=0.0005, seed=7)
    lightB = random_csr(300, n, density=0.0005, seed=8)
    full = np.sort(rng.choice(n, 10000, replace=False))
    rowsA = [full, np.sort(rng.choice(n, 5000, replace=False)), np.zeros(0, np.int64),
             np.arange(0, 12000, 2), np.sort(rng.choice(n, 3000, replace=False))]
    rowsB = [full, np.zeros(0, np.int64), np.sort(rng.choice(n, 8000, replace=False)),
             np.arange(1, 12000, 2), np.sort(rng.choice(n, 3000, replace=False))]

    def build(heavy_rows, L):
        rows = heavy_rows + [L.col[L.rowptr[i]:L.rowptr[i + 1]] for i in range(L.nrows)]
        rp = np.zeros(len(rows) + 1, dtype=np.int64)
        rp[1:] = np.cumsum([len(r) for r in rows])
        col = np.concatenate(rows).astype(np.int32)
        return HostCSR(len(rows), n, rp, col, rng.uniform(-1, 1, col.size))
    A, B = build(rowsA, light), build(rowsB, lightB)
    check_sum(ops.spadd(ctx, A.to_device(), B.to_device()), A, B)
    check_sum(ops.spadd(ctx, B.to_device(rowptr_bits=32), A.to_device()), B, A)


def test_sp_mma_accumulates_stages(ctx):
    # C = sum_q A_q B_q over 3 stages, as a SUMMA stage loop does
    As = [random_csr(400, 300, density=0.02, seed=20 + q) for q in range(3)]
    Bs = [random_csr(300, 500, density=0.02, seed=30 + q) for q in range(3)]
    C = None
    ref = None
    for A, B in zip(As, Bs):
        C = ops.sp_mma(ctx, A.to_device(), B.to_device(), C)
        rp, cj, cx, _ = oracle.spgemm(A, B)
        prod = HostCSR(A.nrows, B.ncols, rp, cj, cx)
        if ref is None:
            ref = prod
        else:
            cp, cj2, cx2 = oracle.spadd(prod, ref)
            ref = HostCSR(A.nrows, B.ncols, cp, cj2, cx2)
    H = C.to_host()
    np.testing.assert_array_equal(H.rowptr, ref.rowptr)
    np.testing.assert_array_equal(H.col, ref.col)
    np.testing.assert_allclose(H.val, ref.val, rtol=1e-12, atol=1e-12)


def _acc_reference(A, B, E):
    """E + A·B: E canonicalised (rows sorted, duplicates summed), then the
    oracle's union merge with the oracle's product."""
    import scipy.sparse as sp
    rp, cj, cx, _ = oracle.spgemm(A, B)
    P = HostCSR(A.nrows, B.ncols, rp, cj, cx)
    S = sp.csr_matrix((E.val, E.col, E.rowptr), shape=(E.nrows, E.ncols))
    S.sum_duplicates()
    S.sort_indices()
    Ec = HostCSR(E.nrows, E.ncols, S.indptr.astype(np.int64), S.indices.astype(np.int32), S.data)
    cp, cj2, cx2 = oracle.spadd(P, Ec)
    return HostCSR(A.nrows, B.ncols, cp, cj2, cx2)


def _check_acc(C, ref):
    H = C.to_host()
    np.testing.assert_array_equal(H.rowptr.astype(np.int64), ref.rowptr)
    np.testing.assert_array_equal(H.col, ref.col)
    np.testing.assert_allclose(H.val, ref.val, rtol=1e-12, atol=1e-11)


@pytest.mark.parametrize("mode", [TSPG_F_ACC_FUSE, TSPG_F_ACC_SPLIT])
def test_sp_mma_fused_all_row_forms(ctx, mode):
    # C_in joins every row form: R-MAT rows (warp ... DENSE), rows where A is
    # empty but C_in is not, and C_in rows unsorted with repeated columns
    # (the split form merges, so its C_in must be canonical)
    R = workloads.rmat(scale=12, edge_factor=16, seed=8)
    E = random_csr(R.nrows, R.ncols, density=0.003, seed=10)
    _check_acc(ops.sp_mma(ctx, R.to_device(), R.to_device(), E.to_device(), flags=mode),
               _acc_reference(R, R, E))
    if mode != TSPG_F_ACC_FUSE:
        return
    A0 = random_csr(500, 400, density=0.01, seed=11)
    cut = A0.rowptr[100]  # rows 0..99 of A emptied
    rp = np.concatenate([np.zeros(100, np.int64), A0.rowptr[100:] - cut])
    A = HostCSR(A0.nrows, A0.ncols, rp, A0.col[cut:], A0.val[cut:])
    B = random_csr(400, 700, density=0.02, seed=12)
    Ed = random_csr(500, 700, per_row=30, seed=13, sort=False, dup=True)
    _check_acc(ops.sp_mma(ctx, A.to_device(), B.to_device(), Ed.to_device(), flags=mode),
               _acc_reference(A, B, Ed))


def test_sp_mma_fused_wide_b(ctx):
    # the windowed DENSE form (ncols above the whole-row bitmap) with an addend
    n = 1_250_000
    B = random_csr(2000, n, per_row=30, seed=14)
    A = random_csr(5, 2000, per_row=900, seed=15)
    E = random_csr(5, n, per_row=5000, seed=16)
    _check_acc(ops.sp_mma(ctx, A.to_device(), B.to_device(), E.to_device(), flags=TSPG_F_ACC_FUSE),
               _acc_reference(A, B, E))


def test_gen_bitmask_kats(ctx):
    for case in _kat()["gen_bitmask"]:
        for bits, dt in ((32, torch.int32), (64, torch.int64)):
            ptr = torch.tensor(case["ptr"], dtype=dt, device="cuda")
            m = ops.gen_bitmask(ctx, ptr, len(case["ptr"]) - 1)
            assert m.cpu().tolist() == case["mask"]


def test_intersect_kat(ctx):
    for case in _kat()["intersect_bitmasks"]:
        a = torch.tensor(case["a"], dtype=torch.uint8, device="cuda")
        b = torch.tensor(case["b"], dtype=torch.uint8, device="cuda")
        assert ops.intersect_bitmasks(ctx, a, b).cpu().tolist() == case["out"]


def test_tmp_test1_compress_kat(ctx):
    k = _kat()["tmp_test1"]
    M = HostCSR(8, 11, np.array(k["ptr"]), np.array(k["col"], np.int32), np.array(k["val"]))
    mask = torch.tensor(k["mask"], dtype=torch.uint8, device="cuda")
    for vb in (64, 32):
        buf, kept = ops.compress(ctx, M.to_device(val_bits=vb), mask)
        assert kept == k["expect_nnz"]
        U = ops.unpack(buf, 8, 11, kept, TSPG_ROWS, val_bits=vb, ptr_bits=32)
        assert U.rowptr.cpu().tolist() == k["expect_ptr"]
        assert U.col.cpu().tolist() == k["expect_col"]
        assert U.val.cpu().tolist() == k["expect_val"]


@pytest.mark.parametrize("n", [1, 7, 8, 31, 33, 1000, 100003])
def test_gen_and_random(ctx, n):
    rng = np.random.default_rng(n)
    ptr = np.concatenate([[0], np.cumsum(rng.integers(0, 2, size=n))])
    m = ops.gen_bitmask(ctx, torch.tensor(ptr, device="cuda"), n)
    np.testing.assert_array_equal(m.cpu().numpy(), oracle.bitmask_gen(ptr, n))
    a = rng.integers(0, 256, size=n, dtype=np.uint8)
    b = rng.integers(0, 256, size=n, dtype=np.uint8)
    ta, tb = torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda")
    np.testing.assert_array_equal(ops.intersect_bitmasks(ctx, ta, tb).cpu().numpy(), a & b)
    # unaligned views take the byte path
    np.testing.assert_array_equal(ops.intersect_bitmasks(ctx, ta[1:], tb[1:]).cpu().numpy(), (a & b)[1:])


@pytest.mark.parametrize("major", [TSPG_ROWS, TSPG_COLS])
@pytest.mark.parametrize("ptr_bits", [32, 64])
def test_pack_roundtrip_random(ctx, major, ptr_bits):
    M = random_csr(5000, 3000, density=0.003, seed=7)
    rng = np.random.default_rng(8)
    length = 5000
    mask = rng.integers(0, 256, size=(length + 7) // 8, dtype=np.uint8)
    # a CSC tile is the same arrays read column-major: nrows/ncols swap roles
    nrows, ncols = (5000, 3000) if major == TSPG_ROWS else (3000, 5000)
    D = M.to_device(rowptr_bits=ptr_bits)
    D.nrows, D.ncols = nrows, ncols
    buf, kept = ops.compress(ctx, D, torch.tensor(mask, device="cuda"), major)
    optr, oidx, oval = oracle.pack(M.rowptr, M.col, M.val, mask)
    assert kept == len(oidx)
    U = ops.unpack(buf, nrows, ncols, kept, major, val_bits=64, ptr_bits=ptr_bits)
    np.testing.assert_array_equal(U.rowptr.cpu().numpy().astype(np.int64), optr)
    np.testing.assert_array_equal(U.col.cpu().numpy(), oidx)
    np.testing.assert_array_equal(U.val.cpu().numpy(), oval)  # bit-exact copy
    # unpack(pack(T, m)) == T restricted to m
    H = U.to_host()
    for r in range(0, length, 37):
        keep = (mask[r // 8] >> (r % 8)) & 1
        seg = slice(M.rowptr[r], M.rowptr[r + 1])
        got = H.col[H.rowptr[r]:H.rowptr[r + 1]]
        np.testing.assert_array_equal(got, M.col[seg] if keep else M.col[seg][:0])


def test_pack_all_and_none(ctx):
    M = random_csr(64, 64, density=0.2, seed=3)
    D = M.to_device()
    full = torch.full((8,), 255, dtype=torch.uint8, device="cuda")
    buf, kept = ops.compress(ctx, D, full)
    assert kept == M.nnz
    U = ops.unpack(buf, 64, 64, kept).to_host()
    np.testing.assert_array_equal(U.col, M.col)
    np.testing.assert_array_equal(U.val, M.val)
    buf, kept = ops.compress(ctx, D, torch.zeros(8, dtype=torch.uint8, device="cuda"))
    assert kept == 0
    assert ops.unpack(buf, 64, 64, 0).rowptr.cpu().tolist() == [0] * 65


def test_packed_tile_multiplies_like_masked_tile(ctx):
    # the SUMMA use: packing A's columns / B's rows by the intersected masks
    # leaves the product unchanged
    A = random_csr(300, 256, density=0.03, seed=40)
    B = random_csr(256, 200, density=0.03, seed=41)
    dB = B.to_device()
    rowmask = ops.gen_bitmask(ctx, dB.rowptr, 256)
    buf, kept = ops.compress(ctx, dB, rowmask)
    Bp = ops.unpack(buf, 256, 200, kept)
    check_product(ops.spgemm(ctx, A.to_device(), Bp), A, B)
