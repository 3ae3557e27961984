"""CPU: the oracle against the reference's known answers and independent checks."""
import json
import os

import numpy as np
import pytest

import oracle
from helpers import random_csr
from trident_b200 import workloads

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _kat():
    with open(os.path.join(GOLD, "kat_bitmask.json")) as fh:
        return json.load(fh)


def test_gen_bitmask_kats():
    for case in _kat()["gen_bitmask"]:
        ptr = np.array(case["ptr"])
        assert list(oracle.bitmask_gen(ptr, len(ptr) - 1)) == case["mask"]


def test_intersect_kat():
    for case in _kat()["intersect_bitmasks"]:
        assert list(oracle.bitmask_and(case["a"], case["b"])) == case["out"]


def test_tmp_test1_pack_kat():
    k = _kat()["tmp_test1"]
    ptr, idx, val = oracle.pack(np.array(k["ptr"]), np.array(k["col"]), np.array(k["val"]),
                                np.array(k["mask"], dtype=np.uint8))
    assert list(ptr) == k["expect_ptr"]
    assert list(idx) == k["expect_col"]
    assert list(val) == k["expect_val"]
    assert len(idx) == k["expect_nnz"]


def _dense(M):
    D = np.zeros((M.nrows, M.ncols))
    for i in range(M.nrows):
        for p in range(M.rowptr[i], M.rowptr[i + 1]):
            D[i, M.col[p]] += M.val[p]
    return D


def _pattern(M):
    D = np.zeros((M.nrows, M.ncols), dtype=bool)
    for i in range(M.nrows):
        D[i, M.col[M.rowptr[i]:M.rowptr[i + 1]]] = True
    return D


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_spgemm_vs_dense(seed):
    A = random_csr(37, 29, density=0.15, seed=seed)
    B = random_csr(29, 41, density=0.2, seed=seed + 100)
    rp, cj, cx, ca = oracle.spgemm(A, B)
    P = (_pattern(A).astype(int) @ _pattern(B).astype(int)) > 0
    D = _dense(A) @ _dense(B)
    for i in range(A.nrows):
        cols = cj[rp[i]:rp[i + 1]]
        assert list(cols) == sorted(np.nonzero(P[i])[0])
        np.testing.assert_allclose(cx[rp[i]:rp[i + 1]], D[i, cols], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(ca, np.abs(ca))


def test_structural_zero_kept():
    from trident_b200.csr import HostCSR
    A = HostCSR(1, 2, np.array([0, 2]), np.array([0, 1], np.int32), np.array([1.0, 1.0]))
    B = HostCSR(2, 1, np.array([0, 1, 2]), np.array([0, 0], np.int32), np.array([1.0, -1.0]))
    rp, cj, cx, ca = oracle.spgemm(A, B)
    assert list(rp) == [0, 1] and list(cj) == [0] and cx[0] == 0.0 and ca[0] == 2.0


def test_spgemm_row_range_matches_full():
    A = random_csr(60, 50, density=0.1, seed=5)
    B = random_csr(50, 70, density=0.1, seed=6)
    rp, cj, cx, _ = oracle.spgemm(A, B)
    rp2, cj2, cx2, _ = oracle.spgemm(A, B, 17, 44)
    np.testing.assert_array_equal(rp2, rp[17:45] - rp[17])
    np.testing.assert_array_equal(cj2, cj[rp[17]:rp[44]])
    np.testing.assert_array_equal(cx2, cx[rp[17]:rp[44]])


def test_spadd_vs_dense():
    A = random_csr(30, 40, density=0.2, seed=3)
    B = random_csr(30, 40, density=0.2, seed=4)
    cp, cj, cx = oracle.spadd(A, B)
    P = _pattern(A) | _pattern(B)
    D = _dense(A) + _dense(B)
    for i in range(30):
        cols = cj[cp[i]:cp[i + 1]]
        assert list(cols) == list(np.nonzero(P[i])[0])
        np.testing.assert_allclose(cx[cp[i]:cp[i + 1]], D[i, cols], rtol=1e-15, atol=0)


def test_pack_keeps_masked_segments():
    M = random_csr(50, 20, density=0.3, seed=9)
    rng = np.random.default_rng(1)
    mask = rng.integers(0, 256, size=(50 + 7) // 8, dtype=np.uint8)
    ptr, idx, val = oracle.pack(M.rowptr, M.col, M.val, mask)
    o = 0
    for r in range(50):
        seg = slice(M.rowptr[r], M.rowptr[r + 1])
        keep = (mask[r // 8] >> (r % 8)) & 1
        n = (M.rowptr[r + 1] - M.rowptr[r]) if keep else 0
        assert ptr[r + 1] - ptr[r] == n
        if keep:
            np.testing.assert_array_equal(idx[o:o + n], M.col[seg])
            np.testing.assert_array_equal(val[o:o + n], M.val[seg])
        o += n


def test_bmtx_fixture_digests():
    import hashlib
    with open(os.path.join(GOLD, "oracle_bmtx.json")) as fh:
        gold = json.load(fh)
    for name, g in gold.items():
        A = workloads.read_bmtx(os.path.join(GOLD, name))
        assert A.nrows == g["nrows"] and A.nnz == g["nnz_A"]
        rp, cj, cx, ca = oracle.spgemm(A, A)
        assert int(rp[-1]) == g["nnz_C"]
        assert hashlib.sha256(np.ascontiguousarray(rp).tobytes()).hexdigest() == g["rowptr_sha256"]
        assert hashlib.sha256(np.ascontiguousarray(cj).tobytes()).hexdigest() == g["col_sha256"]
        assert abs(float(np.sum(cx)) - g["val_sum"]) <= 1e-9 * abs(g["val_sum"])


def test_bmtx_values_vs_scipy():
    A = workloads.read_bmtx(os.path.join(GOLD, "n1024.bmtx"))
    rp, cj, cx, _ = oracle.spgemm(A, A)
    S = (A.to_scipy() @ A.to_scipy()).tocsr()
    S.sort_indices()
    # fixture values are in [1, 2], so no cancellation: scipy keeps every entry
    np.testing.assert_array_equal(S.indptr, rp)
    np.testing.assert_array_equal(S.indices, cj)
    np.testing.assert_allclose(S.data, cx, rtol=1e-13)


def test_coo_to_csx_follows_reference_steps():
    # the reference's host builder, step by step in plain Python: sort the
    # triples by row, count rows into ptr[r + 1], inclusive scan, emit in
    # sorted order; its order inside a row is unspecified (std::sort), so the
    # rows are compared as multisets and the oracle's order checked separately
    rng = np.random.default_rng(11)
    n, m, nnz = 40, 30, 500
    r = rng.integers(0, n, nnz)
    c = rng.integers(0, m, nnz)
    c[:50] = c[50:100]
    r[:50] = r[50:100]  # repeated coordinates
    v = rng.uniform(-1, 1, nnz)
    trip = sorted(zip(r.tolist(), c.tolist(), v.tolist()), key=lambda t: t[0])
    ptr = [0] * (n + 1)
    for t in trip:
        ptr[t[0] + 1] += 1
    for i in range(n):
        ptr[i + 1] += ptr[i]
    optr, ocol, oval = oracle.coo_to_csx(n, r, c, v)
    assert optr.tolist() == ptr
    for i in range(n):
        want = sorted((t[1], t[2]) for t in trip if t[0] == i)
        got = sorted(zip(ocol[ptr[i]:ptr[i + 1]].tolist(), oval[ptr[i]:ptr[i + 1]].tolist()))
        assert got == want
        seg = ocol[ptr[i]:ptr[i + 1]]
        assert np.all(np.diff(seg) >= 0)
    # equal coordinates keep their input order
    pos = np.lexsort((np.arange(nnz), c, r))
    np.testing.assert_array_equal(oval, v[pos])


def test_mcl_updates_follow_reference_loops():
    # prune / normalize / inflation of the reference's MCL driver, written out
    # as its host loops (row by row, in entry order) in plain Python
    rng = np.random.default_rng(12)
    n = 30
    rowptr = [0]
    col, val = [], []
    for i in range(n):
        k = int(rng.integers(0, 6))
        cs = sorted(rng.choice(n, k, replace=False).tolist())
        col += cs
        val += rng.uniform(0, 1, k).tolist()
        rowptr.append(len(col))
    val[rowptr[3]:rowptr[4]] = [0.0] * (rowptr[4] - rowptr[3])  # a row summing to 0

    def normalize(v):
        out = list(v)
        for i in range(n):
            s = sum(v[rowptr[i]:rowptr[i + 1]])
            for j in range(rowptr[i], rowptr[i + 1]):
                out[j] = v[j] / s if s > 1e-20 else 0.0
        return out

    want = normalize([x ** 2.0 for x in val])
    np.testing.assert_allclose(oracle.mcl_inflate(rowptr, val, 2.0), want, rtol=1e-14)
    np.testing.assert_allclose(oracle.mcl_normalize(rowptr, val), normalize(val), rtol=1e-14)
    tol = 0.3
    prp, pcol, pval = [0], [], []
    for i in range(n):
        for j in range(rowptr[i], rowptr[i + 1]):
            if abs(val[j]) > tol:
                pcol.append(col[j])
                pval.append(val[j])
        prp.append(len(pcol))
    grp, gcol, gval = oracle.mcl_prune(rowptr, col, val, tol)
    assert grp.tolist() == prp and gcol.tolist() == pcol and gval.tolist() == pval


def test_summa_tiles_cover_the_matrix():
    # the host-side q x q tile cut of the SUMMA emulation: every entry lands in
    # exactly one tile, rebased, and the tiles put back together give the matrix
    import scipy.sparse as sp
    from trident_b200 import summa
    A = workloads.rmat(scale=9, edge_factor=8, seed=4)
    q = 4
    tiles, rb, cb = summa.cut_tiles(A, q)
    assert rb[0] == cb[0] == 0 and rb[-1] == A.nrows and cb[-1] == A.ncols
    blocks = [[sp.csr_matrix((t.val, t.col, t.rowptr), shape=(rb[i + 1] - rb[i], cb[j + 1] - cb[j]))
               for j, t in enumerate(row)] for i, row in enumerate(tiles)]
    M = sp.bmat(blocks, format="csr")
    M.sort_indices()
    assert sum(t.nnz for row in tiles for t in row) == A.nnz
    np.testing.assert_array_equal(M.indptr, A.rowptr)
    np.testing.assert_array_equal(M.indices, A.col)
    np.testing.assert_array_equal(M.data, A.val)


def test_transpose_vs_scipy_and_host_generator():
    """The oracle's transpose (the checker of the device transpose) equals
    scipy's and keeps entries of a column in row order."""
    from helpers import random_csr
    M = random_csr(300, 200, density=0.03, seed=9)
    rp, col, val = oracle.transpose(M)
    T = M.to_scipy().T.tocsr()
    T.sort_indices()
    np.testing.assert_array_equal(rp, T.indptr)
    np.testing.assert_array_equal(col, T.indices)
    np.testing.assert_array_equal(val, T.data)
    R = workloads.transpose(M)
    np.testing.assert_array_equal(R.rowptr, rp)
    np.testing.assert_array_equal(R.col, col)
