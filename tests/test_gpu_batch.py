"""GPU parity: the batched persistent path against the oracle and the plain path."""
import numpy as np
import pytest
import torch

from helpers import check_product, random_csr
from trident_b200 import ops, workloads

pytestmark = pytest.mark.gpu


def test_batch_mixed_sizes_match_oracle(ctx):
    specs = workloads.batched_specs(count=12, seed=5, rows_lo=300, rows_hi=20000)
    hosts, devs = [], []
    b = ops.Batch(ctx)
    for spec in specs:
        A, B = workloads.batched_product(spec)
        dA, dB = A.to_device(), B.to_device()
        hosts.append((A, B))
        devs.append((dA, dB))
        b.add(dA, dB)
    total = b.run()
    got = 0
    for i, (A, B) in enumerate(hosts):
        H = check_product(b.result(i), A, B)
        got += H.nnz
    assert got == total
    b.close()


def test_batch_replay_and_heavy_rows(ctx):
    # includes an R-MAT square (DENSE rows) next to tiny products; run twice
    # (the second run replays the captured graphs)
    R = workloads.rmat(scale=12, edge_factor=16, seed=4)
    small = [random_csr(50, 40, density=0.1, seed=s) for s in range(3)]
    smallB = [random_csr(40, 60, density=0.1, seed=10 + s) for s in range(3)]
    b = ops.Batch(ctx)
    pairs = [(R, R)] + list(zip(small, smallB))
    keep = []
    for A, B in pairs:
        dA, dB = A.to_device(), B.to_device()
        keep.append((dA, dB))
        b.add(dA, dB)
    for _ in range(2):
        b.run()
        for i, (A, B) in enumerate(pairs):
            check_product(b.result(i), A, B)
    b.close()


def test_batch_matches_plain_calls(ctx):
    pairs = [(workloads.poisson_rows(3000, 12.0, s), workloads.poisson_rows(3000, 12.0, s + 100)) for s in range(4)]
    b = ops.Batch(ctx)
    keep = []
    for A, B in pairs:
        dA, dB = A.to_device(), B.to_device()
        keep.append((dA, dB))
        b.add(dA, dB)
    b.run()
    for i, (dA, dB) in enumerate(keep):
        P = ops.spgemm(ctx, dA, dB).to_host()
        Q = b.result(i).to_host()
        np.testing.assert_array_equal(P.rowptr, Q.rowptr)
        np.testing.assert_array_equal(P.col, Q.col)
        np.testing.assert_allclose(P.val, Q.val, rtol=1e-12, atol=1e-14)
    b.close()


def test_batch_with_empty_products(ctx):
    from trident_b200.csr import HostCSR
    E = HostCSR(0, 5, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0))
    Z = HostCSR(7, 5, np.zeros(8, np.int64), np.zeros(0, np.int32), np.zeros(0))
    B = random_csr(5, 9, density=0.5, seed=1)
    A = random_csr(7, 5, density=0.5, seed=2)
    b = ops.Batch(ctx)
    keep = [(E.to_device(), B.to_device()), (Z.to_device(), B.to_device()), (A.to_device(), B.to_device())]
    for dA, dB in keep:
        b.add(dA, dB)
    b.run()
    assert b.result(0).rowptr.cpu().tolist() == [0]
    assert b.result(1).rowptr.cpu().tolist() == [0] * 8
    check_product(b.result(2), A, B)
    b.close()


def test_batch_reuse_grows_rows_not_nnz(ctx):
    # a second composition with more rows but fewer nonzeros reuses the slab
    b = ops.Batch(ctx)
    A1 = workloads.poisson_rows(2000, 30.0, 1)
    d1 = (A1.to_device(), A1.to_device())
    b.add(*d1)
    b.run()
    check_product(b.result(0), A1, A1)
    b.clear()
    A2 = workloads.poisson_rows(30000, 1.5, 2)
    d2 = (A2.to_device(), A2.to_device())
    b.add(*d2)
    b.add(*d1)
    b.run()
    check_product(b.result(0), A2, A2)
    check_product(b.result(1), A1, A1)
    b.close()


def test_batch_count_matches_oracle(ctx):
    # per-product flop counts of one launch, mixed offset widths, empty
    # products and long rows among short ones
    from trident_b200.csr import HostCSR
    import oracle
    E = HostCSR(0, 5, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0))
    B5 = random_csr(5, 9, density=0.5, seed=1)
    pairs = [(workloads.poisson_rows(3000, 12.0, 3), workloads.poisson_rows(3000, 12.0, 4), 32, 64),
             (E, B5, 64, 64),
             (random_csr(40, 3000, per_row=900, seed=5), random_csr(3000, 700, per_row=20, seed=6), 64, 32),
             (workloads.rmat(scale=10, edge_factor=16, seed=7), None, 32, 32)]
    b = ops.Batch(ctx)
    keep = []
    for A, B, ra, rb in pairs:
        B = A if B is None else B
        dA, dB = A.to_device(rowptr_bits=ra), B.to_device(rowptr_bits=rb)
        keep.append((A, B, dA, dB))
        b.add(dA, dB)
    got = b.count()
    for (A, B, dA, dB), (m, u) in zip(keep, got):
        rm = oracle.row_mults(A, B)
        assert m == int(rm.sum())
        assert u == int(np.minimum(rm, B.ncols).sum())
        assert (m, u) == ops.spgemm_count(ctx, dA, dB)
    b.close()
