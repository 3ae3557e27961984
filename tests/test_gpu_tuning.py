"""GPU: the row binning changes speed only — results equal the oracle's under
non-default tunings, invalid tunings are refused, batches re-capture."""
import pytest

from helpers import check_product, random_csr
from trident_b200 import ops, tune, workloads
from trident_b200._lib import TSPG_EINVAL, TspgError

pytestmark = pytest.mark.gpu

TUNINGS = [
    {"sym_lim": [128, 1024, 2048, 8192], "num_lim": [128, 512, 1024, 4096], "hash_load": 4, "dense_win_log2": 17, "dense_win_fill_log2": 4, "dense_win_cluster": 0},
    {"sym_lim": [512, 512, 512, 512], "num_lim": [256, 256, 256, 256], "hash_load": 2, "dense_win_log2": 0, "dense_win_fill_log2": 4, "dense_win_cluster": 0},
    {"sym_lim": [1, 1, 1, 1], "num_lim": [1, 1, 1, 1], "hash_load": 8, "dense_win_log2": 10, "dense_win_fill_log2": 12, "dense_win_cluster": 2},
]


@pytest.fixture
def tctx():
    c = ops.Context(0)
    yield c
    c.close()


def test_invalid_tuning_refused(tctx):
    for bad in ({"num_lim": [1024, 1024, 2048, 8192]}, {"sym_lim": [512, 256, 4096, 24576]},
                {"hash_load": 3}, {"num_lim": [0, 1024, 2048, 8192]}, {"dense_win_log2": 9}):
        with pytest.raises(TspgError) as e:
            tctx.set_tuning(bad)
        assert e.value.status == TSPG_EINVAL
    assert tctx.get_tuning() == tune.default_tuning()


@pytest.mark.parametrize("t", TUNINGS)
def test_results_do_not_depend_on_tuning(tctx, t):
    tctx.set_tuning(t)
    assert tctx.get_tuning() == t
    R = workloads.rmat(scale=12, edge_factor=16, seed=3)
    check_product(ops.spgemm(tctx, R.to_device(), R.to_device()), R, R)
    A = random_csr(3000, 2500, per_row=14, seed=8)
    B = random_csr(2500, 4000, per_row=9, seed=9)
    check_product(ops.spgemm(tctx, A.to_device(), B.to_device()), A, B)


def test_batch_recaptures_on_tuning_change(tctx):
    specs = workloads.batched_specs(count=6, seed=9, rows_lo=300, rows_hi=8000)
    hosts, keep = [], []
    b = ops.Batch(tctx)
    for spec in specs:
        A, B = workloads.batched_product(spec)
        dA, dB = A.to_device(), B.to_device()
        hosts.append((A, B))
        keep.append((dA, dB))
        b.add(dA, dB)
    n0 = b.run()
    tctx.set_tuning(TUNINGS[0])
    assert b.run() == n0
    for i, (A, B) in enumerate(hosts):
        check_product(b.result(i), A, B)
    b.close()


@pytest.mark.parametrize("t", TUNINGS[1:])
def test_batch_results_do_not_depend_on_tuning(tctx, t):
    """Products of different shapes in one batch, with most rows (or all) in
    the DENSE forms: the rank-form kernel takes rows of several products,
    each with its own column count."""
    tctx.set_tuning(t)
    specs = workloads.batched_specs(count=5, seed=21, rows_lo=200, rows_hi=5000)
    hosts, keep = [], []
    b = ops.Batch(tctx)
    for spec in specs:
        A, B = workloads.batched_product(spec)
        dA, dB = A.to_device(), B.to_device()
        hosts.append((A, B))
        keep.append((dA, dB))
        b.add(dA, dB)
    b.run()
    for i, (A, B) in enumerate(hosts):
        check_product(b.result(i), A, B)
    b.close()


def test_plan_numeric_with_dense_rows(tctx):
    """The plan API's numeric re-runs (new values, same structure) with every
    row above 256 outputs in the DENSE forms."""
    tctx.set_tuning(TUNINGS[1])
    R = workloads.rmat(scale=12, edge_factor=16, seed=5)
    dR = R.to_device()
    plan = ops.Plan(tctx, dR, dR)
    try:
        check_product(plan.numeric(dR, dR), R, R)
        R.val[:] = R.val * -0.5 + 0.25
        dR2 = R.to_device()
        check_product(plan.numeric(dR2, dR2), R, R)
    finally:
        plan.close()
