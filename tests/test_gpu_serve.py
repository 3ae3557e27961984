"""GPU: the continuous-batching server.  Each result must be the same alone
(a plain call) and in the mix (batched with other requests): both equal the
oracle's product, structure bit-exact and FP64 values within
1e-12 * max(|y|, sum |a b|); requests that arrive while others run are
admitted and complete."""
import threading

import numpy as np
import pytest

import oracle
from helpers import TOL64, random_csr
from trident_b200 import ops, workloads
from trident_b200.synth import HostCSR

pytestmark = pytest.mark.gpu


def _ref_ab(A, B):
    rp, cj, cx, ca = oracle.spgemm(A, B)
    return rp, cj, cx, ca


def _ref_rap(R, A, P):
    """R·(A·P) by the oracle, with the error scale of the chained product:
    sum_k |r_ik| * (sum |a p|)_kj."""
    rp1, cj1, cx1, ca1 = oracle.spgemm(A, P)
    rp, cj, cx, _ = oracle.spgemm(R, HostCSR(A.nrows, P.ncols, rp1, cj1, cx1))
    Rabs = HostCSR(R.nrows, R.ncols, R.rowptr, R.col, np.abs(R.val))
    _, _, scale, _ = oracle.spgemm(Rabs, HostCSR(A.nrows, P.ncols, rp1, cj1, ca1), with_abs=False)
    return rp, cj, cx, scale


def _same(H, ref):
    rp, cj, cx, scale = ref
    np.testing.assert_array_equal(H.rowptr.astype(np.int64), rp)
    np.testing.assert_array_equal(H.col, cj)
    assert np.all(np.abs(H.val - cx) <= TOL64 * np.maximum(np.abs(cx), scale))


def test_server_mix_matches_alone(ctx):
    ab = [(workloads.poisson_rows(r, l, s), workloads.poisson_rows(r, l, s + 1))
          for r, l, s in [(2000, 10.0, 1), (15000, 20.0, 3), (600, 30.0, 5), (40000, 8.0, 7)]]
    raps = [workloads.galerkin_operands(n=side, pts=7, agg=2) for side in (12, 20)]
    dab = [(A.to_device(), B.to_device()) for A, B in ab]
    drap = [(R.to_device(), A.to_device(), P.to_device()) for R, A, P in raps]
    ref_ab = [_ref_ab(A, B) for A, B in ab]
    ref_rap = [_ref_rap(R, A, P) for R, A, P in raps]
    for (A, B), ref in zip(dab, ref_ab):  # alone
        _same(ops.spgemm(ctx, A, B).to_host(), ref)
    for (R, A, P), ref in zip(drap, ref_rap):
        _same(ops.spgemm(ctx, R, ops.spgemm(ctx, A, P)).to_host(), ref)
    srv = ops.Server(ctx, mem_budget=8 << 30, lanes=2, max_batch=16)
    tickets = []
    lock = threading.Lock()

    def client(k):
        for rep in range(3):
            for i, (A, B) in enumerate(dab):
                t = srv.submit(A, B)
                with lock:
                    tickets.append(("ab", i, t))
            for i, (R, A, P) in enumerate(drap):
                t = srv.submit(A, P, R)
                with lock:
                    tickets.append(("rap", i, t))

    th = [threading.Thread(target=client, args=(k,)) for k in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    lat = []
    for kind, i, t in tickets:
        res, ms = srv.wait(t, timeout_ms=60000)
        lat.append(ms)
        _same(res.to_host(), ref_ab[i] if kind == "ab" else ref_rap[i])  # in the mix
        srv.release(t)
    st = srv.stats()
    assert st["completed"] == len(tickets) and st["reserved"] == 0 and st["status"] == 0
    assert st["batches"] < len(tickets)  # requests were batched together
    srv.close()


def test_server_rejects_oversized_request(ctx):
    # the bound of the first request alone exceeds the budget: it completes
    # with ENOMEM; the small one behind it still runs
    A = workloads.poisson_rows(5000, 20.0, 2)
    S = workloads.poisson_rows(50, 2.0, 3)
    dA, dS = A.to_device(), S.to_device()
    srv = ops.Server(ctx, mem_budget=1 << 20, lanes=1, max_batch=4)
    from trident_b200._lib import TSPG_ENOMEM, TspgError
    t_big, t_small = srv.submit(dA, dA), srv.submit(dS, dS)
    with pytest.raises(TspgError) as e:
        srv.wait(t_big, timeout_ms=60000)
    assert e.value.status == TSPG_ENOMEM
    srv.release(t_big)
    res, _ = srv.wait(t_small, timeout_ms=60000)
    _same(res.to_host(), _ref_ab(S, S))
    srv.release(t_small)
    st = srv.stats()
    assert st["completed"] == 1 and st["reserved"] == 0
    srv.close()


def test_server_refuses_bad_shapes(ctx):
    A = workloads.poisson_rows(300, 4.0, 4).to_device()
    B = random_csr(200, 300, density=0.02, seed=5).to_device()
    srv = ops.Server(ctx, mem_budget=1 << 30, lanes=1, max_batch=4)
    from trident_b200._lib import TSPG_EINVAL, TspgError
    with pytest.raises(TspgError) as e:
        srv.submit(A, B)  # 300 columns against 200 rows
    assert e.value.status == TSPG_EINVAL
    R = random_csr(10, 200, density=0.1, seed=6).to_device()
    with pytest.raises(TspgError) as e:
        srv.submit(A, A, R)  # R has 200 columns against A's 300 rows
    assert e.value.status == TSPG_EINVAL
    assert srv.stats()["queued"] == 0
    srv.close()


def test_server_admits_in_submission_order_under_a_tight_budget(ctx):
    # a budget that holds a few requests at a time, three lanes claiming
    # large batches, and a consumer that waits and releases in ticket order:
    # a later request admitted before an earlier one would hold the budget
    # the earlier one needs (the wait times out instead of hanging)
    ops_pairs = [(workloads.poisson_rows(6000, 12.0, s), workloads.poisson_rows(6000, 12.0, s + 1))
                 for s in (11, 13, 15, 17)]
    dev = [(A.to_device(), B.to_device()) for A, B in ops_pairs]
    mults, upper = ops.spgemm_count(ctx, *dev[0])
    one = upper * 12 + 6001 * 8
    srv = ops.Server(ctx, mem_budget=int(3.5 * one), lanes=3, max_batch=16)
    want = [_ref_ab(A, B) for A, B in ops_pairs]
    tickets = [(k % 4, srv.submit(*dev[k % 4])) for k in range(48)]
    for k, t in tickets:
        res, _ = srv.wait(t, timeout_ms=60000)
        _same(res.to_host(), want[k])
        srv.release(t)
    st = srv.stats()
    assert st["completed"] == 48 and st["reserved"] == 0 and st["status"] == 0
    srv.close()
