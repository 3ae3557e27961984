"""GPU: the continuous-batching server.  Each result must be the same alone
(a plain call) and in the mix (batched with other requests), within the FP64
tolerance; requests that arrive while others run are admitted and complete."""
import threading

import numpy as np
import pytest

from helpers import TOL64
from trident_b200 import ops, workloads

pytestmark = pytest.mark.gpu


def _same(P, Q):
    np.testing.assert_array_equal(P.rowptr.astype(np.int64), Q.rowptr.astype(np.int64))
    np.testing.assert_array_equal(P.col, Q.col)
    assert np.all(np.abs(P.val - Q.val) <= TOL64 * np.maximum(np.abs(P.val), 1.0) * 64)


def test_server_mix_matches_alone(ctx):
    ab = [(workloads.poisson_rows(r, l, s), workloads.poisson_rows(r, l, s + 1))
          for r, l, s in [(2000, 10.0, 1), (15000, 20.0, 3), (600, 30.0, 5), (40000, 8.0, 7)]]
    raps = [workloads.galerkin_operands(n=side, pts=7, agg=2) for side in (12, 20)]
    dab = [(A.to_device(), B.to_device()) for A, B in ab]
    drap = [(R.to_device(), A.to_device(), P.to_device()) for R, A, P in raps]
    alone_ab = [ops.spgemm(ctx, A, B).to_host() for A, B in dab]
    alone_rap = [ops.spgemm(ctx, R, ops.spgemm(ctx, A, P)).to_host() for R, A, P in drap]
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
        _same(res.to_host(), alone_ab[i] if kind == "ab" else alone_rap[i])
        srv.release(t)
    st = srv.stats()
    assert st["completed"] == len(tickets) and st["reserved"] == 0 and st["status"] == 0
    assert st["batches"] < len(tickets)  # requests were batched together
    srv.close()


def test_server_rejects_oversized_request(ctx):
    A = workloads.poisson_rows(5000, 20.0, 2).to_device()
    srv = ops.Server(ctx, mem_budget=1 << 20, lanes=1, max_batch=4)
    from trident_b200._lib import TSPG_ENOMEM, TspgError
    with pytest.raises(TspgError) as e:
        srv.submit(A, A)
    assert e.value.status == TSPG_ENOMEM
    srv.close()
