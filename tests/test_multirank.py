"""CPU: the N > 1 path with gloo ranks on 127.0.0.1.

The benchmark splits one product C = A·A over N GPUs by row panels: rank 0
holds A and broadcasts it, the rows are cut into panels of equal products,
every rank multiplies its panel, and the panels of C concatenate to the whole
product with no reduction.  Here two gloo ranks run that host logic
(trident_b200.panels) with the oracle standing in for each rank's GPU, and the
assembled result must equal the single-process product; the job's step time
is the slowest rank's."""
import os
import socket
import sys
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    import oracle
    from trident_b200 import panels, workloads
    from trident_b200.synth import HostCSR
    # rank 0 holds A; everyone receives it (B = A replicated)
    if rank == 0:
        H = workloads.rmat(scale=9, edge_factor=16, seed=3)
        src = (torch.from_numpy(H.rowptr.astype(np.int32)), torch.from_numpy(H.col), torch.from_numpy(H.val))
        shape = (H.nrows, H.ncols)
    else:
        src, shape = (None, None, None), None
    m, n, rp, col, val = panels.broadcast_csr(*src, 0, "cpu", torch.int32, torch.float64, shape=shape)
    A = HostCSR(m, n, rp.numpy().astype(np.int64), col.numpy(), val.numpy())
    rowf = oracle.row_mults(A, A)  # stand-in for tspg_spgemm_row_products
    cuts = panels.panel_cuts(rowf, world)
    r0, r1 = panels.panel_rows(cuts, rank)
    prp, pcj, pcx, _ = oracle.spgemm(A, A, r0, r1, with_abs=False)
    gathered = [None] * world
    dist.all_gather_object(gathered, (rank, prp, pcj, pcx, int(rowf[r0:r1].sum())))
    ms = bench.max_over_ranks(100.0 + 50.0 * rank, world, device="cpu")
    dist.barrier()
    q.put((rank, ms, cuts.tolist(), gathered if rank == 0 else None, A if rank == 0 else None))
    dist.destroy_process_group()


def test_two_gloo_ranks_row_panels_assemble_the_product():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=180) for _ in procs), key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # the job's step time is the slowest rank's
    assert [o[1] for o in out] == [150.0, 150.0]
    # both ranks cut the same panels: contiguous, covering every row once
    cuts = out[0][2]
    assert cuts == out[1][2] and cuts[0] == 0 and cuts[-1] == out[0][4].nrows
    assert all(a <= b for a, b in zip(cuts, cuts[1:]))
    sys.path.insert(0, ROOT)
    import oracle
    from trident_b200 import panels
    A = out[0][4]
    parts = sorted(out[0][3], key=lambda g: g[0])
    rp, cj, cx = panels.assemble([(g[1], g[2], g[3]) for g in parts], A.ncols)
    wrp, wcj, wcx, _ = oracle.spgemm(A, A, with_abs=False)
    np.testing.assert_array_equal(rp, wrp)
    np.testing.assert_array_equal(cj, wcj)
    np.testing.assert_array_equal(cx, wcx)
    # equal work: no panel holds more than half the products plus one row
    rowf = oracle.row_mults(A, A)
    assert max(g[4] for g in parts) <= rowf.sum() / 2 + rowf.max()


def test_panel_cuts_edges():
    sys.path.insert(0, ROOT)
    from trident_b200.panels import panel_cuts
    np.testing.assert_array_equal(panel_cuts(np.zeros(5, np.int64), 3), [0, 0, 0, 5])
    np.testing.assert_array_equal(panel_cuts(np.array([100, 1, 1, 1]), 2), [0, 1, 4])
    np.testing.assert_array_equal(panel_cuts(np.array([1, 1]), 4), [0, 1, 1, 2, 2])
    np.testing.assert_array_equal(panel_cuts(np.ones(8, np.int64), 4), [0, 2, 4, 6, 8])
    assert panel_cuts(np.zeros(0, np.int64), 2).tolist() == [0, 0, 0]
    with pytest.raises(ValueError):
        panel_cuts(np.ones(3, np.int64), 0)


def test_single_rank_is_unchanged():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, 1) == 12.5
