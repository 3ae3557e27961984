"""Benchmark of the on-node SpGEMM path (one JSON line on rank 0).

Default workload: plain C = A·A on an R-MAT graph, scale 20 (1,048,576 rows),
edge factor 16, (a, b, c, d) = (.57, .19, .19, .05), duplicates merged,
self-loops kept, FP64 values uniform in [-1, 1], int32 CSR in, int64 row
offsets out (nnz(C) > 2^31).  One step = one full two-phase SpGEMM through
the C ABI (flop count, symbolic, scan, numeric) into preallocated C.

  value   GFLOP/s = 2 * mults / device time per step, inputs resident in HBM
  e2e     the same metric with host buffers: pinned host A -> device, the
          SpGEMM, and C back to pinned host memory inside the timed region
  roofline  the dominant persistent kernel (symbolic or numeric phase) timed
          with CUDA events the library records on the call's stream; its
          algorithmic bytes are bytes(A) + bytes(B) + bytes(C) with
          bytes(X) = (rows+1)*s + 12*nnz(X)
  cpu_baseline  the CPU restatement (oracle) on a strided row sample, all host
          threads

Multi-GPU: the rows of A are cut into N panels of equal products; rank 0
generates A and broadcasts it over NCCL (B = A is replicated), every rank
multiplies its panel, no reduction ("rowpanels<N>", strong scaling: the
product is fixed); value = the product's flops / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 2**20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="rmat",
                   choices=["rmat", "uniform", "batched", "rap", "served", "summa", "coo"])
    p.add_argument("--rate", type=float, default=2000.0)
    # one lane: the lanes' persistent kernels take the whole GPU in turn, so
    # more lanes only split the queue into smaller batches (served, 2000 req/s
    # offered: 515 req/s with 1 lane, 462 with 2 or 3; at 80 % of the loop's
    # rate p50 48 ms with 1 lane, 0.6 s with 2, 2.1 s with 3, one run each)
    p.add_argument("--lanes", type=int, default=1, help="server worker lanes (served)")
    p.add_argument("--max-batch", type=int, default=128, help="requests per server batch (served)")
    p.add_argument("--duration", type=float, default=5.0)
    p.add_argument("--products", type=int, default=512)
    p.add_argument("--scale", type=int, default=20)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--dense-win", type=int, default=None,
                   help="override the tuning's dense_win_log2 (0 = whole-row rank form for every DENSE row)")
    p.add_argument("--dense-fill", type=int, default=None,
                   help="override the tuning's dense_win_fill_log2 (window form when nnz(row) >= ncols / 2^fill)")
    p.add_argument("--dense-cluster", type=int, default=None,
                   help="override the tuning's dense_win_cluster (CTAs per cluster for the window form; 0 = one CTA)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    return p.parse_args()


def csr_bytes(rows, nnz, s):
    return (rows + 1) * s + 12 * nnz


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                smax = float(f[2].split()[0])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        busy = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- workload
def make_workload(args):
    """The operand and the workload description shared by both arms' `config`."""
    from trident_b200 import workloads
    if args.workload == "rmat":
        A = workloads.rmat(scale=args.scale, edge_factor=args.edge_factor, seed=args.seed)
        cfg = {"workload": f"rmat{args.scale}_AxA", "rows": A.nrows, "nnz_A": A.nnz,
               "edge_factor": args.edge_factor, "abcd": [0.57, 0.19, 0.19, 0.05], "seed": args.seed}
    else:
        A = workloads.uniform_rows(1024, 16, True, seed=args.seed)
        cfg = {"workload": "uniform1024_AxA", "rows": A.nrows, "nnz_A": A.nnz, "seed": args.seed}
    a_bytes = csr_bytes(A.nrows, A.nnz, 4)
    cfg["l2"] = ("inputs and outputs larger than L2 (A %.0f MB; C holds at least nnz(A) entries)" % (a_bytes / 1e6)
                 if a_bytes > L2_BYTES else "A fits L2 (launch-bound case)")
    return A, cfg


def sample_rows(A, mults_total, target=6e9):
    """The CPU sample of a workload: rows i = 1 mod s of A (all rows when
    s = 1), s the smallest power of two that keeps the sample at or below
    `target` multiply-adds (about 10 s of the oracle on 16 host cores).  The
    timed CPU baseline, the reference arm and the parity check all use it."""
    import numpy as np
    s = 1
    while mults_total / s > target:
        s *= 2
    return s, np.arange(1 if s > 1 else 0, A.nrows, s, dtype=np.int64)


def cpu_baseline(A, rows, stride, rm):
    """Oracle (CPU restatement, all host threads) on the sample rows of A·A."""
    import oracle
    S = A.rows(rows)
    mu = int(rm[rows].sum())
    t0 = time.perf_counter()
    oracle.spgemm(S, A, with_abs=False)
    dt = time.perf_counter() - t0
    return {"value": round(2 * mu / dt / 1e9, 4), "unit": "GFLOP/s", "cores": oracle.num_threads(),
            "kind": "port", "ms": round(dt * 1e3, 1),
            "sample": f"rows i = 1 mod {stride} of A times A ({S.nrows} rows, {mu} mults)"
            if stride > 1 else f"all rows of A times A ({S.nrows} rows, {mu} mults)"}


def gather_rows(Crp, Ccol, Cval, rows):
    """Rows `rows` (numpy int64, ascending) of a device CSR, copied to the host:
    (row lengths, columns, values)."""
    import numpy as np
    import torch
    rr = torch.from_numpy(rows).to(Crp.device)
    starts = Crp[rr].to(torch.int64)
    lens = Crp[rr + 1].to(torch.int64) - starts
    tot = int(lens.sum().item())
    if tot == 0:
        return lens.cpu().numpy(), np.zeros(0, np.int32), np.zeros(0, np.float64)
    excl = torch.cumsum(lens, 0) - lens
    idx = torch.repeat_interleave(starts - excl, lens) + torch.arange(tot, device=Crp.device)
    cols, vals = Ccol[idx].cpu().numpy(), Cval[idx].cpu().numpy()
    del idx
    return lens.cpu().numpy(), cols, vals


def parity_rows(A, B, rows, Crp, Ccol, Cval, chunk=150_000_000):
    """Rows `rows` of the GPU's C = A·B against the oracle: row lengths and
    sorted columns bit-exact, values within 1e-12 * max(|y|, sum |a_ik b_kj|).
    Chunked by output entries so host and device memory stay bounded."""
    import numpy as np
    import oracle
    import torch
    TOL = 1e-12
    rr = torch.from_numpy(rows).to(Crp.device)
    lens_all = (Crp[rr + 1].to(torch.int64) - Crp[rr].to(torch.int64)).cpu().numpy()
    cum = np.cumsum(lens_all)
    cuts = [0]
    while cuts[-1] < rows.size:
        base = cum[cuts[-1] - 1] if cuts[-1] else 0
        nxt = int(np.searchsorted(cum, base + chunk, side="right"))
        cuts.append(min(rows.size, max(nxt, cuts[-1] + 1)))
    ok, worst, nnz = True, 0.0, 0
    for c0, c1 in zip(cuts[:-1], cuts[1:]):
        sub = rows[c0:c1]
        lens, cols, vals = gather_rows(Crp, Ccol, Cval, sub)
        rp, cj, cx, ca = oracle.spgemm(A.rows(sub), B, with_abs=True)
        if not (np.array_equal(lens, np.diff(rp)) and np.array_equal(cols, cj)):
            ok = False
            break
        if cx.size:
            rel = np.abs(vals - cx) / np.maximum(np.maximum(np.abs(cx), ca), 1e-300)
            worst = max(worst, float(rel.max()))
        nnz += int(cx.size)
    rowptr_ok = bool(int(Crp[0].item()) == 0 and bool((Crp[1:] >= Crp[:-1]).all().item()))
    return {"rows_checked": int(rows.size), "entries_checked": nnz, "structure_equal": bool(ok),
            "rowptr_monotone": rowptr_ok, "max_rel_err": worst, "tolerance": TOL,
            "values_within_tolerance": bool(ok and worst <= TOL),
            "rule": "row lengths and columns bit-exact; |x - y| <= 1e-12 * max(|y|, sum |a_ik b_kj|)"}


# ---------------------------------------------------------------- our arm
def max_over_ranks(ms: float, world: int, device: str = "cuda") -> float:
    """The job's step time: the slowest rank's (every rank calls this, in the
    same order, after its own timed region)."""
    if world <= 1:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, rank, world):
    """One product C = A·A.  At N GPUs the rows of A are cut into N panels of
    equal products (row-panel split: A is generated on rank 0 and broadcast
    over NCCL, every rank multiplies its panel by the whole of A, no
    reduction); at N = 1 the panel is all of A."""
    import ctypes as C

    import numpy as np
    import torch

    from trident_b200 import ops, panels
    from trident_b200._lib import TSPG_F_B_SORTED, TspgCsrOut, check, lib
    from trident_b200.csr import DeviceCSR

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    ctx = ops.Context(dev)
    cfg_tuning = apply_tuning(ctx, "rmat") if args.workload == "rmat" else None
    if args.dense_win is not None:
        ctx.set_tuning({"dense_win_log2": args.dense_win})
    if args.dense_fill is not None:
        ctx.set_tuning({"dense_win_fill_log2": args.dense_fill})
    if args.dense_cluster is not None:
        ctx.set_tuning({"dense_win_cluster": args.dense_cluster})
    cur = ctx.get_tuning()
    cfg_tuning = dict(cfg_tuning or {}, dense_win_log2=cur["dense_win_log2"],
                      dense_win_fill_log2=cur["dense_win_fill_log2"],
                      dense_win_cluster=cur["dense_win_cluster"])
    A = cfg = None
    if rank == 0:
        A, cfg = make_workload(args)
    if world > 1:
        # B (= A) replicated: one broadcast from rank 0 over NCCL
        if rank == 0:
            dA0 = A.to_device(rowptr_bits=32)
            src = (dA0.rowptr, dA0.col, dA0.val)
        else:
            src = (None, None, None)
        m, n, rp_t, col_t, val_t = panels.broadcast_csr(*src, 0, "cuda", torch.int32, torch.float64,
                                                        shape=(A.nrows, A.ncols) if rank == 0 else None)
        dA = DeviceCSR(m, n, rp_t, col_t, val_t)
        if rank != 0:
            from trident_b200.synth import HostCSR
            A = HostCSR(m, n, rp_t.cpu().numpy().astype(np.int64), col_t.cpu().numpy(), val_t.cpu().numpy())
    else:
        dA = A.to_device(rowptr_bits=32)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    # the row panel of this rank, cut by products
    rowf = panels.row_products(ctx, dA, dA).cpu().numpy()
    mults_total = int(rowf.sum())
    cuts = panels.panel_cuts(rowf, world)
    r0, r1 = panels.panel_rows(cuts, rank)
    a_rp = A.rowptr
    dP = DeviceCSR(r1 - r0, A.ncols, dA.rowptr[r0:r1 + 1], dA.col, dA.val, nnz=int(a_rp[r1] - a_rp[r0]))
    pa, b = dP.abi(), dA.abi()
    mults, upper = ops.spgemm_count(ctx, dP, dA)
    assert mults == int(rowf[r0:r1].sum())
    plan = ops.Plan(ctx, dP, dA)
    nnz_c = plan.c_nnz
    plan.close()
    pm = r1 - r0
    rp_bits = 64 if nnz_c > 2**31 - 1 else 32
    Crp = torch.empty(pm + 1, dtype=torch.int64 if rp_bits == 64 else torch.int32, device="cuda")
    Ccol = torch.empty(max(nnz_c, 1), dtype=torch.int32, device="cuda")
    Cval = torch.empty(max(nnz_c, 1), dtype=torch.float64, device="cuda")

    def out():
        o = TspgCsrOut()
        o.nrows, o.ncols = pm, A.ncols
        o.rowptr, o.rowptr_bits, o.val_bits = Crp.data_ptr(), rp_bits, 64
        o.col, o.val, o.capacity = Ccol.data_ptr(), Cval.data_ptr(), nnz_c
        return o

    def step():
        o = out()
        check(lib.tspg_spgemm(ctx.h, sp, C.byref(pa), C.byref(b), C.byref(o), TSPG_F_B_SORTED), "tspg_spgemm")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    check(lib.tspg_ctx_phase_timing(ctx.h, 1), "phase timing")
    launches0 = C.c_int64()
    lib.tspg_ctx_stats(ctx.h, C.byref(launches0))
    sym_ms, num_ms = [], []
    clocks = ClockSampler(dev)
    clocks.start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fs, fn = C.c_float(), C.c_float()
    for _ in range(args.steps):
        step()
        lib.tspg_ctx_phase_ms(ctx.h, C.byref(fs), C.byref(fn))
        sym_ms.append(fs.value)
        num_ms.append(fn.value)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    check(lib.tspg_ctx_phase_timing(ctx.h, 0), "phase timing")
    launches1 = C.c_int64()
    lib.tspg_ctx_stats(ctx.h, C.byref(launches1))
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    value = 2.0 * mults_total / (ms * 1e-3) / 1e9

    # roofline of the dominant persistent phase of this rank's panel
    bytes_a = csr_bytes(A.nrows, A.nnz, 4)
    bytes_p = csr_bytes(pm, int(a_rp[r1] - a_rp[r0]), 4)
    bytes_c = csr_bytes(pm, nnz_c, rp_bits // 8)
    algo = bytes_p + bytes_a + bytes_c
    sym, num = statistics.mean(sym_ms), statistics.mean(num_ms)
    dom_ms, dom_name = ((num, "numeric phase (k_dense_rank + k_phase + k_groups)") if num >= sym
                        else (sym, "symbolic phase (k_phase + k_groups)"))
    try:
        peak, peak_src = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    achieved = algo / (dom_ms * 1e-3) / 1e9
    gather = algo + 8 * int(a_rp[r1] - a_rp[r0]) + 12 * mults
    traffic = traffic_src = None
    if world == 1 and rank == 0:
        try:
            prof = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
            ent = prof.get(cfg["workload"], {}).get(dom_name)
            if ent:
                traffic, traffic_src = int(ent["dram_bytes_per_launch"]), ent.get("source")
        except Exception:
            pass

    # e2e through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, A, ctx, mults_total, nnz_c, rp_bits, world, (Crp, Ccol, Cval), (r0, r1))

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        import oracle
        rm = oracle.row_mults(A, A)
        stride, rows = sample_rows(A, mults)
        cpu = cpu_baseline(A, rows, stride, rm)
        # the same rows of the GPU's C (the last timed call's output) against the oracle
        parity = parity_rows(A, A, rows, Crp, Ccol, Cval)
        parity["sample"] = cpu["sample"]

    line = None
    if rank == 0:
        line = {
            "metric": "A·A SpGEMM GFLOP/s (2 x multiply-adds), FP64",
            "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded R-MAT, values U[-1,1])",
            "config": dict(cfg, mults=mults_total),
            "parallelism": f"rowpanels{world}" if world > 1 else "single",
            "panels": {"cuts": [int(x) for x in cuts], "rank0_mults": mults} if world > 1 else None,
            "output": {"nnz_C": nnz_c, "c_rowptr_bits": rp_bits, "C_MB": round(bytes_c / 1e6)},
            "tuning": cfg_tuning,
            "phase_ms": {"symbolic": round(sym, 3), "numeric": round(num, 3)},
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1), "peak": peak,
                         "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "traffic_source": traffic_src, "algorithmic_bytes": algo,
                         "step_frac": round(algo / (ms * 1e-3) / 1e9 / peak, 4),
                         # Gustavson gather model: + B row offsets per A entry + B row contents per product
                         "gather_model_bytes": gather,
                         "gather_frac": round(gather / (dom_ms * 1e-3) / 1e9 / peak, 4)},
            "gpu_launches": int(launches1.value - launches0.value),
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "parity": parity,
        }
    ctx.close()
    return line


def run_e2e(args, A, ctx, mults_total, nnz_c, rp_bits, world, cbufs, panel):
    """Host A (pinned) -> device, this rank's panel of A·A through the ABI,
    the panel of C -> pinned host."""
    import ctypes as C

    import numpy as np
    import torch

    from trident_b200._lib import TSPG_F_B_SORTED, TspgCsr, TspgCsrOut, check, lib

    r0, r1 = panel
    pm = r1 - r0
    hrp = torch.from_numpy(A.rowptr.astype(np.int32)).pin_memory()
    hcol = torch.from_numpy(A.col).pin_memory()
    hval = torch.from_numpy(A.val).pin_memory()
    drp, dcol, dval = torch.empty_like(hrp, device="cuda"), torch.empty_like(hcol, device="cuda"), \
        torch.empty_like(hval, device="cuda")
    # C lands in pinned host memory; when that does not fit, it is streamed
    # through a pinned staging ring (every byte still crosses to the host)
    c_bytes = nnz_c * 12 + (pm + 1) * (rp_bits // 8)
    try:
        avail = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_AVPHYS_PAGES")
    except Exception:
        avail = 0
    full = c_bytes * world < 0.5 * avail
    rdt = torch.int64 if rp_bits == 64 else torch.int32
    Crp, Ccol, Cval = cbufs
    if full:
        hC = (torch.empty(Crp.numel(), dtype=rdt, pin_memory=True),
              torch.empty(Ccol.numel(), dtype=torch.int32, pin_memory=True),
              torch.empty(Cval.numel(), dtype=torch.float64, pin_memory=True))
    else:
        ring = 1 << 30
        hC = torch.empty(ring, dtype=torch.uint8, pin_memory=True)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    pnnz = int(A.rowptr[r1] - A.rowptr[r0])

    def d2h_ring(t):
        flat = t.view(torch.uint8)
        for o in range(0, flat.numel(), hC.numel()):
            n = min(hC.numel(), flat.numel() - o)
            hC[:n].copy_(flat[o:o + n], non_blocking=True)

    def step():
        drp.copy_(hrp, non_blocking=True)
        dcol.copy_(hcol, non_blocking=True)
        dval.copy_(hval, non_blocking=True)
        b = TspgCsr(A.nrows, A.ncols, A.nnz, drp.data_ptr(), 32, 64, dcol.data_ptr(), dval.data_ptr())
        a = TspgCsr(pm, A.ncols, pnnz, drp.data_ptr() + 4 * r0, 32, 64, dcol.data_ptr(), dval.data_ptr())
        o = TspgCsrOut()
        o.nrows, o.ncols = pm, A.ncols
        o.rowptr, o.rowptr_bits, o.val_bits = Crp.data_ptr(), rp_bits, 64
        o.col, o.val, o.capacity = Ccol.data_ptr(), Cval.data_ptr(), nnz_c
        check(lib.tspg_spgemm(ctx.h, sp, C.byref(a), C.byref(b), C.byref(o), TSPG_F_B_SORTED), "tspg_spgemm")
        if full:
            hC[0].copy_(Crp, non_blocking=True)
            hC[1].copy_(Ccol[:nnz_c], non_blocking=True)
            hC[2].copy_(Cval[:nnz_c], non_blocking=True)
        else:
            d2h_ring(Crp)
            d2h_ring(Ccol[:nnz_c])
            d2h_ring(Cval[:nnz_c])

    steps = max(1, min(args.steps, 3))
    step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / steps, world)
    h2d = (hrp.numel() * 4 + hcol.numel() * 4 + hval.numel() * 8)
    d2h = c_bytes
    if world > 1:
        t = torch.tensor([c_bytes], dtype=torch.int64, device="cuda")
        torch.distributed.all_reduce(t)
        d2h = int(t.item())
    return {"value": round(2.0 * mults_total / (ms * 1e-3) / 1e9, 3), "unit": "GFLOP/s",
            "ms_per_step": round(ms, 3), "h2d_bytes_per_step": int(h2d * world), "d2h_bytes_per_step": int(d2h),
            "per": "whole job: every rank copies all of A (its panel and the replicated B) and its panel of C"
            if world > 1 else "A to the device, C to the host",
            "c_to_host": "pinned result arrays" if full else "pinned 1 GiB staging ring (host RAM < 2x C)",
            "steps": steps}


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's CPU path for the same product: the oracle restatement
    of KokkosKernels SpGEMM semantics (KokkosKernels itself is not vendored
    and cannot be built here), all host threads.  Every step multiplies the
    same row sample as the GPU arm's cpu_baseline leg (rows i = 1 mod s of
    A·A); the operand comes from the host-only generator library, so this arm
    maps no device code."""
    import oracle
    A, cfg = make_workload(args)
    rm = oracle.row_mults(A, A)
    mults = int(rm.sum())
    stride, rows = sample_rows(A, mults)
    times = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(A, rows, stride, rm)
        if i >= args.warmup:
            times.append(r["ms"])
    ms = statistics.mean(times)
    mu = int(rm[rows].sum())
    v = 2 * mu / (ms * 1e-3) / 1e9
    return {"impl": "reference", "metric": "A·A SpGEMM GFLOP/s (2 x multiply-adds), FP64", "value": round(v, 4),
            "unit": "GFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded R-MAT, values U[-1,1])", "config": dict(cfg, mults=mults),
            "cpu_baseline": {"value": round(v, 4), "unit": "GFLOP/s", "cores": r["cores"], "kind": "port",
                             "sample": r["sample"]},
            "e2e": {"value": round(v, 4), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------------- batched
def run_batched(args):
    """512 independent products C_i = A_i B_i (rows log-uniform in [1k, 200k],
    Poisson row lengths with mean U[8, 32]): one batched run (two persistent
    launches in two CUDA graphs) against a loop of plain tspg_spgemm calls."""
    import ctypes as C

    import numpy as np
    import torch

    from trident_b200 import ops, workloads
    from trident_b200._lib import TSPG_F_B_SORTED, TspgCsrOut, check, lib
    torch.cuda.set_device(0)
    specs = workloads.batched_specs(args.products, seed=args.seed)
    ctx = ops.Context(0)
    tuning = apply_tuning(ctx, "batched")
    dev, mults = [], 0
    for spec in specs:
        A, B = workloads.batched_product(spec)
        dA, dB = A.to_device(), B.to_device()
        dev.append((dA, dB))
    bt = ops.Batch(ctx)
    for dA, dB in dev:
        bt.add(dA, dB)
    stream = torch.cuda.current_stream()
    total_nnz = bt.run(TSPG_F_B_SORTED)
    for dA, dB in dev:
        mults += ops.spgemm_count(ctx, dA, dB)[0]
    for _ in range(args.warmup):
        bt.run(TSPG_F_B_SORTED)
    torch.cuda.synchronize()
    l0 = C.c_int64()
    lib.tspg_ctx_stats(ctx.h, C.byref(l0))
    clocks = ClockSampler(0)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        bt.run(TSPG_F_B_SORTED)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    l1 = C.c_int64()
    lib.tspg_ctx_stats(ctx.h, C.byref(l1))
    ms = e0.elapsed_time(e1) / args.steps
    # parity: a seeded subset of the products (results of the last timed run)
    # against the oracle, and the oracle's time on them as the CPU baseline
    import oracle
    pick = sorted(int(i) for i in np.random.default_rng(args.seed).choice(len(dev), size=min(8, len(dev)),
                                                                             replace=False))
    checks, cpu_s, cpu_mults = [], 0.0, 0
    for i in pick:
        Ai, Bi = workloads.batched_product(specs[i])
        Ri = bt.result(i)
        checks.append(parity_rows(Ai, Bi, np.arange(Ai.nrows, dtype=np.int64), Ri.rowptr, Ri.col, Ri.val))
        t0 = time.perf_counter()
        oracle.spgemm(Ai, Bi, with_abs=False)
        cpu_s += time.perf_counter() - t0
        cpu_mults += int(oracle.row_mults(Ai, Bi).sum())
    parity = {"products_checked": pick, "entries_checked": sum(c["entries_checked"] for c in checks),
              "structure_equal": all(c["structure_equal"] for c in checks),
              "max_rel_err": max(c["max_rel_err"] for c in checks), "tolerance": 1e-12,
              "values_within_tolerance": all(c["values_within_tolerance"] for c in checks)}
    mean_mults = mults / len(dev)
    cpu = {"value": round(cpu_mults / cpu_s / mean_mults, 2), "unit": "products/s", "cores": oracle.num_threads(),
           "kind": "port", "sample": f"products {pick} ({cpu_mults} mults, {cpu_s:.2f} s), scaled to the mean "
                                     f"product of the batch ({mean_mults:.0f} mults)"}
    # the same products as a loop of plain calls (output buffer reused)
    maxnnz = max(int(bt.result(i).nnz) for i in range(len(dev)))
    maxrows = max(dA.nrows for dA, _ in dev)
    Crp = torch.empty(maxrows + 1, dtype=torch.int64, device="cuda")
    Ccol = torch.empty(max(maxnnz, 1), dtype=torch.int32, device="cuda")
    Cval = torch.empty(max(maxnnz, 1), dtype=torch.float64, device="cuda")

    def loop():
        for dA, dB in dev:
            a, b = dA.abi(), dB.abi()
            o = TspgCsrOut()
            o.nrows, o.ncols = dA.nrows, dB.ncols
            o.rowptr, o.rowptr_bits, o.val_bits = Crp.data_ptr(), 64, 64
            o.col, o.val, o.capacity = Ccol.data_ptr(), Cval.data_ptr(), maxnnz
            check(lib.tspg_spgemm(ctx.h, stream.cuda_stream, C.byref(a), C.byref(b), C.byref(o),
                                  TSPG_F_B_SORTED), "tspg_spgemm")
    loop()
    torch.cuda.synchronize()
    e0.record(stream)
    loop()
    e1.record(stream)
    torch.cuda.synchronize()
    loop_ms = e0.elapsed_time(e1)
    n = len(dev)
    line = {
        "metric": "batched products/s (512 independent FP64 A_i B_i, all in one launch of each persistent kernel per phase)",
        "value": round(n / (ms * 1e-3), 1), "unit": "products/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Poisson-row matrices, values U[-1,1])",
        "config": {"tuning": tuning, "workload": f"batched{n}", "products": n, "rows_total": int(sum(d[0].nrows for d in dev)),
                   "nnz_A_total": int(sum(d[0].nnz for d in dev)), "mults": int(mults),
                   "nnz_C_total": int(total_nnz), "rows": "log-uniform [1e3, 2e5]", "lambda": "U[8, 32]"},
        "gflops": round(2.0 * mults / (ms * 1e-3) / 1e9, 3),
        "loop_of_plain_calls": {"ms": round(loop_ms, 3), "products_per_s": round(n / (loop_ms * 1e-3), 1)},
        "speedup_vs_loop": round(loop_ms / ms, 3),
        "gpu_launches": int(l1.value - l0.value),
        "clocks": clk,
        "cpu_baseline": cpu,
        "parity": parity,
    }
    bt.close()
    ctx.close()
    return line


def run_rap(args):
    """AMG Galerkin product on the 27-point Laplacian of an n^3 grid (n = 128 by
    default, --scale sets n): AP = A·P, then RAP = R·(AP), R = P^T built by an
    untimed host transpose.  One step = both products.  Parity: the whole AP
    and RAP against the oracle; CPU baseline: the oracle on both products."""
    import ctypes as C

    import numpy as np
    import torch

    import oracle
    from trident_b200 import ops, workloads
    from trident_b200._lib import TSPG_F_B_SORTED, TspgCsrOut, check, lib
    n = args.scale if args.scale != 20 else 128
    torch.cuda.set_device(0)
    R, A, P = workloads.galerkin_operands(n=n, pts=27, agg=3)
    ctx = ops.Context(0)
    tuning = apply_tuning(ctx, "rap")
    dR, dA, dP = R.to_device(), A.to_device(), P.to_device()
    m1 = ops.spgemm_count(ctx, dA, dP)[0]
    AP = ops.spgemm(ctx, dA, dP, rowptr_bits=32)
    m2 = ops.spgemm_count(ctx, dR, AP)[0]
    RAP = ops.spgemm(ctx, dR, AP, rowptr_bits=32)
    stream = torch.cuda.current_stream()

    def call(X, Y, Cout):
        x, y = X.abi(), Y.abi()
        o = TspgCsrOut()
        o.nrows, o.ncols = X.nrows, Y.ncols
        o.rowptr, o.rowptr_bits, o.val_bits = Cout.rowptr.data_ptr(), 32, 64
        o.col, o.val, o.capacity = Cout.col.data_ptr(), Cout.val.data_ptr(), Cout.nnz
        check(lib.tspg_spgemm(ctx.h, stream.cuda_stream, C.byref(x), C.byref(y), C.byref(o), TSPG_F_B_SORTED),
              "tspg_spgemm")

    for _ in range(max(args.warmup, 3)):
        call(dA, dP, AP)
        call(dR, AP, RAP)
    torch.cuda.synchronize()
    check(lib.tspg_ctx_phase_timing(ctx.h, 1), "phase timing")
    l0 = C.c_int64()
    lib.tspg_ctx_stats(ctx.h, C.byref(l0))
    clocks = ClockSampler(0)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_ap = 0.0
    fs, fn = C.c_float(), C.c_float()
    num = {"AP": [], "RAP": []}
    sym = {"AP": [], "RAP": []}
    # one R·A·P takes ~10 ms: enough steps for a timed region of about a second,
    # so the clock sampler (200 ms period) sees it
    steps = max(args.steps, 100)
    e0.record(stream)
    for _ in range(steps):
        ea.record(stream)
        call(dA, dP, AP)
        eb.record(stream)
        lib.tspg_ctx_phase_ms(ctx.h, C.byref(fs), C.byref(fn))
        num["AP"].append(fn.value)
        sym["AP"].append(fs.value)
        call(dR, AP, RAP)
        lib.tspg_ctx_phase_ms(ctx.h, C.byref(fs), C.byref(fn))
        num["RAP"].append(fn.value)
        sym["RAP"].append(fs.value)
        t_ap += ea.elapsed_time(eb)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    check(lib.tspg_ctx_phase_timing(ctx.h, 0), "phase timing")
    l1 = C.c_int64()
    lib.tspg_ctx_stats(ctx.h, C.byref(l1))
    ms = e0.elapsed_time(e1) / steps
    ap_ms = t_ap / steps
    peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    bap = csr_bytes(A.nrows, A.nnz, 4) + csr_bytes(P.nrows, P.nnz, 4) + csr_bytes(AP.nrows, AP.nnz, 4)
    brap = csr_bytes(R.nrows, R.nnz, 4) + csr_bytes(AP.nrows, AP.nnz, 4) + csr_bytes(RAP.nrows, RAP.nnz, 4)
    ap_num = statistics.mean(num["AP"])
    rap_num = statistics.mean(num["RAP"])
    ap_sym = statistics.mean(sym["AP"])
    rap_sym = statistics.mean(sym["RAP"])
    # the A·P rows are one-pass rows (multiplied whole in the first launch), so
    # the roofline takes both launches of the call
    ap_phases = ap_sym + ap_num
    ap_traffic = (None, None)
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        ent = prof.get(f"rap27pt_{n}^3", {}).get(
            "A·P, both launches (k_groups + k_onepass, then the copy of the one-pass rows)")
        if ent:
            ap_traffic = (int(ent["dram_bytes_per_launch"]), ent.get("source"))
    except Exception:
        pass
    # CPU baseline: the oracle on both products, repeated for at least ~5 s
    from trident_b200.synth import HostCSR
    reps, t0 = 0, time.perf_counter()
    while True:
        orp, oj, ox, _ = oracle.spgemm(A, P, with_abs=False)
        Ho = HostCSR(A.nrows, P.ncols, orp, oj, ox)
        oracle.spgemm(R, Ho, with_abs=False)
        reps += 1
        if time.perf_counter() - t0 >= 5.0:
            break
    cpu_s = (time.perf_counter() - t0) / reps
    # parity: the whole AP and RAP of the last timed step against the oracle
    # (RAP = R times the oracle's own AP)
    parity = {name: parity_rows(X, Y, np.arange(X.nrows, dtype=np.int64), G.rowptr, G.col, G.val)
              for name, X, Y, G in (("AP", A, P, AP), ("RAP", R, Ho, RAP))}
    line = {
        "metric": "Galerkin R·A·P GFLOP/s (2 x multiply-adds), FP64", "value": round(2.0 * (m1 + m2) / (ms * 1e-3) / 1e9, 3),
        "unit": "GFLOP/s", "n_gpus": 1, "steps": steps, "warmup": max(args.warmup, 3), "ms_per_step": round(ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (27-point Laplacian, SA prolongator)",
        "config": {"workload": f"rap27pt_{n}^3", "nnz_A": A.nnz, "nnz_P": P.nnz, "nnz_AP": AP.nnz,
                   "nnz_RAP": RAP.nnz, "mults_AP": int(m1), "mults_RAP": int(m2),
                   "l2": "A (%.0f MB) larger than L2; P, AP, RAP re-read from L2/HBM" % (csr_bytes(A.nrows, A.nnz, 4) / 1e6)},
        "tuning": tuning,
        "AP": {"ms": round(ap_ms, 3), "symbolic_ms": round(ap_sym, 3), "numeric_ms": round(ap_num, 3),
               "hbm_frac": round(bap / (ap_ms * 1e-3) / 1e9 / peak, 4)},
        "RAP": {"ms": round(ms - ap_ms, 3), "symbolic_ms": round(rap_sym, 3), "numeric_ms": round(rap_num, 3),
                "hbm_frac": round(brap / ((ms - ap_ms) * 1e-3) / 1e9 / peak, 4)},
        "roofline": {"bound": "hbm",
                     "kernel": "A·P, both launches (k_groups + k_onepass, then the copy of the one-pass rows)",
                     "achieved": round(bap / (ap_phases * 1e-3) / 1e9, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(bap / (ap_phases * 1e-3) / 1e9 / peak, 4), "traffic": ap_traffic[0],
                     "traffic_source": ap_traffic[1],
                     "algorithmic_bytes": bap},
        "gpu_launches": int(l1.value - l0.value),
        "clocks": clk,
        "cpu_baseline": {"value": round(2.0 * (m1 + m2) / cpu_s / 1e9, 4), "unit": "GFLOP/s",
                         "cores": oracle.num_threads(), "kind": "port",
                         "sample": f"the whole workload (A·P then R·AP), {reps} times, {cpu_s:.3f} s each"},
        "parity": parity,
    }
    ctx.close()
    return line


def run_served(args):
    """Poisson arrivals (mean --rate req/s for --duration s): 70% A·B with
    operands sized like the batched workload, 30% Galerkin R·A·P on 7-point
    Laplacians (grid side U{32..160}, 2x2x2 aggregation, one Jacobi step,
    omega 2/3); operands are drawn from a resident pool; 120 GB admission
    budget.  Reports completed req/s and p50/p99 latency (submission to
    completion), and the same request sequence as a loop of plain calls."""
    import threading

    import numpy as np
    import torch

    from trident_b200 import ops, workloads
    torch.cuda.set_device(0)
    rng = np.random.Generator(np.random.Philox(args.seed))
    ctx = ops.Context(0)
    tuning = apply_tuning(ctx, "batched")
    ab_pool = []
    for spec in workloads.batched_specs(24, seed=args.seed + 1000):
        A, B = workloads.batched_product(spec)
        ab_pool.append((A.to_device(), B.to_device()))
    rap_pool = []
    for side in rng.integers(32, 161, size=8):
        R, A, P = workloads.galerkin_operands(n=int(side), pts=7, agg=2)
        rap_pool.append((R.to_device(), A.to_device(), P.to_device()))
    def sequence(rate, duration, seed):
        r = np.random.Generator(np.random.Philox(seed))
        n = int(rate * duration)
        kinds = r.random(n) < 0.7
        picks = [int(r.integers(0, len(ab_pool) if k else len(rap_pool))) for k in kinds]
        return n, kinds, picks, r.exponential(1.0 / rate, size=n)

    def serve(rate, duration, seed):
        """Poisson arrivals at `rate` for `duration` s through a fresh server:
        (completed req/s, p50 ms, p99 ms, batches)."""
        n_req, kinds, picks, gaps = sequence(rate, duration, seed)
        srv = ops.Server(ctx, mem_budget=120 << 30, lanes=args.lanes, max_batch=args.max_batch)
        # warm-up: one full batch of the request mix (the lanes' batches map
        # their output memory on the first admissions of that size)
        warm = []
        for i in range(min(n_req, args.max_batch * args.lanes)):
            if kinds[i]:
                warm.append(srv.submit(*ab_pool[picks[i]]))
            else:
                R, A, P = rap_pool[picks[i]]
                warm.append(srv.submit(A, P, R))
        for t in warm:
            srv.wait(t)
            srv.release(t)
        torch.cuda.synchronize()
        tickets = [None] * n_req
        t_start = time.perf_counter()

        def producer():
            due = t_start
            for i in range(n_req):
                due += gaps[i]
                d = due - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                if kinds[i]:
                    A, B = ab_pool[picks[i]]
                    tickets[i] = srv.submit(A, B)
                else:
                    R, A, P = rap_pool[picks[i]]
                    tickets[i] = srv.submit(A, P, R)

        th = threading.Thread(target=producer)
        th.start()
        lat = []
        for i in range(n_req):
            while tickets[i] is None:
                time.sleep(0.0002)
            _, ms = srv.wait(tickets[i])
            lat.append(ms)
            srv.release(tickets[i])
        t_end = time.perf_counter()
        th.join()
        stats = srv.stats()
        srv.close()
        lat = np.array(lat)
        return (n_req / (t_end - t_start), float(np.percentile(lat, 50)), float(np.percentile(lat, 99)),
                stats["batches"], n_req)

    # the offered-rate sequence as plain calls, back to back: the capacity of a
    # loop (warmed up like the server: the first requests once, untimed, so
    # the allocators hold their output sizes)
    n_req, kinds, picks, _ = sequence(args.rate, args.duration, args.seed)

    def plain(i):
        if kinds[i]:
            A, B = ab_pool[picks[i]]
            return ops.spgemm(ctx, A, B)
        R, A, P = rap_pool[picks[i]]
        return ops.spgemm(ctx, R, ops.spgemm(ctx, A, P))

    for i in range(min(n_req, args.max_batch * args.lanes)):
        del_ = plain(i)
        del del_
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(n_req):
        del_ = plain(i)
        del del_
    torch.cuda.synchronize()
    loop_rate = n_req / (time.perf_counter() - t0)
    served, p50, p99, batches, _ = serve(args.rate, args.duration, args.seed)
    # a rate the GPU sustains: 80 % of what the loop of plain calls completes
    sus_rate = 0.8 * loop_rate
    s_served, s_p50, s_p99, s_batches, s_n = serve(sus_rate, args.duration, args.seed + 1)
    line = {
        "metric": "served R·A·P + A·B req/s (Poisson arrivals), p50/p99 latency", "value": round(served, 1),
        "unit": "req/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (resident pool: 24 A·B pairs, 8 R·A·P sets)",
        "config": {"tuning": tuning, "workload": "served", "rate": args.rate, "duration_s": args.duration, "requests": n_req,
                   "ab_share": 0.7, "budget_gb": 120, "lanes": args.lanes, "max_batch": args.max_batch},
        "p50_ms": round(p50, 3), "p99_ms": round(p99, 3), "batches": batches,
        "overloaded": served < 0.95 * args.rate,
        "loop_of_plain_calls": {"req_per_s": round(loop_rate, 1)},
        "speedup_vs_loop": round(served / loop_rate, 3),
        "sustained": {"rate": round(sus_rate, 1), "requests": s_n, "req_per_s": round(s_served, 1),
                      "p50_ms": round(s_p50, 3), "p99_ms": round(s_p99, 3), "batches": s_batches,
                      "note": "offered at 80 % of the plain-call loop's capacity"},
    }
    ctx.close()
    return line


def run_summa(args):
    """R-MAT A·A as a 4 x 4 tile grid with bitmask-compressed tiles, the four
    SUMMA stages in sequence on one GPU (per stage and output tile: masks,
    pack / unpack of A(i,q) and B(q,j), C(i,j) += A'·B').  Scale --scale
    (default 19 here: the tiles, the stage partials and their merges of scale
    20 need more than the GPU's memory at once); one step = the whole SUMMA."""
    import torch

    from trident_b200 import ops, summa, workloads
    scale = args.scale if args.scale != 20 else 19
    torch.cuda.set_device(0)
    A = workloads.rmat(scale=scale, edge_factor=args.edge_factor, seed=args.seed)
    ctx = ops.Context(0)
    tuning = apply_tuning(ctx, "rmat")
    q = 4
    tiles, rb, cb = summa.cut_tiles(A, q)
    dT = [[tiles[i][j].to_device() for j in range(q)] for i in range(q)]
    mults = ops.spgemm_count(ctx, A.to_device(), A.to_device())[0]
    stats = summa.StageStats()
    C = summa.summa(ctx, dT, dT, q, use_masks=True, stats=stats)  # warm-up, sizes
    nnz_c = sum(C[i][j].nnz for i in range(q) for j in range(q))
    del C
    torch.cuda.synchronize()
    modes = {}
    for batched in (False, True):
        summa.summa(ctx, dT, dT, q, use_masks=True, batched=batched)  # warm-up of this mode
        torch.cuda.synchronize()
        times = []
        for _ in range(max(1, args.steps)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            C = summa.summa(ctx, dT, dT, q, use_masks=True, batched=batched)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            del C
        modes["batched_stages" if batched else "tile_by_tile"] = sorted(times)[len(times) // 2]
    best = min(modes, key=modes.get)
    ms = modes[best]
    line = {
        "metric": "A·A SpGEMM GFLOP/s (2 x multiply-adds), FP64, 4x4 SUMMA with bitmask-compressed tiles",
        "value": round(2.0 * mults / (ms * 1e-3) / 1e9, 3), "unit": "GFLOP/s", "n_gpus": 1,
        "steps": len(times), "ms_per_step": round(ms, 3), "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (seeded R-MAT, values U[-1,1])",
        "config": {"tuning": tuning, "workload": f"rmat{scale}_summa4x4", "rows": A.nrows, "nnz_A": A.nnz,
                   "mults": int(mults), "nnz_C": int(nnz_c), "grid": "4x4 tiles, 4 stages x 16 products"},
        "stage_modes_ms": {k: round(v, 3) for k, v in modes.items()}, "mode": best,
        "tiles": {"a_nnz": stats.a_nnz, "a_kept": stats.a_kept, "b_nnz": stats.b_nnz,
                  "b_kept": stats.b_kept, "packed_bytes": stats.packed_bytes,
                  "full_bytes": stats.full_bytes},
    }
    ctx.close()
    return line


def run_coo(args):
    """COO -> CSR on the device (tspg_coo_to_csx) for the coordinates of R-MAT
    scale --scale (default 20: 16.1M entries), shuffled by a seeded
    permutation (the order a reader hands them over); the reference builds the
    CSR on the host (std::sort of the triples by row, then an H2D copy).  One
    step = one build from device-resident COO arrays into preallocated output
    arrays; the CPU baseline is the oracle's restatement of the host builder
    (numpy stable sort) on the same triples."""
    import ctypes as C

    import numpy as np
    import torch

    import oracle
    from trident_b200 import ops, workloads
    from trident_b200._lib import TSPG_ROWS, TspgCsrOut, check, lib
    torch.cuda.set_device(0)
    A = workloads.rmat(scale=args.scale, edge_factor=args.edge_factor, seed=args.seed)
    rows = np.repeat(np.arange(A.nrows, dtype=np.int32), np.diff(A.rowptr))
    perm = np.random.default_rng(args.seed).permutation(A.nnz)
    hr, hc, hv = rows[perm], A.col[perm], A.val[perm]
    dr, dc, dv = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (hr, hc, hv))
    ctx = ops.Context(0)
    M = ops.coo_to_csx(ctx, A.nrows, A.ncols, dr, dc, dv)
    ok = bool(np.array_equal(M.col.cpu().numpy(), A.col) and np.array_equal(M.val.cpu().numpy(), A.val))
    stream = torch.cuda.current_stream()

    def step():
        o = TspgCsrOut()
        o.nrows, o.ncols = A.nrows, A.ncols
        o.rowptr, o.rowptr_bits, o.val_bits = M.rowptr.data_ptr(), 64, 64
        o.col, o.val, o.capacity = M.col.data_ptr(), M.val.data_ptr(), A.nnz
        check(lib.tspg_coo_to_csx(ctx.h, stream.cuda_stream, A.nrows, A.ncols, A.nnz, dr.data_ptr(),
                                  dc.data_ptr(), dv.data_ptr(), 64, TSPG_ROWS, C.byref(o)), "tspg_coo_to_csx")

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    clk = ClockSampler(0)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / args.steps
    peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    algo = A.nnz * (4 + 4 + 8) + A.nnz * (4 + 8) + (A.nrows + 1) * 8  # COO read, CSR written
    t0 = time.perf_counter()
    oracle.coo_to_csx(A.nrows, hr, hc, hv)
    cpu_s = time.perf_counter() - t0
    line = {
        "metric": "COO -> CSR build, M entries/s", "value": round(A.nnz / (ms * 1e-3) / 1e6, 1),
        "unit": "M entries/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": round(ms, 3), "higher_is_better": True, "dtype": "int32 indices, f64 values",
        "data": "synthetic (seeded R-MAT coordinates, shuffled)",
        "config": {"workload": f"rmat{args.scale}_coo", "rows": A.nrows, "nnz": A.nnz, "matches_generator": ok},
        "roofline": {"bound": "hbm", "achieved": round(algo / (ms * 1e-3) / 1e9, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(algo / (ms * 1e-3) / 1e9 / peak, 4), "algorithmic_bytes": algo},
        "cpu_baseline": {"value": round(A.nnz / cpu_s / 1e6, 1), "unit": "M entries/s", "cores": 1, "kind": "port",
                         "sample": f"the whole workload, numpy stable sort by (row, col, position), {cpu_s:.1f} s"},
        "clocks": clocks,
    }
    ctx.close()
    return line


def apply_tuning(ctx, name):
    """Apply the committed autotuner file of a workload (trident_b200/tuning/
    <name>.json, written by `python -m trident_b200.tune`), if there is one;
    returns what goes into the JSON line's config."""
    from trident_b200 import tune
    path = tune.tuning_path(name)
    if not os.path.exists(path):
        return None
    t = ctx.load_tuning(path)
    return {"file": os.path.relpath(path, os.path.dirname(os.path.abspath(__file__))), **t}


def main():
    args = parse()
    if args.impl == "ours" and args.workload in ("batched", "rap", "served", "summa", "coo"):
        fn = {"batched": run_batched, "rap": run_rap, "served": run_served,
              "summa": run_summa, "coo": run_coo}[args.workload]
        print(json.dumps(fn(args)), flush=True)
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    line = run_ours(args, rank, world)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
