"""Autotuner of the SpGEMM row binning (tspg_tuning).

The persistent kernels bin rows into warp / 128-thread / 256-thread / CTA
groups by the bounds `sym_lim` (symbolic phase, on min(products, ncols)) and
`num_lim` (numeric phase, on the row's nnz), and size each row's hash table
as pow2 >= hash_load x the row bound.  Which bounds are best depends on the
row-length mix of the workload, so this module sweeps them by coordinate
descent on a representative workload, timing every candidate with CUDA events
(median of `reps` runs after a warm-up run), and writes the winner as JSON:

    {"workload": ..., "device": ..., "tuning": {"sym_lim": [...],
     "num_lim": [...], "hash_load": k}, "ms": best, "default_ms": ...,
     "trials": [[tuning, ms], ...]}

`Context.load_tuning(path)` applies such a file; bench.py applies the
committed file of its workload.  Results do not depend on the tuning (the
GPU tests check that); only the speed does.

    python -m trident_b200.tune --workload batched --out trident_b200/tuning/batched.json
"""
from __future__ import annotations

import argparse
import json
import os
import time

# Candidate bounds per slot; each slot is capped by the table capacity of its
# class (the defaults), and bounds stay non-decreasing over the classes.
SYM_CAP = [512, 2048, 4096, 24576]
NUM_CAP = [256, 1024, 2048, 8192]
SYM_CHOICES = [[128, 256, 512], [1024, 2048], [2048, 3072, 4096], [4096, 6144, 8192, 12288, 24576]]
NUM_CHOICES = [[128, 192, 256], [512, 768, 1024], [1024, 1536, 2048], [2048, 3072, 4096, 6144, 8192]]
LOAD_CHOICES = [2, 4]
# DENSE numeric rows with >= 2^w products (and an output filling >= 1/16 of the
# columns) take the column-window form; 0 = never
WIN_DEFAULT = 0
WIN_CHOICES = [0, 17, 20]
FILL_DEFAULT = 4
FILL_CHOICES = [3, 4, 5, 6]
CLUSTER_DEFAULT = 0
CLUSTER_CHOICES = [0, 2, 4]

TUNING_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning")


def default_tuning() -> dict:
    return {"sym_lim": list(SYM_CAP), "num_lim": list(NUM_CAP), "hash_load": 2, "dense_win_log2": WIN_DEFAULT,
            "dense_win_fill_log2": FILL_DEFAULT, "dense_win_cluster": CLUSTER_DEFAULT}


def valid(t: dict) -> bool:
    """The rule tspg_ctx_set_tuning enforces."""
    for key, cap in (("sym_lim", SYM_CAP), ("num_lim", NUM_CAP)):
        v = t[key]
        if len(v) != 4:
            return False
        for i in range(4):
            if v[i] < 1 or v[i] > cap[i] or (i and v[i] < v[i - 1]):
                return False
    w = t.get("dense_win_log2", WIN_DEFAULT)
    if w != 0 and not 10 <= w <= 40:
        return False
    if not 0 <= t.get("dense_win_fill_log2", FILL_DEFAULT) <= 12:
        return False
    if t.get("dense_win_cluster", CLUSTER_DEFAULT) not in (0, 2, 4, 8):
        return False
    return t["hash_load"] in (2, 4, 8)


def slots():
    """The tuning slots as (key, index, options); index None for a scalar."""
    out = [("sym_lim", i, opts) for i, opts in enumerate(SYM_CHOICES)]
    out += [("num_lim", i, opts) for i, opts in enumerate(NUM_CHOICES)]
    out.append(("hash_load", None, LOAD_CHOICES))
    out.append(("dense_win_log2", None, WIN_CHOICES))
    out.append(("dense_win_fill_log2", None, FILL_CHOICES))
    out.append(("dense_win_cluster", None, CLUSTER_CHOICES))
    return out


_SCALAR_DEFAULT = {"hash_load": 2, "dense_win_log2": WIN_DEFAULT, "dense_win_fill_log2": FILL_DEFAULT,
                   "dense_win_cluster": CLUSTER_DEFAULT}


def with_slot(t: dict, key: str, i, v) -> dict:
    u = {"sym_lim": list(t["sym_lim"]), "num_lim": list(t["num_lim"]), "hash_load": t["hash_load"],
         "dense_win_log2": t.get("dense_win_log2", WIN_DEFAULT),
         "dense_win_fill_log2": t.get("dense_win_fill_log2", FILL_DEFAULT),
         "dense_win_cluster": t.get("dense_win_cluster", CLUSTER_DEFAULT)}
    if i is None:
        u[key] = v
    else:
        u[key][i] = v
    return u


def neighbours(t: dict):
    """Every valid tuning that differs from t in one slot."""
    for key, i, opts in slots():
        for v in opts:
            if v != (t.get(key, _SCALAR_DEFAULT[key]) if i is None else t[key][i]):
                u = with_slot(t, key, i, v)
                if valid(u):
                    yield u


def tuning_path(workload: str) -> str:
    return os.path.join(TUNING_DIR, f"{workload}.json")


# ----------------------------------------------------------------- workloads

def _batched_runner(ctx, products: int, seed: int):
    """A sample of the batched workload (same size distribution) as one batch."""
    from . import ops, workloads
    from ._lib import TSPG_F_B_SORTED
    specs = workloads.batched_specs(products, seed=seed)
    bt = ops.Batch(ctx)
    keep = []
    for spec in specs:
        A, B = workloads.batched_product(spec)
        dA, dB = A.to_device(), B.to_device()
        keep.append((dA, dB))
        bt.add(dA, dB)

    def run():
        return bt.run(TSPG_F_B_SORTED)
    return run, keep


def _rap_runner(ctx, grid: int):
    from . import ops, workloads
    R, A, P = workloads.galerkin_operands(grid)
    dR, dA, dP = R.to_device(), A.to_device(), P.to_device()

    def run():
        AP = ops.spgemm(ctx, dA, dP)
        return ops.spgemm(ctx, dR, AP).nnz
    return run, (dR, dA, dP)


def _rmat_runner(ctx, scale: int):
    from . import ops, workloads
    A = workloads.rmat(scale=scale, edge_factor=16, seed=1)
    dA = A.to_device()

    def run():
        return ops.spgemm(ctx, dA, dA).nnz
    return run, dA


def make_runner(ctx, workload: str, size: int | None = None, seed: int = 101):
    if workload == "batched":
        return _batched_runner(ctx, size or 64, seed)
    if workload == "rap":
        return _rap_runner(ctx, size or 96)
    if workload == "rmat":
        return _rmat_runner(ctx, size or 20)
    raise ValueError(f"unknown workload {workload}")


# ------------------------------------------------------------------- search

def time_run(run, reps: int) -> tuple[float, int]:
    import torch
    out = run()  # warm-up (and graph capture after a tuning change)
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = run()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        if r != out:
            raise RuntimeError(f"result size changed under tuning: {r} != {out}")
    times.sort()
    return times[len(times) // 2], out


def autotune(ctx, run, reps: int = 3, sweeps: int = 2, log=print):
    """Coordinate descent from the defaults; returns (best, best_ms, default_ms, trials)."""
    best = default_tuning()
    ctx.set_tuning(best)
    best_ms, ref = time_run(run, reps)
    default_ms = best_ms
    trials = [[best, best_ms]]
    log(f"default {best} {best_ms:.3f} ms")
    # coordinate descent: one slot at a time, every option of the slot with
    # the others held at the current best; repeat while a sweep improves
    for sweep in range(sweeps):
        improved = False
        for key, i, opts in slots():
            for v in opts:
                cand = with_slot(best, key, i, v)
                if cand == best or not valid(cand):
                    continue
                ctx.set_tuning(cand)
                ms, out = time_run(run, reps)
                if out != ref:
                    raise RuntimeError("output size differs under tuning")
                trials.append([cand, ms])
                if ms < best_ms * 0.99:
                    best, best_ms, improved = cand, ms, True
                    log(f"sweep {sweep}: {best} {best_ms:.3f} ms")
        if not improved:
            break
    ctx.set_tuning(best)
    return best, best_ms, default_ms, trials


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", choices=["batched", "rap", "rmat"], default="batched")
    ap.add_argument("--size", type=int, default=None,
                    help="products (batched), grid side (rap) or scale (rmat)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--sweeps", type=int, default=2)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    import torch

    from . import ops
    ctx = ops.Context(0)
    run, _keep = make_runner(ctx, args.workload, args.size)
    best, best_ms, default_ms, trials = autotune(ctx, run, args.reps, args.sweeps)
    doc = {
        "workload": args.workload,
        "size": args.size,
        "device": torch.cuda.get_device_name(0),
        "date": time.strftime("%Y-%m-%d"),
        "tuning": best,
        "ms": round(best_ms, 4),
        "default_ms": round(default_ms, 4),
        "trials": [[t, round(ms, 4)] for t, ms in trials],
    }
    out = args.out or tuning_path(args.workload)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out, "w") as fh:
        json.dump(doc, fh, indent=1)
    print(json.dumps({k: doc[k] for k in ("workload", "tuning", "ms", "default_ms")}))
    ctx.close()


if __name__ == "__main__":
    main()
