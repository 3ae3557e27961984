"""Row-panel split of one product C = A·B over several GPUs (one process per GPU).

Row i of C needs only row i of A and all of B, so the rows of A are cut into
contiguous panels of about equal work — the cut points come from the prefix
sum of the per-row products (tspg_spgemm_row_products) — B is replicated to
every rank (one broadcast over NCCL/NVLink from the rank that holds it), and
each rank multiplies its panel on its own GPU.  No reduction follows: rank r's
panel of C is rows [cuts[r], cuts[r + 1]) of C.  This replaces, for one
product, the reference's 2D / 2D-1D tiling with its partial-C merges
(src/hns_spgemm.cu, src/sparse_summa.cu) and node gather of B
(include/tile_holder.cuh:236-330).

The host logic here (cuts, broadcast, assembly) is backend-neutral, so the
multi-rank path is tested with gloo ranks on CPU as well.
"""
from __future__ import annotations

import numpy as np


def panel_cuts(row_products: np.ndarray, nparts: int) -> np.ndarray:
    """Cut rows 0..m into `nparts` contiguous panels of about equal products:
    cuts[k] is the first row whose products before it reach k/nparts of the
    total.  Returns nparts + 1 non-decreasing row indices, cuts[0] = 0,
    cuts[-1] = m; every row lies in exactly one panel."""
    f = np.asarray(row_products, dtype=np.int64)
    m = f.size
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    pre = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(f, out=pre[1:])
    total = int(pre[-1])
    cuts = np.zeros(nparts + 1, dtype=np.int64)
    for k in range(1, nparts):
        target = (total * k + nparts - 1) // nparts
        cuts[k] = int(np.searchsorted(pre, target, side="left"))
    cuts[nparts] = m
    return np.maximum.accumulate(np.minimum(cuts, m))


def panel_rows(cuts: np.ndarray, rank: int) -> tuple[int, int]:
    return int(cuts[rank]), int(cuts[rank + 1])


def broadcast_csr(rowptr, col, val, src: int, device, rowptr_dtype, val_dtype, shape=None):
    """Broadcast a CSR's three arrays from rank `src` (which passes them) to
    every rank (which pass None and get fresh tensors on `device`).  Works
    with any torch.distributed backend: NCCL with CUDA tensors, gloo with CPU
    tensors.  Returns (nrows, ncols, rowptr, col, val)."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank()
    meta = torch.zeros(3, dtype=torch.int64, device=device)
    if rank == src:
        meta[0], meta[1], meta[2] = shape[0], shape[1], col.numel()
    dist.broadcast(meta, src)
    m, n, nnz = (int(x) for x in meta.tolist())
    if rank != src:
        rowptr = torch.empty(m + 1, dtype=rowptr_dtype, device=device)
        col = torch.empty(nnz, dtype=torch.int32, device=device)
        val = torch.empty(nnz, dtype=val_dtype, device=device)
    dist.broadcast(rowptr, src)
    if nnz:
        dist.broadcast(col, src)
        dist.broadcast(val, src)
    return m, n, rowptr, col, val


def assemble(panels, ncols: int):
    """Concatenate host panels (rowptr rebased to 0, col, val) in rank order
    into one host CSR (rowptr, col, val)."""
    rps, cols, vals, off = [np.zeros(1, np.int64)], [], [], 0
    for rp, c, v in panels:
        rp = np.asarray(rp, dtype=np.int64)
        rps.append(rp[1:] + off)
        off += int(rp[-1])
        cols.append(np.asarray(c))
        vals.append(np.asarray(v))
    return (np.concatenate(rps), np.concatenate(cols) if cols else np.zeros(0, np.int32),
            np.concatenate(vals) if vals else np.zeros(0))


def row_products(ctx, A, B, stream=None):
    """Per-row products of A·B on the device (int64 tensor of A.nrows)."""
    import ctypes as C

    import torch

    from ._lib import check, lib
    out = torch.empty(max(A.nrows, 1), dtype=torch.int64, device=A.rowptr.device)
    s = (stream or torch.cuda.current_stream()).cuda_stream
    a, b = A.abi(), B.abi()
    check(lib.tspg_spgemm_row_products(ctx.h, s, C.byref(a), C.byref(b), out.data_ptr()),
          "tspg_spgemm_row_products")
    return out[:A.nrows]


def panel_view(A, r0: int, r1: int, a_rowptr_host: np.ndarray):
    """C-ABI view of rows [r0, r1) of the device CSR A: row offsets advanced
    by r0 (they keep their absolute values), columns and values unchanged."""
    from ._lib import TspgCsr
    nnz = int(a_rowptr_host[r1] - a_rowptr_host[r0])
    esz = A.rowptr.element_size()
    return TspgCsr(r1 - r0, A.ncols, nnz, A.rowptr.data_ptr() + r0 * esz, A.rowptr_bits, A.val_bits,
                   A.col.data_ptr() if A.nnz else None, A.val.data_ptr() if A.nnz else None)
