"""Single-GPU emulation of Trident's 2D sparse SUMMA with bitmask-compressed tiles.

Mirrors src/sparse_summa.cu:6-146 (stage loop: tile_bcast of A(i,q) and
B(q,j), then sp_mma_hybrid) and the sparsity-aware exchange of
include/spacomm.cuh:165-352 / 962-1091, with every "rank" of the q x q grid
living on one GPU.  For stage q and output tile (i, j):

  mask      = colmask(A_iq) & rowmask(B_qj)         (fused into the flop-count
                                                     pass: tspg_spgemm_count_mask)
  A'_iq     = csc_to_csr(unpack(pack_COLS(A_iq^CSC, mask)))
  B'_qj     = unpack(pack_ROWS(B_qj, mask))
  C_ij     += A'_iq · B'_qj                          (tspg_spgemm_acc)

A column k of A_iq is dropped only when row k of B_qj is empty (and the other
way round), so the product is unchanged; the packed sizes are what the
reference would send.  Tiles are cut on the host (setup, like the reference's
distributed reader); everything per stage runs through the C ABI.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import ops
from ._lib import TSPG_COLS, TSPG_ROWS
from .csr import DeviceCSR, HostCSR


def cut_tiles(M: HostCSR, q: int):
    """q x q tiles of M (rows and columns split evenly, indices rebased)."""
    S = M.to_scipy().tocsr()
    rb = [(M.nrows * i) // q for i in range(q + 1)]
    cb = [(M.ncols * j) // q for j in range(q + 1)]
    tiles = [[None] * q for _ in range(q)]
    for i in range(q):
        rows = S[rb[i]:rb[i + 1], :]
        for j in range(q):
            T = rows[:, cb[j]:cb[j + 1]].tocsr()
            T.sort_indices()
            tiles[i][j] = HostCSR(T.shape[0], T.shape[1], T.indptr.astype(np.int64),
                                  T.indices.astype(np.int32), T.data.astype(np.float64))
    return tiles, rb, cb


def col_mask(ctx, T: DeviceCSR) -> torch.Tensor:
    """Non-empty-column mask of a CSR tile: the row mask of its CSC form."""
    return ops.gen_bitmask(ctx, ops.transpose(ctx, T).rowptr, T.ncols)


@dataclass
class StageStats:
    a_nnz: int = 0
    a_kept: int = 0
    b_nnz: int = 0
    b_kept: int = 0
    packed_bytes: int = 0
    full_bytes: int = 0
    per_stage: list = field(default_factory=list)


def summa(ctx, A_tiles, B_tiles, q: int, use_masks: bool = True, stats: StageStats | None = None,
          batched: bool = False):
    """C tiles of A·B from device tiles A_tiles[i][k], B_tiles[k][j].

    batched=True runs the q*q tile products of a stage as one batch (one
    launch of each persistent kernel per phase, tspg_batch_*), then merges
    every product into its C tile (tspg_spadd) — the split accumulate; the
    default multiplies and accumulates tile by tile (tspg_spgemm_acc)."""
    C = [[None] * q for _ in range(q)]
    batch = ops.Batch(ctx) if batched else None
    # per-tile CSC of A (what the reference keeps with --Acsc), packed by columns
    A_csc = [[ops.transpose(ctx, A_tiles[i][k]) for k in range(q)] for i in range(q)]
    for s in range(q):  # stage
        st = {"stage": s, "a_kept": 0, "b_kept": 0}
        pairs = []
        for i in range(q):
            for j in range(q):
                Aik, Bkj = A_tiles[i][s], B_tiles[s][j]
                if use_masks:
                    mask, _, _ = ops.spgemm_count_mask(ctx, Aik, Bkj)
                    Acsc = A_csc[i][s]  # nrows = tile cols: a CSR over the k dimension
                    abuf, akept = ops.compress(ctx, Acsc, mask, TSPG_ROWS)
                    Ap_csc = ops.unpack(abuf, Acsc.nrows, Acsc.ncols, akept, TSPG_ROWS,
                                        val_bits=Acsc.val_bits, ptr_bits=Acsc.rowptr_bits)
                    Ap = ops.csc_to_csr(ctx, Ap_csc, rowptr_bits=Aik.rowptr_bits)
                    bbuf, bkept = ops.compress(ctx, Bkj, mask, TSPG_ROWS)
                    Bp = ops.unpack(bbuf, Bkj.nrows, Bkj.ncols, bkept, TSPG_ROWS,
                                    val_bits=Bkj.val_bits, ptr_bits=Bkj.rowptr_bits)
                    if stats is not None:
                        stats.a_nnz += Aik.nnz
                        stats.a_kept += akept
                        stats.b_nnz += Bkj.nnz
                        stats.b_kept += bkept
                        stats.packed_bytes += ops.packed_bytes(akept, Acsc.nrows, Acsc.val_bits,
                                                               Acsc.rowptr_bits)
                        stats.packed_bytes += ops.packed_bytes(bkept, Bkj.nrows, Bkj.val_bits,
                                                               Bkj.rowptr_bits)
                        stats.full_bytes += ops.packed_bytes(Aik.nnz, Acsc.nrows, Acsc.val_bits,
                                                             Acsc.rowptr_bits)
                        stats.full_bytes += ops.packed_bytes(Bkj.nnz, Bkj.nrows, Bkj.val_bits,
                                                             Bkj.rowptr_bits)
                    st["a_kept"] += akept
                    st["b_kept"] += bkept
                else:
                    Ap, Bp = Aik, Bkj
                if batch is None:
                    C[i][j] = ops.sp_mma(ctx, Ap, Bp, C[i][j])
                else:
                    pairs.append((i, j, Ap, Bp))
        if batch is not None and pairs:
            batch.clear()
            for _, _, Ap, Bp in pairs:
                batch.add(Ap, Bp)
            batch.run()
            for t, (i, j, _, _) in enumerate(pairs):
                P = batch.result(t)
                # the slab is rewritten by the next stage's run: merge (or copy) out now
                C[i][j] = ops.spadd(ctx, P, C[i][j]) if C[i][j] is not None else _copy(P)
        if stats is not None:
            stats.per_stage.append(st)
    if batch is not None:
        batch.close()
    return C


def _copy(M: DeviceCSR) -> DeviceCSR:
    return DeviceCSR(M.nrows, M.ncols, M.rowptr.clone(), M.col[:max(M.nnz, 1)].clone(),
                     M.val[:max(M.nnz, 1)].clone(), nnz=M.nnz)


def assemble(C_tiles, rb, cb) -> HostCSR:
    """Host CSR of the full C from its q x q tiles (for checking)."""
    import scipy.sparse as sp
    q = len(C_tiles)
    blocks = []
    for i in range(q):
        row = []
        for j in range(q):
            H = C_tiles[i][j].to_host()
            row.append(sp.csr_matrix((H.val, H.col, H.rowptr), shape=(rb[i + 1] - rb[i], cb[j + 1] - cb[j])))
        blocks.append(row)
    M = sp.bmat(blocks, format="csr")
    M.sort_indices()
    return HostCSR(M.shape[0], M.shape[1], M.indptr.astype(np.int64), M.indices.astype(np.int32),
                   M.data.astype(np.float64))
