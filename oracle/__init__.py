"""Python binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker or the timed CPU baseline.  The
product never imports it.

Parity pinning: the bitmask functions are pinned to the known answers of the
reference's test/test_compression.cu (tests/golden/kat_bitmask.json); SpGEMM
and merge are "parity unpinned" at the library boundary (KokkosKernels and
cuSPARSE cannot run here and the reference ships no outputs) and are
cross-checked against dense products and scipy in tests/test_oracle.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build() -> None:
    subprocess.run(["make", "-C", _HERE, "CXX=g++"], check=True, capture_output=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    vp, i64 = C.c_void_p, C.c_int64
    lib.orc_num_threads.restype = C.c_int
    lib.orc_set_threads.argtypes = [C.c_int]
    lib.orc_row_mults.restype = i64
    lib.orc_row_mults.argtypes = [i64, i64, vp, vp, vp, vp]
    lib.orc_spgemm_count.restype = i64
    lib.orc_spgemm_count.argtypes = [i64, i64, i64, vp, vp, vp, vp, vp]
    lib.orc_spgemm_numeric.restype = C.c_int
    lib.orc_spgemm_numeric.argtypes = [i64, i64, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.orc_spadd_count.restype = i64
    lib.orc_spadd_count.argtypes = [i64, vp, vp, vp, vp, vp]
    lib.orc_spadd_numeric.restype = C.c_int
    lib.orc_spadd_numeric.argtypes = [i64, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.orc_bitmask_gen.argtypes = [vp, i64, vp]
    lib.orc_bitmask_and.argtypes = [vp, vp, i64, vp]
    lib.orc_pack.restype = i64
    lib.orc_pack.argtypes = [vp, i64, vp, vp, C.c_int, vp, vp, vp, vp]
    return lib


lib = _load()


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _csr(M):
    rp = np.ascontiguousarray(M.rowptr, dtype=np.int64)
    col = np.ascontiguousarray(M.col, dtype=np.int32)
    val = np.ascontiguousarray(M.val, dtype=np.float64)
    return rp, col, val


def set_threads(n: int) -> None:
    lib.orc_set_threads(n)


def num_threads() -> int:
    return lib.orc_num_threads()


def row_mults(A, B, r0: int = 0, r1: int | None = None) -> np.ndarray:
    ap, aj, _ = _csr(A)
    bp, _, _ = _csr(B)
    r1 = A.nrows if r1 is None else r1
    out = np.zeros(max(r1 - r0, 1), dtype=np.int64)
    lib.orc_row_mults(r0, r1, _p(ap), _p(aj), _p(bp), _p(out))
    return out[: r1 - r0]


def spgemm(A, B, r0: int = 0, r1: int | None = None, with_abs: bool = True):
    """C = A·B for rows [r0, r1): returns (rowptr int64 rebased to 0, col, val, abs)."""
    ap, aj, ax = _csr(A)
    bp, bj, bx = _csr(B)
    r1 = A.nrows if r1 is None else r1
    m = r1 - r0
    cnt = np.zeros(max(m, 1), dtype=np.int64)
    lib.orc_spgemm_count(r0, r1, B.ncols, _p(ap), _p(aj), _p(bp), _p(bj), _p(cnt))
    cp_full = np.zeros(A.nrows + 1, dtype=np.int64)
    cp_full[r0 + 1: r1 + 1] = np.cumsum(cnt[:m])
    cp_full[r1 + 1:] = cp_full[r1]
    nnz = int(cp_full[r1])
    cj = np.zeros(max(nnz, 1), dtype=np.int32)
    cx = np.zeros(max(nnz, 1), dtype=np.float64)
    ca = np.zeros(max(nnz, 1), dtype=np.float64) if with_abs else None
    lib.orc_spgemm_numeric(r0, r1, B.ncols, _p(ap), _p(aj), _p(ax), _p(bp), _p(bj), _p(bx), _p(cp_full),
                           _p(cj), _p(cx), _p(ca) if with_abs else None)
    rp = cp_full[r0: r1 + 1] - cp_full[r0]
    return rp, cj[:nnz], cx[:nnz], (ca[:nnz] if with_abs else None)


def spadd(A, B):
    ap, aj, ax = _csr(A)
    bp, bj, bx = _csr(B)
    m = A.nrows
    cnt = np.zeros(max(m, 1), dtype=np.int64)
    lib.orc_spadd_count(m, _p(ap), _p(aj), _p(bp), _p(bj), _p(cnt))
    cp = np.zeros(m + 1, dtype=np.int64)
    cp[1:] = np.cumsum(cnt[:m])
    nnz = int(cp[-1])
    cj = np.zeros(max(nnz, 1), dtype=np.int32)
    cx = np.zeros(max(nnz, 1), dtype=np.float64)
    lib.orc_spadd_numeric(m, _p(ap), _p(aj), _p(ax), _p(bp), _p(bj), _p(bx), _p(cp), _p(cj), _p(cx))
    return cp, cj[:nnz], cx[:nnz]


def bitmask_gen(ptr, n: int) -> np.ndarray:
    p = np.ascontiguousarray(ptr, dtype=np.int64)
    out = np.zeros(max((n + 7) // 8, 1), dtype=np.uint8)
    lib.orc_bitmask_gen(_p(p), n, _p(out))
    return out[: (n + 7) // 8]


def bitmask_and(a, b) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint8)
    b = np.ascontiguousarray(b, dtype=np.uint8)
    out = np.zeros_like(a)
    lib.orc_bitmask_and(_p(a), _p(b), a.size, _p(out))
    return out


def pack(ptr, idx, val, mask):
    """select_entries + select_ptrs on one tile: (kept ptr int64, idx, val)."""
    p = np.ascontiguousarray(ptr, dtype=np.int64)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    val = np.ascontiguousarray(val)
    mask = np.ascontiguousarray(mask, dtype=np.uint8)
    length = p.size - 1
    nnz = int(p[-1])
    optr = np.zeros(length + 1, dtype=np.int64)
    oidx = np.zeros(max(nnz, 1), dtype=np.int32)
    oval = np.zeros(max(nnz, 1), dtype=val.dtype)
    kept = lib.orc_pack(_p(p), length, _p(idx), _p(val), val.dtype.itemsize, _p(mask), _p(optr), _p(oidx),
                        _p(oval))
    return optr, oidx[:kept], oval[:kept]


def transpose(M):
    """T = M^T as CSR with sorted rows: the CSR of a CSC tile, the job of
    cusparse_csc_to_csr (include/cusparse_helpers.cuh:607-705) and
    LocalMatrix::csc_to_csr (include/KokkosWrap.hpp:442-531).  Restated as a
    stable counting sort of M's entries by column: row j of T lists the
    entries of column j of M in M's row order (repeated entries kept).
    Returns (rowptr int64 of M.ncols + 1, col int32, val)."""
    rp = np.asarray(M.rowptr, dtype=np.int64)
    col = np.asarray(M.col, dtype=np.int64)
    rows = np.repeat(np.arange(M.nrows, dtype=np.int64), np.diff(rp))
    order = np.argsort(col, kind="stable")
    trp = np.zeros(M.ncols + 1, dtype=np.int64)
    np.cumsum(np.bincount(col, minlength=M.ncols), out=trp[1:])
    return trp, rows[order].astype(np.int32), np.asarray(M.val)[order]


def coo_to_csx(nmaj: int, maj, mnr, val):
    """COO -> compressed by `maj`: the host builders coo_to_row_csx /
    coo_to_col_csx (include/cusparse_helpers.cuh:17-131) and coo_to_kokkos_crs
    / _ccs (include/kokkos_helpers.cuh:52-352) sort the triples by the major
    index (std::sort, so the order inside a segment is unspecified), count each
    major index into ptr[i + 1], take the inclusive scan and emit the minor
    indices and values in sorted order, repeated entries kept.  Restated with
    the order inside a segment fixed to (minor index, input position), the
    order the device builder produces.  Returns (ptr int64, minor int32, val)."""
    maj = np.asarray(maj, dtype=np.int64)
    mnr = np.asarray(mnr, dtype=np.int64)
    order = np.lexsort((np.arange(maj.size), mnr, maj))
    ptr = np.zeros(nmaj + 1, dtype=np.int64)
    np.add.at(ptr, maj + 1, 1)
    ptr = np.cumsum(ptr)
    return ptr, mnr[order].astype(np.int32), np.asarray(val)[order]


def mcl_normalize(rowptr, val):
    """Rows scaled to sum 1; a row whose sum is <= 1e-20 becomes zeros
    (normalize, src/mcl.cu:97-127: row sums in row order, then v / s)."""
    rp = np.asarray(rowptr, dtype=np.int64)
    v = np.array(val, copy=True)
    for i in range(rp.size - 1):
        seg = v[rp[i]:rp[i + 1]]
        s = seg.sum(dtype=v.dtype)
        v[rp[i]:rp[i + 1]] = seg / s if s > 1e-20 else 0
    return v


def mcl_inflate(rowptr, val, power):
    """Values raised to `power`, then normalized (inflation, src/mcl.cu:130-149)."""
    v = np.power(np.asarray(val), np.asarray(power, dtype=np.asarray(val).dtype))
    return mcl_normalize(rowptr, v)


def mcl_prune(rowptr, col, val, tol):
    """The entries with |v| > tol in their order, with the new row offsets
    (prune, src/mcl.cu:56-93: per-row kept counts, inclusive scan)."""
    rp = np.asarray(rowptr, dtype=np.int64)
    v = np.asarray(val)
    keep = np.abs(v) > np.asarray(tol, dtype=v.dtype)
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    cnt = np.bincount(rows[keep], minlength=rp.size - 1)
    return np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64), np.asarray(col)[keep], v[keep]
