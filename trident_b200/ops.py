"""Python host API over the C ABI (device operands as torch CUDA tensors).

Function names follow the reference's operators: ``spgemm`` / ``sp_mma`` /
``spadd`` are LocalMatrix::spgemm / sp_mma / spadd
(include/KokkosWrap.hpp:60-66), ``spgeam`` is cusparse_spgeam
(include/cusparse_helpers.cuh:799), ``gen_bitmask`` / ``intersect_bitmasks`` /
``compress`` are SpaComm::gen_bitmask / intersect_bitmasks /
SpaCommHandler::Compress (include/spacomm.cuh:29,126,962).
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import (ALLOC_FN, TSPG_COLS, TSPG_EINVAL, TSPG_ENOMEM, TSPG_OK, TSPG_ROWS, TspgCsr, TspgTuning,
                   TspgCsrOut, TspgError, check, lib)
from .csr import DeviceCSR


def _stream_ptr(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


class _TorchAlloc:
    """Allocator callback handing torch tensors to the library (kept alive here).

    The callback never raises: an exception inside a ctypes callback is
    printed and the C caller receives an undefined pointer, so a failed
    allocation returns NULL instead, which the library reports as
    TSPG_ENOMEM.  The callback closes over the tensor list, not over this
    object, so no reference cycle keeps the outputs alive after the call."""

    def __init__(self, device):
        self.device = device
        tensors = self.tensors = []

        def _alloc(user, nbytes, stream):
            try:
                t = torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=device)
            except Exception:  # out of device memory: NULL -> TSPG_ENOMEM
                return None
            tensors.append(t)
            return t.data_ptr()

        self.cb = ALLOC_FN(_alloc)


class Context:
    """A library context: device, workspace pool (resident), budget."""

    def __init__(self, device: int = 0, budget: int = 0):
        torch.cuda.set_device(device)
        self.device = device
        h = C.c_void_p()
        check(lib.tspg_ctx_create(device, budget, C.byref(h)), "tspg_ctx_create")
        self.h = h

    def close(self):
        if self.h:
            lib.tspg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mem(self):
        a, b = C.c_size_t(), C.c_size_t()
        check(lib.tspg_ctx_mem(self.h, C.byref(a), C.byref(b)), "tspg_ctx_mem")
        return a.value, b.value

    def get_tuning(self) -> dict:
        """Row binning in force: {"sym_lim": [4], "num_lim": [4], "hash_load": k,
        "dense_win_log2": w, "dense_win_fill_log2": d, "dense_win_cluster": k}."""
        t = TspgTuning()
        check(lib.tspg_ctx_get_tuning(self.h, C.byref(t)), "tspg_ctx_get_tuning")
        return {"sym_lim": list(t.sym_lim), "num_lim": list(t.num_lim), "hash_load": t.hash_load,
                "dense_win_log2": t.dense_win_log2, "dense_win_fill_log2": t.dense_win_fill_log2,
                "dense_win_cluster": t.dense_win_cluster}

    def set_tuning(self, tuning: dict):
        """Set the row binning (keys as get_tuning returns; missing keys keep
        their current values).  Raises TspgError(TSPG_EINVAL) when a bound is
        out of range."""
        cur = self.get_tuning()
        keys = ("sym_lim", "num_lim", "hash_load", "dense_win_log2", "dense_win_fill_log2", "dense_win_cluster")
        cur.update({k: tuning[k] for k in keys if k in tuning})
        t = TspgTuning()
        for i in range(4):
            t.sym_lim[i] = int(cur["sym_lim"][i])
            t.num_lim[i] = int(cur["num_lim"][i])
        t.hash_load = int(cur["hash_load"])
        t.dense_win_log2 = int(cur["dense_win_log2"])
        t.dense_win_fill_log2 = int(cur["dense_win_fill_log2"])
        t.dense_win_cluster = int(cur["dense_win_cluster"])
        check(lib.tspg_ctx_set_tuning(self.h, C.byref(t)), "tspg_ctx_set_tuning")

    def load_tuning(self, path: str) -> dict:
        """Apply the "tuning" object of an autotuner JSON file; returns it."""
        import json
        with open(path) as fh:
            doc = json.load(fh)
        self.set_tuning(doc["tuning"])
        return doc["tuning"]


def _out_struct(nrows, ncols, rowptr, val_bits, col=None, val=None, capacity=0, alloc=None):
    o = TspgCsrOut()
    o.nrows, o.ncols = nrows, ncols
    o.rowptr = rowptr.data_ptr()
    o.rowptr_bits = 32 if rowptr.element_size() == 4 else 64
    o.val_bits = val_bits
    o.col = col.data_ptr() if col is not None else None
    o.val = val.data_ptr() if val is not None else None
    o.capacity = capacity
    if alloc is not None:
        o.alloc = alloc.cb
    return o


def _vdtype(bits):
    return torch.float64 if bits == 64 else torch.float32


class Plan:
    """Symbolic result kept for numeric re-runs (cusparse_spgemm_reuse)."""

    def __init__(self, ctx: Context, A: DeviceCSR, B: DeviceCSR, flags: int = 0, stream=None):
        self.ctx = ctx
        h = C.c_void_p()
        nnz = C.c_int64()
        a, b = A.abi(), B.abi()
        check(lib.tspg_spgemm_symbolic(ctx.h, _stream_ptr(stream), C.byref(a), C.byref(b), flags,
                                       C.byref(h), C.byref(nnz)), "tspg_spgemm_symbolic")
        self.h = h
        self.c_nnz = nnz.value
        self.shape = (A.nrows, B.ncols)

    def numeric(self, A: DeviceCSR, B: DeviceCSR, rowptr_bits: int = 64, stream=None) -> DeviceCSR:
        m, n = self.shape
        dev = A.rowptr.device
        rp = torch.empty(m + 1, dtype=torch.int32 if rowptr_bits == 32 else torch.int64, device=dev)
        col = torch.empty(max(self.c_nnz, 1), dtype=torch.int32, device=dev)
        val = torch.empty(max(self.c_nnz, 1), dtype=_vdtype(A.val_bits), device=dev)
        o = _out_struct(m, n, rp, A.val_bits, col, val, self.c_nnz)
        a, b = A.abi(), B.abi()
        check(lib.tspg_spgemm_numeric(self.ctx.h, _stream_ptr(stream), self.h, C.byref(a), C.byref(b),
                                      C.byref(o)), "tspg_spgemm_numeric")
        return DeviceCSR(m, n, rp, col, val, nnz=self.c_nnz)

    def close(self):
        if self.h:
            lib.tspg_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spgemm(ctx: Context, A: DeviceCSR, B: DeviceCSR, rowptr_bits: int = 64, flags: int = 0,
           stream=None) -> DeviceCSR:
    """C = A·B (LocalMatrix::spgemm, include/KokkosWrap.hpp:367-391): one
    tspg_spgemm call, its column and value arrays from the allocator hook once
    nnz(C) is known (a plan kept for new values is `Plan`)."""
    m, n = A.nrows, B.ncols
    rp = torch.empty(m + 1, dtype=torch.int32 if rowptr_bits == 32 else torch.int64, device=A.rowptr.device)
    alloc = _TorchAlloc(A.rowptr.device)
    o = _out_struct(m, n, rp, A.val_bits, alloc=alloc)
    a, b = A.abi(), B.abi()
    check(lib.tspg_spgemm(ctx.h, _stream_ptr(stream), C.byref(a), C.byref(b), C.byref(o), flags), "tspg_spgemm")
    return _finish(o, rp, alloc, A.val_bits)


def spgemm_count(ctx: Context, A: DeviceCSR, B: DeviceCSR, stream=None):
    """(mults, sum_i min(mults_i, ncols)) — the flop-count pass."""
    mults, up = C.c_int64(), C.c_int64()
    a, b = A.abi(), B.abi()
    check(lib.tspg_spgemm_count(ctx.h, _stream_ptr(stream), C.byref(a), C.byref(b), C.byref(mults),
                                C.byref(up)), "tspg_spgemm_count")
    return mults.value, up.value


def spgemm_count_mask(ctx: Context, A: DeviceCSR, B: DeviceCSR, stream=None):
    """(mask, mults, sum_i min(mults_i, ncols)): the flop-count pass fused
    with the stage mask colmask(A) & rowmask(B) (ceil(ncols(A) / 8) bytes)."""
    mults, up = C.c_int64(), C.c_int64()
    a, b = A.abi(), B.abi()
    n = (A.ncols + 7) // 8
    out = torch.empty(max(n, 1), dtype=torch.uint8, device=A.rowptr.device)
    check(lib.tspg_spgemm_count_mask(ctx.h, _stream_ptr(stream), C.byref(a), C.byref(b), out.data_ptr(),
                                     C.byref(mults), C.byref(up)), "tspg_spgemm_count_mask")
    return out[:n], mults.value, up.value


def _finish(o: TspgCsrOut, rp, alloc: _TorchAlloc, val_bits: int) -> DeviceCSR:
    nnz = int(o.nnz)
    if nnz == 0:
        col = torch.empty(1, dtype=torch.int32, device=rp.device)
        val = torch.empty(1, dtype=_vdtype(val_bits), device=rp.device)
        return DeviceCSR(int(o.nrows), int(o.ncols), rp, col, val, nnz=0)
    if len(alloc.tensors) < 2:
        raise TspgError(TSPG_ENOMEM, "output allocation")
    colbuf, valbuf = alloc.tensors[-2], alloc.tensors[-1]
    col = colbuf.view(torch.int32)[:nnz]
    val = valbuf.view(_vdtype(val_bits))[:nnz]
    return DeviceCSR(int(o.nrows), int(o.ncols), rp, col, val, nnz=nnz)


def sp_mma(ctx: Context, A: DeviceCSR, B: DeviceCSR, C_in: DeviceCSR | None, rowptr_bits: int = 64,
           flags: int = 0, stream=None) -> DeviceCSR:
    """C_out = C_in + A·B (LocalMatrix::sp_mma / sp_mma_hybrid)."""
    m, n = A.nrows, B.ncols
    rp = torch.empty(m + 1, dtype=torch.int32 if rowptr_bits == 32 else torch.int64, device=A.rowptr.device)
    alloc = _TorchAlloc(A.rowptr.device)
    o = _out_struct(m, n, rp, A.val_bits, alloc=alloc)
    a, b = A.abi(), B.abi()
    cin = C_in.abi() if C_in is not None else None
    check(lib.tspg_spgemm_acc(ctx.h, _stream_ptr(stream), C.byref(a), C.byref(b),
                              C.byref(cin) if cin is not None else None, C.byref(o), flags),
          "tspg_spgemm_acc")
    return _finish(o, rp, alloc, A.val_bits)


def spadd(ctx: Context, A: DeviceCSR, B: DeviceCSR, rowptr_bits: int = 64, stream=None) -> DeviceCSR:
    """C = A + B, union pattern (cusparse_spgeam / LocalMatrix::spadd)."""
    m, n = A.nrows, A.ncols
    rp = torch.empty(m + 1, dtype=torch.int32 if rowptr_bits == 32 else torch.int64, device=A.rowptr.device)
    alloc = _TorchAlloc(A.rowptr.device)
    o = _out_struct(m, n, rp, A.val_bits, alloc=alloc)
    a, b = A.abi(), B.abi()
    check(lib.tspg_spadd(ctx.h, _stream_ptr(stream), C.byref(a), C.byref(b), C.byref(o)), "tspg_spadd")
    return _finish(o, rp, alloc, A.val_bits)


spgeam = spadd


def transpose(ctx: Context, M: DeviceCSR, rowptr_bits: int = 64, stream=None) -> DeviceCSR:
    """T = M^T, rows sorted (csc_to_csr: a CSC tile is the CSR of its transpose)."""
    rp = torch.empty(M.ncols + 1, dtype=torch.int32 if rowptr_bits == 32 else torch.int64,
                     device=M.rowptr.device)
    alloc = _TorchAlloc(M.rowptr.device)
    o = _out_struct(M.ncols, M.nrows, rp, M.val_bits, alloc=alloc)
    m = M.abi()
    check(lib.tspg_transpose(ctx.h, _stream_ptr(stream), C.byref(m), C.byref(o)), "tspg_transpose")
    return _finish(o, rp, alloc, M.val_bits)


csc_to_csr = transpose


def coo_to_csx(ctx: Context, nrows: int, ncols: int, row: torch.Tensor, col: torch.Tensor,
               val: torch.Tensor, major: int = TSPG_ROWS, rowptr_bits: int = 64,
               stream=None) -> DeviceCSR:
    """Device COO (int32 row, col; FP64 / FP32 values) -> CSR (TSPG_ROWS) or
    CSC (TSPG_COLS, returned as the CSR of the transpose); repeated entries
    kept, each segment ordered by minor index then input position."""
    nnz = int(row.numel())
    if col.numel() != nnz or val.numel() != nnz or row.dtype != torch.int32 or col.dtype != torch.int32:
        raise TspgError(TSPG_EINVAL, "coo_to_csx (int32 row / col and values of one length)")
    vb = 64 if val.dtype == torch.float64 else 32
    nmaj, nmin = (nrows, ncols) if major == TSPG_ROWS else (ncols, nrows)
    rp = torch.empty(nmaj + 1, dtype=torch.int32 if rowptr_bits == 32 else torch.int64, device=row.device)
    alloc = _TorchAlloc(row.device)
    o = _out_struct(nmaj, nmin, rp, vb, alloc=alloc)
    check(lib.tspg_coo_to_csx(ctx.h, _stream_ptr(stream), nrows, ncols, nnz, row.data_ptr(), col.data_ptr(),
                              val.data_ptr(), vb, major, C.byref(o)), "tspg_coo_to_csx")
    return _finish(o, rp, alloc, vb)


def mcl_normalize(ctx: Context, M: DeviceCSR, stream=None) -> DeviceCSR:
    """Rows of M scaled to sum 1 in place (rows summing to <= 1e-20 become 0)."""
    m = M.abi()
    check(lib.tspg_mcl_normalize(ctx.h, _stream_ptr(stream), C.byref(m), M.val.data_ptr()),
          "tspg_mcl_normalize")
    return M


def mcl_inflate(ctx: Context, M: DeviceCSR, power: float = 2.0, stream=None) -> DeviceCSR:
    """Values of M raised to `power`, then rows normalized, in place."""
    m = M.abi()
    check(lib.tspg_mcl_inflate(ctx.h, _stream_ptr(stream), C.byref(m), float(power), M.val.data_ptr()),
          "tspg_mcl_inflate")
    return M


def mcl_prune(ctx: Context, M: DeviceCSR, tol: float, rowptr_bits: int = 64, stream=None) -> DeviceCSR:
    """The entries of M with |v| > tol, as a new CSR."""
    rp = torch.empty(M.nrows + 1, dtype=torch.int32 if rowptr_bits == 32 else torch.int64,
                     device=M.rowptr.device)
    alloc = _TorchAlloc(M.rowptr.device)
    o = _out_struct(M.nrows, M.ncols, rp, M.val_bits, alloc=alloc)
    m = M.abi()
    check(lib.tspg_mcl_prune(ctx.h, _stream_ptr(stream), C.byref(m), float(tol), C.byref(o)),
          "tspg_mcl_prune")
    return _finish(o, rp, alloc, M.val_bits)


def gen_bitmask(ctx: Context, ptr: torch.Tensor, n: int, stream=None) -> torch.Tensor:
    """Bit i of the mask = segment i of ptr non-empty (SpaComm::gen_bitmask, MASK_SIZE 8)."""
    out = torch.empty(max((n + 7) // 8, 1), dtype=torch.uint8, device=ptr.device)
    bits = 32 if ptr.element_size() == 4 else 64
    check(lib.tspg_bitmask_gen(ctx.h, _stream_ptr(stream), ptr.data_ptr(), bits, n, out.data_ptr()),
          "tspg_bitmask_gen")
    return out[: (n + 7) // 8]


def intersect_bitmasks(ctx: Context, a: torch.Tensor, b: torch.Tensor, out: torch.Tensor | None = None,
                       stream=None) -> torch.Tensor:
    n = a.numel()
    out = torch.empty_like(a) if out is None else out
    check(lib.tspg_bitmask_and(ctx.h, _stream_ptr(stream), a.data_ptr(), b.data_ptr(), n, out.data_ptr()),
          "tspg_bitmask_and")
    return out


def packed_bytes(nnz: int, ptr_len: int, val_bits: int = 64, ptr_bits: int = 32) -> int:
    return int(lib.tspg_packed_bytes(nnz, ptr_len, val_bits, ptr_bits))


def compress(ctx: Context, M: DeviceCSR, mask: torch.Tensor, major: int = TSPG_ROWS,
             out: torch.Tensor | None = None, stream=None):
    """Pack one tile by its segment mask; returns (wire buffer, kept nnz)."""
    length = M.nrows if major == TSPG_ROWS else M.ncols
    cap = packed_bytes(M.nnz, length, M.val_bits, M.rowptr_bits)
    if out is None:
        out = torch.empty(max(cap, 16), dtype=torch.uint8, device=M.rowptr.device)
    kept = C.c_int64()
    m = M.abi()
    check(lib.tspg_pack(ctx.h, _stream_ptr(stream), C.byref(m), major, mask.data_ptr(), out.data_ptr(),
                        out.numel(), None, C.byref(kept)), "tspg_pack")
    return out, kept.value


def unpack(buf: torch.Tensor, nrows: int, ncols: int, nnz: int, major: int = TSPG_ROWS,
           val_bits: int = 64, ptr_bits: int = 32) -> DeviceCSR:
    """View a packed tile as a CSX (TileHolder::form_mmiocsx); shares buf's memory."""
    v = TspgCsr()
    check(lib.tspg_unpack(buf.data_ptr(), nrows, ncols, major, nnz, val_bits, ptr_bits, C.byref(v)),
          "tspg_unpack")
    base = buf.data_ptr()
    length = nrows if major == TSPG_ROWS else ncols
    vb, pb = val_bits // 8, ptr_bits // 8
    val = buf[0: nnz * vb].view(_vdtype(val_bits))
    col = buf[v.col - base: v.col - base + nnz * 4].view(torch.int32)
    off = v.rowptr - base
    rp = buf[off: off + (length + 1) * pb].view(torch.int32 if ptr_bits == 32 else torch.int64)
    return DeviceCSR(nrows, ncols, rp, col, val, nnz=nnz)


__all__ = ["Context", "Plan", "spgemm", "spgemm_count", "spgemm_count_mask", "sp_mma", "spadd", "spgeam", "transpose",
           "csc_to_csr", "coo_to_csx", "mcl_normalize", "mcl_inflate", "mcl_prune", "gen_bitmask",
           "intersect_bitmasks", "compress", "unpack", "packed_bytes", "TSPG_ROWS", "TSPG_COLS",
           "TspgError", "TSPG_OK", "TSPG_ENOMEM"]


class Batch:
    """Many independent products in one launch of each persistent kernel per phase
    (tspg_batch_*).  Operands are borrowed: keep the DeviceCSR objects alive."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = C.c_void_p()
        check(lib.tspg_batch_create(ctx.h, C.byref(h)), "tspg_batch_create")
        self.h = h
        self._keep = []

    def add(self, A: DeviceCSR, B: DeviceCSR) -> int:
        a, b = A.abi(), B.abi()
        i = C.c_int()
        check(lib.tspg_batch_add(self.h, C.byref(a), C.byref(b), C.byref(i)), "tspg_batch_add")
        self._keep.append((A, B))
        return i.value

    def clear(self):
        check(lib.tspg_batch_clear(self.h), "tspg_batch_clear")
        self._keep = []

    def run(self, flags: int = 0, stream=None) -> int:
        tot = C.c_int64()
        check(lib.tspg_batch_run(self.h, _stream_ptr(stream), flags, C.byref(tot)), "tspg_batch_run")
        return tot.value

    def count(self, stream=None) -> list[tuple[int, int]]:
        """(mults, sum_i min(mults_i, ncols)) of every product, one launch."""
        n = len(self._keep)
        mults, up = (C.c_int64 * max(n, 1))(), (C.c_int64 * max(n, 1))()
        check(lib.tspg_batch_count(self.h, _stream_ptr(stream), mults, up), "tspg_batch_count")
        return [(mults[i], up[i]) for i in range(n)]

    def result(self, i: int) -> DeviceCSR:
        """Result i as a DeviceCSR whose tensors alias the batch's output slab."""
        v = TspgCsr()
        check(lib.tspg_batch_result(self.h, i, C.byref(v)), "tspg_batch_result")
        return _alias_csr(v)

    def __len__(self):
        return len(self._keep)

    def close(self):
        if self.h:
            lib.tspg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _alias_csr(v: TspgCsr) -> DeviceCSR:
    """Zero-copy torch views over device arrays owned by the library."""
    nnz = int(v.nnz)
    vdt = _vdtype(v.val_bits)
    rdt = torch.int32 if v.rowptr_bits == 32 else torch.int64
    rp = _device_view(v.rowptr, int(v.nrows) + 1, rdt)
    col = _device_view(v.col, max(nnz, 1), torch.int32) if nnz else torch.empty(1, dtype=torch.int32, device="cuda")
    val = _device_view(v.val, max(nnz, 1), vdt) if nnz else torch.empty(1, dtype=vdt, device="cuda")
    return DeviceCSR(int(v.nrows), int(v.ncols), rp, col, val, nnz=nnz)


def _device_view(ptr: int, count: int, dtype) -> torch.Tensor:
    """A torch tensor over `count` elements of library-owned device memory."""
    itemsize = torch.empty(0, dtype=dtype).element_size()

    class _Arr:
        __cuda_array_interface__ = {
            "shape": (count,),
            "typestr": {torch.int32: "<i4", torch.int64: "<i8", torch.float64: "<f8",
                        torch.float32: "<f4"}[dtype],
            "data": (int(ptr), False),
            "version": 3,
        }

    t = torch.as_tensor(_Arr(), device="cuda")
    assert t.element_size() == itemsize
    return t


__all__ += ["Batch"]


class Server:
    """Continuous-batching server (tspg_server_*): A·B and R·(A·P) requests with
    device-resident operands, admitted by the output upper bound."""

    def __init__(self, ctx: Context, mem_budget: int, lanes: int = 2, max_batch: int = 64):
        from ._lib import TspgServerConfig
        cfg = TspgServerConfig(mem_budget, lanes, max_batch)
        h = C.c_void_p()
        check(lib.tspg_server_create(ctx.h, C.byref(cfg), C.byref(h)), "tspg_server_create")
        self.h = h
        self._ops = {}

    def submit(self, A: DeviceCSR, B: DeviceCSR, R: DeviceCSR | None = None) -> int:
        from ._lib import TSPG_REQ_AB, TSPG_REQ_RAP
        a, b = A.abi(), B.abi()
        r = R.abi() if R is not None else None
        t = C.c_int64()
        check(lib.tspg_server_submit(self.h, TSPG_REQ_RAP if R is not None else TSPG_REQ_AB, C.byref(a),
                                     C.byref(b), C.byref(r) if r is not None else None, C.byref(t)),
              "tspg_server_submit")
        self._ops[t.value] = (A, B, R)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(DeviceCSR view of the result, latency ms); valid until release()."""
        v = TspgCsr()
        lat = C.c_double()
        check(lib.tspg_server_wait(self.h, ticket, timeout_ms, C.byref(v), C.byref(lat)), "tspg_server_wait")
        return _alias_csr(v), lat.value

    def release(self, ticket: int):
        check(lib.tspg_server_release(self.h, ticket), "tspg_server_release")
        self._ops.pop(ticket, None)

    def stats(self):
        b, c, q, r = C.c_int64(), C.c_int64(), C.c_int64(), C.c_size_t()
        st = lib.tspg_server_stats(self.h, C.byref(b), C.byref(c), C.byref(q), C.byref(r))
        return {"batches": b.value, "completed": c.value, "queued": q.value, "reserved": r.value, "status": st}

    def close(self):
        if self.h:
            lib.tspg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ += ["Server"]
