"""Shared checks: compare a device result with the oracle on the same inputs."""
import numpy as np

import oracle
from trident_b200.csr import HostCSR

# FP64 values: |x - y| <= TOL64 * max(|y|, sum |a_ik b_kj|)  (summation order only)
TOL64 = 1e-12
# FP32 twin: same form with the float epsilon scale
TOL32 = 2e-5


def random_csr(m, n, density=None, per_row=None, seed=0, dtype=np.float64, sort=True, dup=False):
    """m x n CSR with binomial(n, density) or fixed per_row entries per row.

    sort=False shuffles each row; dup=True draws columns with replacement
    (repeated columns inside a row)."""
    rng = np.random.default_rng(seed)
    rp = np.zeros(m + 1, dtype=np.int64)
    cols = []
    for i in range(m):
        k = per_row if per_row is not None else rng.binomial(n, density)
        k = int(min(k, n)) if not dup else int(k)
        c = rng.choice(n, size=k, replace=dup) if k and n else np.zeros(0, dtype=np.int64)
        c = np.sort(c) if sort else rng.permutation(c)
        cols.append(c)
        rp[i + 1] = rp[i] + len(c)
    col = np.concatenate(cols).astype(np.int32) if cols else np.zeros(0, np.int32)
    val = rng.uniform(-1, 1, size=col.size).astype(dtype)
    return HostCSR(m, n, rp, col, val)


def check_product(C, A, B, tol=TOL64):
    """Structure bit-exact (sorted canonical CSR), values within tol."""
    H = C.to_host() if not isinstance(C, HostCSR) else C
    rp, cj, cx, ca = oracle.spgemm(A, B)
    assert H.rowptr.shape == rp.shape
    np.testing.assert_array_equal(H.rowptr.astype(np.int64), rp)
    np.testing.assert_array_equal(H.col, cj)
    err = np.abs(H.val.astype(np.float64) - cx)
    bound = tol * np.maximum(np.abs(cx), ca)
    bad = np.nonzero(err > bound)[0]
    assert bad.size == 0, f"{bad.size} values out of tolerance, worst {err[bad].max()} at {bad[:5]}"
    return H


def check_sum(C, A, B, tol=TOL64):
    H = C.to_host() if not isinstance(C, HostCSR) else C
    rp, cj, cx = oracle.spadd(A, B)
    np.testing.assert_array_equal(H.rowptr.astype(np.int64), rp)
    np.testing.assert_array_equal(H.col, cj)
    np.testing.assert_allclose(H.val, cx, rtol=tol, atol=tol)
    return H


def spgemm_poisoned(ctx, A, B, flags=0):
    """C = A·B through the C ABI into output arrays pre-filled with garbage
    (row offsets -3, columns -7, values NaN), so an entry the kernels fail to
    write cannot pass for a stale result of an earlier call that the caching
    allocator handed back."""
    import ctypes as C

    import torch

    from trident_b200 import ops
    from trident_b200._lib import TspgCsrOut, check, lib
    from trident_b200.csr import DeviceCSR
    plan = ops.Plan(ctx, A, B, flags)
    nnz = plan.c_nnz
    plan.close()
    rp = torch.full((A.nrows + 1,), -3, dtype=torch.int64, device="cuda")
    col = torch.full((max(nnz, 1),), -7, dtype=torch.int32, device="cuda")
    val = torch.full((max(nnz, 1),), float("nan"), dtype=A.val.dtype, device="cuda")
    o = TspgCsrOut()
    o.nrows, o.ncols = A.nrows, B.ncols
    o.rowptr, o.rowptr_bits, o.val_bits = rp.data_ptr(), 64, A.val_bits
    o.col, o.val, o.capacity = col.data_ptr(), val.data_ptr(), nnz
    a, b = A.abi(), B.abi()
    check(lib.tspg_spgemm(ctx.h, torch.cuda.current_stream().cuda_stream, C.byref(a), C.byref(b), C.byref(o),
                          flags), "tspg_spgemm")
    return DeviceCSR(A.nrows, B.ncols, rp, col, val, nnz=nnz)
