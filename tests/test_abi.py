"""CPU: the C-ABI libraries load, export every symbol their headers declare,
and their host-side pieces (generators, .bmtx reader, pack layout arithmetic)
behave."""
import ctypes as C
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from trident_b200 import _lib, synth, workloads
from trident_b200._lib import TspgCsr, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def declared_symbols(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return set(re.findall(r"\b(tspg_[a-z0-9_]+)\s*\(", text))


def test_every_declared_symbol_is_exported():
    """Every C header under include/ is bound to the library that exports it."""
    headers = {"tspg.h": lib, "tspg_synth.h": synth.lib}
    assert sorted(n for n in os.listdir(os.path.join(ROOT, "include")) if n.endswith(".h")) == sorted(headers)
    for header, library in headers.items():
        syms = declared_symbols(header)
        assert len(syms) > 5, header
        missing = [s for s in sorted(syms) if not hasattr(library, s)]
        assert not missing, (header, missing)
    assert len(declared_symbols("tspg.h")) > 20


def test_generators_do_not_map_the_device_library():
    """The CPU legs of the benchmark build their operands through
    trident_b200.workloads alone: that loads libtspg_synth.so, never libtspg.so."""
    code = ("import sys; sys.path.insert(0, %r); import trident_b200.workloads as w; "
            "w.rmat(scale=8); m = open('/proc/self/maps').read(); "
            "print(int('libtspg.so' in m), int('libtspg_synth.so' in m))" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["0", "1"]


def test_abi_version_and_strerror():
    assert lib.tspg_abi_version() == 1
    assert _lib.strerror(_lib.TSPG_ENOMEM).startswith("out of memory")
    assert _lib.strerror(99) == "unknown status"


def _valid(M, sorted_rows=True):
    assert M.rowptr[0] == 0 and np.all(np.diff(M.rowptr) >= 0) and M.rowptr[-1] == M.nnz
    assert M.col.size == M.nnz and M.val.size == M.nnz
    if M.nnz:
        assert M.col.min() >= 0 and M.col.max() < M.ncols
    if sorted_rows:
        for i in range(M.nrows):
            c = M.col[M.rowptr[i]:M.rowptr[i + 1]]
            assert np.all(np.diff(c) > 0)


def test_uniform_rows_shape_and_determinism():
    A = workloads.uniform_rows(1024, 16, True, seed=1)
    _valid(A)
    cnt = np.diff(A.rowptr)
    assert set(np.unique(cnt)) <= {16, 17}
    assert all(i in A.col[A.rowptr[i]:A.rowptr[i + 1]] for i in range(0, 1024, 97))
    assert np.all(np.abs(A.val) <= 1.0)
    B = workloads.uniform_rows(1024, 16, True, seed=1)
    np.testing.assert_array_equal(A.col, B.col)
    np.testing.assert_array_equal(A.val, B.val)
    C2 = workloads.uniform_rows(1024, 16, True, seed=2)
    assert not np.array_equal(A.col, C2.col)


def test_rmat_small():
    A = workloads.rmat(scale=10, edge_factor=16, seed=1)
    _valid(A)
    assert A.nrows == 1024 and A.nnz <= 16 * 1024
    deg = np.diff(A.rowptr)
    assert deg[0] > deg.mean() * 5  # R-MAT hub at vertex 0 (a = 0.57)


def test_laplacian_and_prolongator():
    L = workloads.laplacian(6, pts=27)
    _valid(L)
    assert L.nrows == 216 and np.diff(L.rowptr).max() == 27
    dense = L.to_scipy().toarray()
    assert np.allclose(dense, dense.T) and np.allclose(np.diag(dense), 26.0)
    P = workloads.sa_prolongator(6, pts=27, agg=3)
    _valid(P)
    assert P.ncols == 8
    # rows of P sum to 1 - omega/26 * (row sum of A): (I - w D^-1 A) applied to the ones vector
    rowsum = np.asarray(P.to_scipy().sum(axis=1)).ravel()
    arow = dense.sum(axis=1)
    np.testing.assert_allclose(rowsum, 1.0 - (2.0 / 3.0) / 26.0 * arow, rtol=1e-13)
    R = workloads.transpose(P)
    _valid(R)
    np.testing.assert_allclose(R.to_scipy().toarray(), P.to_scipy().toarray().T)


def test_poisson_rows():
    A = workloads.poisson_rows(5000, 20.0, seed=3)
    _valid(A)
    assert abs(np.diff(A.rowptr).mean() - 20.0) < 0.5


def _numpy_bmtx(path):
    with open(path, "rb") as fh:
        data = fh.read()
    l1 = data.index(b"\n")
    l2 = data.index(b"\n", l1 + 1)
    ib, vb = map(int, data[:l1].split()[-2:])
    nr, nc, nz = map(int, data[l1 + 1:l2].split())
    rec = np.dtype([("r", f"<u{ib}"), ("c", f"<u{ib}"), ("v", "<f4" if vb == 4 else "<f8")])
    arr = np.frombuffer(data[l2 + 1:], dtype=rec, count=nz)
    return nr, nc, arr


@pytest.mark.parametrize("name", ["n16_full.bmtx", "n1024.bmtx"])
def test_bmtx_reader(name):
    path = os.path.join(GOLD, name)
    nr, nc, arr = _numpy_bmtx(path)
    A = workloads.read_bmtx(path)
    assert (A.nrows, A.ncols, A.nnz) == (nr, nc, arr.size)
    order = np.argsort(arr["r"], kind="stable")
    np.testing.assert_array_equal(A.col, arr["c"][order])
    np.testing.assert_array_equal(A.val, arr["v"][order].astype(np.float64))


def test_packed_layout_arithmetic():
    assert lib.tspg_packed_bytes(10, 8, 64, 32) == 10 * 12 + 9 * 4
    assert lib.tspg_packed_bytes(11, 8, 64, 64) == ((11 * 12 + 7) // 8) * 8 + 9 * 8
    v = TspgCsr()
    assert lib.tspg_unpack(C.c_void_p(4096), 8, 12, 0, 5, 64, 32, C.byref(v)) == 0
    assert v.val == 4096 and v.col == 4096 + 40 and v.rowptr == 4096 + 60
    assert lib.tspg_unpack(C.c_void_p(4096), 8, 12, 0, 5, 64, 64, C.byref(v)) == 0
    assert v.rowptr == 4096 + 64
    assert lib.tspg_unpack(C.c_void_p(4096), 8, 12, 7, 5, 64, 32, C.byref(v)) == _lib.TSPG_EINVAL


def test_null_context_is_rejected():
    a = TspgCsr()
    assert lib.tspg_spgemm(None, None, C.byref(a), C.byref(a), None, 0) == _lib.TSPG_EINVAL
    assert lib.tspg_ctx_destroy(None) == _lib.TSPG_EINVAL


def test_reference_signature_shim_compiles(tmp_path):
    """include/tspg_trident.hpp exposes the reference's own operator
    signatures (sp_mma_hybrid, cusparse_spgeam, LocalMatrix::spgemm,
    SpaCommHandler::Compress, ...): the C++ test that drives them with the
    reference's call sequence compiles and links against libtspg here (it runs
    in the GPU suite)."""
    exe = str(tmp_path / "shim")
    env = dict(os.environ)
    env.pop("CXX", None)
    cmd = ["g++", "-std=c++17", "-O0", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "test_trident_host.cpp"), "-o", exe,
           "-L", os.path.join(ROOT, "trident_b200"), "-ltspg", "-L", "/usr/local/cuda/lib64", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
