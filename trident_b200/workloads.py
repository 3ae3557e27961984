"""Seeded synthetic operands of the benchmark workloads (host CSR).

The reference measures on SuiteSparse matrices that are not available here;
these generators stand in for them with the shapes and value distributions
of the five workloads:

* ``uniform_rows``  1024 x 1024, 16 distinct uniform columns + diagonal per row
* ``rmat``          R-MAT scale 20, edge factor 16, (.57, .19, .19, .05),
                    duplicates merged, self-loops kept
* ``laplacian`` / ``sa_prolongator``  27-point (26 / -1) Laplacian on 128^3 and
                    the smoothed-aggregation P from 3x3x3 aggregates, one Jacobi
                    step with omega = 2/3 (R = P^T for the Galerkin product)
* ``poisson_rows``  square random matrices with Poisson row lengths (batched
                    and served A·B requests)

Values are uniform in [-1, 1] (FP64) except the stencil operators.  Only the
host-only generator library (libtspg_synth.so) is loaded here.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from .synth import HostCSR, TspgHostCsr, check, lib


def _gen(fn, *args) -> HostCSR:
    h = TspgHostCsr()
    check(fn(*args, C.byref(h)), fn.__name__)
    return HostCSR.from_abi(h)


def uniform_rows(n: int = 1024, k: int = 16, diag: bool = True, seed: int = 1) -> HostCSR:
    return _gen(lib.tspg_gen_uniform_rows, n, k, int(diag), seed)


def rmat(scale: int = 20, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1) -> HostCSR:
    return _gen(lib.tspg_gen_rmat, scale, edge_factor, a, b, c, seed)


def laplacian(nx: int, ny: int | None = None, nz: int | None = None, pts: int = 27) -> HostCSR:
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    return _gen(lib.tspg_gen_laplacian, nx, ny, nz, pts)


def sa_prolongator(nx: int, ny: int | None = None, nz: int | None = None, pts: int = 27, agg: int = 3,
                   omega: float = 2.0 / 3.0) -> HostCSR:
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    return _gen(lib.tspg_gen_sa_prolongator, nx, ny, nz, pts, agg, omega)


def transpose(M: HostCSR) -> HostCSR:
    h = M.abi_host()
    out = TspgHostCsr()
    check(lib.tspg_host_transpose(C.byref(h), C.byref(out)), "tspg_host_transpose")
    return HostCSR.from_abi(out)


def poisson_rows(rows: int, lam: float, seed: int) -> HostCSR:
    return _gen(lib.tspg_gen_poisson_rows, rows, lam, seed)


def read_bmtx(path: str) -> HostCSR:
    return _gen(lib.tspg_read_bmtx, path.encode())


def galerkin_operands(n: int = 128, pts: int = 27, agg: int = 3, omega: float = 2.0 / 3.0):
    """(R, A, P) of the AMG Galerkin product R·A·P on an n^3 grid."""
    A = laplacian(n, pts=pts)
    P = sa_prolongator(n, pts=pts, agg=agg, omega=omega)
    R = transpose(P)
    return R, A, P


def batched_specs(count: int = 512, seed: int = 1, rows_lo: int = 1000, rows_hi: int = 200000,
                  lam_lo: float = 8.0, lam_hi: float = 32.0):
    """Sizes of the batched workload: rows log-uniform in [rows_lo, rows_hi],
    Poisson mean uniform in [lam_lo, lam_hi]; product i uses seeds
    (seed + 2i) for A_i and (seed + 2i + 1) for B_i."""
    rng = np.random.Generator(np.random.Philox(seed))
    rows = np.rint(np.exp(rng.uniform(math.log(rows_lo), math.log(rows_hi), size=count))).astype(np.int64)
    lam = rng.uniform(lam_lo, lam_hi, size=count)
    return [(int(rows[i]), float(lam[i]), seed + 2 * i, seed + 2 * i + 1) for i in range(count)]


def batched_product(spec):
    rows, lam, sa, sb = spec
    return poisson_rows(rows, lam, sa), poisson_rows(rows, lam, sb)
