"""trident_b200 — B200-native (sm_100a) on-node SpGEMM path for Trident.

The compute lives in ``libtspg.so`` (hand-written CUDA, C ABI in
include/tspg.h).  This package is the Python host binding used by the tests
and the benchmark; C++ hosts bind the ABI directly (include/tspg_trident.hpp).
"""
from ._lib import LIB_PATH, TspgError, lib  # noqa: F401  (raises if the library is missing)
from .csr import DeviceCSR, HostCSR  # noqa: F401

__all__ = ["lib", "LIB_PATH", "TspgError", "DeviceCSR", "HostCSR"]
