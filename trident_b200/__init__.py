"""trident_b200 — B200-native (sm_100a) on-node SpGEMM path for Trident.

The compute lives in ``libtspg.so`` (hand-written CUDA, C ABI in
include/tspg.h).  This package is the Python host binding used by the tests
and the benchmark; C++ hosts bind the ABI directly (include/tspg_trident.hpp).

The device library is loaded by the first use of ``lib``, ``DeviceCSR`` or any
module that calls it (``ops``, ``summa``, ``tune``); loading raises when it is
missing — there is no CPU fallback.  ``workloads`` and ``synth`` load only the
host-only generator library, so CPU-only consumers never map the device code.
"""
from __future__ import annotations

import importlib

__all__ = ["lib", "LIB_PATH", "TspgError", "DeviceCSR", "HostCSR"]

_LAZY = {"lib": "._lib", "LIB_PATH": "._lib", "TspgError": "._lib", "DeviceCSR": ".csr",
         "HostCSR": ".synth"}


def __getattr__(name):
    mod = _LAZY.get(name)
    if mod is None:
        raise AttributeError(f"module 'trident_b200' has no attribute {name!r}")
    return getattr(importlib.import_module(mod, __name__), name)
