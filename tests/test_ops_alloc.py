"""The Python binding's output allocator hook (no GPU: CPU tensors).

A failed allocation must come back to the library as NULL (which it reports
as TSPG_ENOMEM): an exception raised inside a ctypes callback is only
printed, and the C caller then receives an undefined pointer.  The hook must
also not keep its outputs alive through a reference cycle once the call's
result is dropped."""
import weakref

from trident_b200.ops import _TorchAlloc


def _call(alloc, nbytes):
    # through the C thunk, as the library calls it
    return alloc.cb(None, nbytes, None)


def test_alloc_returns_pointer_and_keeps_tensor():
    a = _TorchAlloc("cpu")
    p = _call(a, 1000)
    assert p is not None and len(a.tensors) == 1
    assert a.tensors[0].numel() >= 1000 and a.tensors[0].data_ptr() == p


def test_alloc_failure_returns_null_without_raising(capsys):
    a = _TorchAlloc("cpu")
    assert _call(a, 1 << 62) is None
    assert a.tensors == []
    assert "Exception ignored" not in capsys.readouterr().err


def test_alloc_freed_without_cycle_collection():
    a = _TorchAlloc("cpu")
    _call(a, 64)
    t = weakref.ref(a.tensors[0])
    r = weakref.ref(a)
    del a
    assert r() is None and t() is None
