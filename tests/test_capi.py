"""CPU tests of the drop-in boundary: libcollide_b200.so loads and exports
every entry point include/collide_b200.h declares; calls that need no GPU
behave (no compute here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "collide_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^CC_API[^;]*?\b(cc_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_reference_entry_points():
    names = declared()
    for n in ("cc_generate_aabb", "cc_broadphase", "cc_broadphase_bins", "cc_narrowphase", "cc_collide",
              "cc_collide_host", "cc_ctx_create", "cc_ctx_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from collide_b200 import _lib
    for n in declared():
        assert hasattr(_lib.lib, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"
    assert set(_lib.SIGNATURES) == set(declared())


def test_calls_without_gpu():
    from collide_b200 import _lib
    assert b"sm_100a" in _lib.lib.cc_version()
    for s in range(8):
        assert _lib.lib.cc_status_string(s)
    # a null context is rejected, not dereferenced
    assert _lib.lib.cc_set_tuning(None, 4.0, 2.0) == 1
    assert _lib.lib.cc_broadphase(None, 0, None, 1, 1, 1, None, 0, None, None) == 1


def test_ctx_create_fails_cleanly_without_device():
    import torch
    from collide_b200 import _lib
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = _lib.lib.cc_ctx_create(ctypes.byref(h), 0)
    assert st == 4 and not h.value  # CC_ERR_CUDA, no context

