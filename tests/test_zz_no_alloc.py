"""The allocation-free broadphase entry point (cc_broadphase_noalloc).

Who needs it: callers that cannot allocate device memory while they run. A
hard real-time simulation loop cannot afford cudaMalloc/cudaFree, which may
synchronize the whole device and stall for an unbounded time; a framework
that hands out all device memory from its own pool cannot let a library
allocate behind its back. The entry point takes its scratch from one fixed
16 MiB device array instead, so its results must equal those of the
context-based cc_broadphase and of the oracle, call after call, even though
every call reuses (and must first clear) the same scratch.

This file sorts last on purpose (test_zz_*): if it fails, a run that stops at
the first failure has already run everything else. It passes alone in a fresh
process and after the other tests.
"""
import ctypes

import numpy as np
import pytest
import torch

from collide_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _aabbs(seed, n):
    if seed % 2:
        return S.sphere_aabbs(S.spheres_uniform(n, seed=seed, rmin=0.004, rmax=0.015))
    from oracle import aabb as oracle_aabb  # the AABB stage is not under test here
    return oracle_aabb(S.mixed_slab(n, seed=seed, extent=(1.0, 1.0, 0.1)))


def _noalloc(lib, a, grid):
    t = torch.from_numpy(a.copy()).cuda()
    n = a.shape[0] // 2
    out = torch.empty(4 * n + 16, dtype=torch.int64, device="cuda")
    np_ = ctypes.c_uint64()
    st = lib.cc_broadphase_noalloc(n, ctypes.c_void_p(t.data_ptr()), *grid, ctypes.c_void_p(out.data_ptr()),
                                   out.numel(), ctypes.byref(np_), None)
    torch.cuda.synchronize()
    return st, t.cpu().numpy(), out[: np_.value].cpu().numpy()


def _with_context(cb, a, grid):
    t = torch.from_numpy(a.copy()).cuda()
    bp = cb.Broadphase(cb.Context())
    bp.setBinsPerAxis(grid)
    p = bp.detectPossibleCollisions(t)
    torch.cuda.synchronize()
    return t.cpu().numpy(), p.cpu().numpy()


def test_noalloc_matches_context_entry_point_on_consecutive_calls(cb):
    lib = cb._lib.lib
    # two calls in a row on different scenes: the second must not see the first's scratch
    for seed, n, grid in ((1, 20000, (16, 16, 16)), (2, 50000, (8, 8, 4)), (3, 65536, (16, 16, 16))):
        a = _aabbs(seed, n)
        st, sh, p = _noalloc(lib, a, grid)
        assert st == 0, cb._lib.STATUS.get(st, st)
        sh_ref, p_ref = _with_context(cb, a, grid)
        assert np.array_equal(sh.view(np.uint32), sh_ref.view(np.uint32))  # same in-place shift
        assert len(p_ref) > 0 and np.array_equal(p, p_ref)                # bit-identical pair list


def test_noalloc_rejects_inputs_beyond_its_limit(cb):
    lib = cb._lib.lib
    n = 65536 + 1
    t = torch.zeros((2 * n, 3), dtype=torch.float32, device="cuda")
    out = torch.empty(16, dtype=torch.int64, device="cuda")
    np_ = ctypes.c_uint64()
    st = lib.cc_broadphase_noalloc(n, ctypes.c_void_p(t.data_ptr()), 16, 16, 16, ctypes.c_void_p(out.data_ptr()),
                                   16, ctypes.byref(np_), None)
    assert st == 3  # CC_ERR_CAPACITY
    # a pair buffer smaller than the pair count is refused too, with the count reported
    a = _aabbs(1, 20000)
    t = torch.from_numpy(a).cuda()
    st = lib.cc_broadphase_noalloc(20000, ctypes.c_void_p(t.data_ptr()), 16, 16, 16,
                                   ctypes.c_void_p(out.data_ptr()), 1, ctypes.byref(np_), None)
    assert st == 3 and np_.value > 1


def test_noalloc_equals_the_oracle_at_its_body_limit(cb):
    # parity with the reference's algorithm directly, not only through the
    # context path: 65,536 bodies (CC_NOALLOC_MAX_BODIES), two calls in a row
    import oracle as O
    lib = cb._lib.lib
    for seed in (5, 6):
        a = _aabbs(seed, 65536)
        st, sh, p = _noalloc(lib, a, (16, 16, 16))
        assert st == 0, cb._lib.STATUS.get(st, st)
        sh_ref, p_ref = O.broadphase(a, (16, 16, 16))
        assert np.array_equal(sh.view(np.uint32), sh_ref.view(np.uint32))
        assert len(p_ref) > 0 and np.array_equal(p, p_ref)


def _boxes(lo, hi):
    return np.ascontiguousarray(np.concatenate([lo, hi]).astype(np.float32))


def test_noalloc_device_side_limits_then_a_normal_call(cb):
    # the two limits only the device can see (search-grid entries, pair count)
    # return CC_ERR_CAPACITY; the call right after each still gives the
    # correct result from the same scratch
    import oracle as O
    lib = cb._lib.lib
    good = _aabbs(1, 30000)
    _, p_good = O.broadphase(good, (16, 16, 16))

    # 1,000 coincident boxes: 499,500 pairs > CC_NOALLOC_MAX_PAIRS (262,144)
    lo = np.full((1000, 3), 0.5, np.float32)
    dense = _boxes(lo, lo + 0.01)
    np_ = ctypes.c_uint64()
    t = torch.from_numpy(dense.copy()).cuda()
    out = torch.empty(16, dtype=torch.int64, device="cuda")
    st = lib.cc_broadphase_noalloc(1000, ctypes.c_void_p(t.data_ptr()), 16, 16, 16,
                                   ctypes.c_void_p(out.data_ptr()), 16, ctypes.byref(np_), None)
    torch.cuda.synchronize()
    assert st == 3 and np_.value == 1000 * 999 // 2  # CC_ERR_CAPACITY with the count
    st, _, p = _noalloc(lib, good, (16, 16, 16))
    assert st == 0 and np.array_equal(p, p_good)

    # 65,516 small boxes and 20 that span the scene: each of the 20 enters
    # every search cell, > CC_NOALLOC_MAX_ENTRIES (262,144) entries
    rng = np.random.default_rng(7)
    lo = rng.uniform(0.0, 1.0, (65536, 3)).astype(np.float32)
    hi = lo + np.float32(0.01)
    lo[:20], hi[:20] = 0.0, 1.01
    wide = _boxes(lo, hi)
    st, _, _ = _noalloc(lib, wide, (16, 16, 16))
    assert st == 3
    st, _, p = _noalloc(lib, good, (16, 16, 16))
    assert st == 0 and np.array_equal(p, p_good)
