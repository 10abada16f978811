"""The allocation-free broadphase entry point (cc_broadphase_noalloc).

Who needs it: callers that must not allocate device memory while they run —
code executing under CUDA stream capture (cudaMalloc is illegal there), hard
real-time simulation loops (cudaMalloc/cudaFree can synchronize the device and
stall for an unbounded time) and frameworks that own all device memory in
their own pool. The entry point takes its scratch from a fixed 16 MiB device
array instead, so its results must equal those of the context-based
cc_broadphase, call after call, even though every call reuses (and must first
clear) the same scratch.

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
