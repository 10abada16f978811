"""Pipelined host steps (cc_collide_host_submit / cc_collide_host_wait): two
steps in flight give the same results as the blocking host entry point, a
step whose output capacity is too small is redone, and misuse is reported."""
import numpy as np
import pytest
import torch

from collide_b200 import scenes as S

pytestmark = pytest.mark.gpu


def snapshot(hs):
    k, P = hs.n_contacts, hs.n_pairs
    return (P, k, hs.pairs[:P].numpy().copy(), hs.norm[:k].numpy().copy(), hs.depth[:k].numpy().copy(),
            hs.cpta[:k].numpy().copy())


def same(a, b):
    return a[0] == b[0] and a[1] == b[1] and all(np.array_equal(x.view(np.uint8), y.view(np.uint8))
                                                  for x, y in zip(a[2:], b[2:]))


def test_pipelined_steps_equal_blocking_calls(cb):
    m = S.mixed_slab(150_000, seed=5, extent=(2.0, 2.0, 0.2))
    ref = cb.HostSession(m, ctx=cb.Context())
    ref.run()
    want = snapshot(ref)
    hs = cb.HostSession(m, ctx=cb.Context())
    got = []
    hs.submit()
    for _ in range(5):
        hs.submit()
        hs.wait()
        got.append(snapshot(hs))
    hs.wait()
    got.append(snapshot(hs))
    assert want[1] > 100
    assert all(same(g, want) for g in got)


def test_pipelined_capacity_overflow_is_redone(cb):
    m = S.mixed_slab(60_000, seed=6, extent=(0.5, 0.5, 0.05))
    ref = cb.HostSession(m, ctx=cb.Context())
    ref.run()
    want = snapshot(ref)
    hs = cb.HostSession(m, ctx=cb.Context(), pairs_cap=16)
    hs.submit()
    hs.submit()
    a = (hs.wait(), snapshot(hs))
    b = (hs.wait(), snapshot(hs))
    assert want[0] > 16 and same(a[1], want) and same(b[1], want)


def test_pipelined_misuse_is_reported(cb):
    m = S.mixed_slab(5_000, seed=7)
    hs = cb.HostSession(m, ctx=cb.Context())
    hs.submit()
    hs.submit()
    with pytest.raises(cb.CollideError):
        hs.submit()  # a third step in flight
    hs.wait()
    hs.wait()
    with pytest.raises(IndexError):
        hs.wait()  # nothing in flight (the session keeps its own queue)


def test_c_gathered_from_pinned_equals_copied_whole(cb):
    """From pinned host buffers the library reads the third shape array (C)
    only for CONE and TRIANGLEMESH shapes; the results equal those of pageable
    buffers, which are copied whole, even with NaN in every other shape's C."""
    from test_gpu_shape_types import all_types_scene
    sc = all_types_scene(n=4000, seed=3)
    C = sc.C.copy()
    C[sc.T == S.CONE] = np.random.default_rng(1).uniform(-0.04, 0.04, size=((sc.T == S.CONE).sum(), 3))
    C[(sc.T != S.CONE) & (sc.T != S.TRIANGLEMESH)] = np.nan
    sc.C = C.astype(np.float32)
    # the caller bounds RECT and TRIANGLEMESH shapes (GenerateAABB leaves them)
    n = sc.n
    init = np.zeros((2 * n, 3), np.float32)
    p = sc.pos[sc.ID].astype(np.float32)
    init[:n], init[n:] = p - 0.05, p + 0.05
    out = {}
    for pinned in (True, False):
        hs = cb.HostSession(sc, ctx=cb.Context(), want_aabb=True, pinned=pinned)
        snaps = []
        for step in range(3):
            hs.aabb.copy_(torch.from_numpy(init))
            if step < 2:
                hs.run()
            else:
                hs.submit()
                hs.wait()
            snaps.append(snapshot(hs) + (hs.aabb.numpy().copy(),))
        out[pinned] = snaps
    assert out[True][0][1] > 100  # contacts found
    for a, b in zip(out[True], out[False]):
        assert same(a, b)
    hs = cb.HostSession(sc, ctx=cb.Context(), pinned=True)
    assert hs.input_bytes() == sum(t.numel() * t.element_size() for t in hs.inputs) - 12 * (n - hs.c_shapes)
