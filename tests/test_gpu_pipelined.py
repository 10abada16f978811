"""Pipelined host steps (cc_collide_host_submit / cc_collide_host_wait): two
steps in flight give the same results as the blocking host entry point, a
step whose output capacity is too small is redone, and misuse is reported."""
import numpy as np
import pytest

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
