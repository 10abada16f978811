"""Host steps with static shapes (cc_set_static_shapes): the shape arrays are
copied once and reused while the body poses change from step to step. Every
step must equal a host step that copies everything, on the blocking and on the
pipelined path; re-enabling after an in-place shape change picks the change
up, and without it the kept copy is really what the step used."""
import numpy as np
import pytest

from collide_b200 import scenes as S

pytestmark = pytest.mark.gpu


def snapshot(hs):
    k, P = hs.n_contacts, hs.n_pairs
    return (P, k, hs.pairs[:P].numpy().copy(), hs.norm[:k].numpy().copy(), hs.depth[:k].numpy().copy(),
            hs.cpta[:k].numpy().copy(), hs.bids[:k].numpy().copy())


def same(a, b):
    return a[0] == b[0] and a[1] == b[1] and all(np.array_equal(x.view(np.uint8), y.view(np.uint8))
                                                  for x, y in zip(a[2:], b[2:]))


def reference(cb, hs):
    """The same host arrays through a session that copies every array."""
    ref = cb.HostSession(_scene_of(hs), ctx=cb.Context())
    ref.run()
    return snapshot(ref)


def _scene_of(hs):
    T, A, B, C, R, ID, pos, rot, act = (t.numpy() for t in hs.inputs)
    return S.Scene(T=T.copy(), A=A.copy(), B=B.copy(), C=C.copy(), R=R.copy(), ID=ID.view(np.uint32).copy(),
                   pos=pos.copy(), rot=rot.copy(), active=act.copy(), name="static_shapes_step")


def move(hs, rng, sigma=2e-4):
    pos = hs.inputs[6].numpy()
    pos += rng.normal(0.0, sigma, size=pos.shape).astype(np.float32)


def test_static_shapes_blocking_steps_equal_full_copies(cb):
    rng = np.random.default_rng(3)
    m = S.mixed_slab(80_000, seed=11, extent=(1.5, 1.5, 0.15))
    ctx = cb.Context()
    ctx.set_static_shapes(True)
    hs = cb.HostSession(m, ctx=ctx)
    for step in range(4):
        hs.run()
        got = snapshot(hs)
        assert got[1] > 50
        assert same(got, reference(cb, hs)), step
        move(hs, rng)


def test_static_shapes_pipelined_steps_equal_full_copies(cb):
    rng = np.random.default_rng(4)
    m = S.mixed_slab(80_000, seed=12, extent=(1.5, 1.5, 0.15))
    ctx = cb.Context()
    ctx.set_static_shapes(True)
    hs = cb.HostSession(m, ctx=ctx)
    for step in range(5):  # both slots of the pipeline, each reusing its copy
        hs.submit()
        hs.wait()
        assert same(snapshot(hs), reference(cb, hs)), step
        move(hs, rng)


def test_static_shapes_in_place_change(cb):
    m = S.mixed_slab(60_000, seed=13, extent=(1.2, 1.2, 0.12))
    ctx = cb.Context()
    ctx.set_static_shapes(True)
    hs = cb.HostSession(m, ctx=ctx)
    hs.run()
    before = snapshot(hs)
    hs.inputs[2].numpy()[:] *= 1.5  # grow every shape (B: half extents / radii) in place
    hs.run()  # the kept copy: the step still sees the old shapes
    assert same(snapshot(hs), before)
    ctx.set_static_shapes(True)  # drops the kept copy
    hs.run()
    after = snapshot(hs)
    assert after[0] > before[0]
    assert same(after, reference(cb, hs))
