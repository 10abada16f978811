"""cc_collide replayed as a CUDA graph gives the same results as plain stream
launches, including when the scene's data changes between replays (same
buffers) and when a size change forces a new capture."""
import numpy as np
import pytest
import torch

from collide_b200 import scenes as S

pytestmark = pytest.mark.gpu


def steps(cb, scene, graph, k=5):
    ds = cb.DeviceScene(scene)
    ctx = cb.Context()
    ctx.set_graph_replay(graph)
    pipe = cb.DevicePipeline(ds, ctx=ctx)
    g = torch.Generator(device="cuda").manual_seed(7)
    out = []
    for _ in range(k):
        pipe.run()
        P, C = pipe.n_pairs, pipe.n_contacts
        out.append(dict(P=P, C=C, pairs=pipe.pairs[:P].cpu().numpy(), norm=pipe.norm[:C].cpu().numpy(),
                        depth=pipe.depth[:C].cpu().numpy(), aabb=pipe.aabb.cpu().numpy()))
        # move every body a little, in place (the captured graph reads the same buffers)
        ds.pos.add_(torch.randn(ds.pos.shape, generator=g, device="cuda") * 2e-3)
    return out, ctx.launches()


def test_graph_replay_equals_stream_launches(cb):
    m = S.mixed_slab(100_000, seed=3, extent=(2.0, 2.0, 0.2))
    plain, _ = steps(cb, m, False)
    graph, _ = steps(cb, m, True)
    assert len({o["P"] for o in plain}) > 1  # the scene really changed between steps
    for a, b in zip(plain, graph):
        assert a["P"] == b["P"] and a["C"] == b["C"]
        assert np.array_equal(a["pairs"], b["pairs"])
        assert np.array_equal(a["aabb"].view(np.uint32), b["aabb"].view(np.uint32))
        assert np.array_equal(a["norm"].view(np.uint32), b["norm"].view(np.uint32))
        assert np.array_equal(a["depth"].view(np.uint32), b["depth"].view(np.uint32))


def test_graph_recaptures_on_size_change(cb):
    ctx = cb.Context()
    for n in (20_000, 30_000, 20_000):
        m = S.mixed_slab(n, seed=n, extent=(1.0, 1.0, 0.1))
        ds = cb.DeviceScene(m)
        pipe = cb.DevicePipeline(ds, ctx=ctx)
        ref = cb.collide(cb.DeviceScene(m), grid=(16, 16, 16))
        for _ in range(3):  # stream launches, capture, replay
            pipe.run()
            assert pipe.n_pairs == ref["n_pairs"] and pipe.n_contacts == ref["n_contacts"]
            assert torch.equal(pipe.pairs[: pipe.n_pairs], ref["pairs"])
            assert torch.equal(pipe.norm[: pipe.n_contacts], ref["norm"])


@pytest.mark.parametrize("n,extent", [(100_000, (1.0, 1.0, 0.1)), (300_000, (4.0, 4.0, 0.3))])
def test_overlapped_narrowphase_equals_in_order(cb, n, extent):
    # the MPR on the unsorted pairs (second stream) joined through the contact
    # hash gives the in-order path's output bit for bit: on the first call the
    # hash is sized for no previous pairs, so a scene with thousands of
    # contacts overflows it and is redone in order; later calls replay graphs
    m = S.mixed_slab(n, seed=n, extent=extent)
    ref_ctx, ov_ctx = cb.Context(), cb.Context()
    ref_ctx.set_narrowphase_overlap(False)
    ov_ctx.set_narrowphase_overlap(True)
    a = cb.DevicePipeline(cb.DeviceScene(m), ctx=ref_ctx)
    b = cb.DevicePipeline(cb.DeviceScene(m), ctx=ov_ctx)
    for step in range(4):
        P, C = a.run()
        assert b.run() == (P, C) and C > 0
        assert torch.equal(a.pairs[:P], b.pairs[:P]), step
        for k in ("norm", "cpta", "cptb", "depth"):
            assert torch.equal(getattr(a, k)[:C].view(torch.int32), getattr(b, k)[:C].view(torch.int32)), (step, k)
        assert torch.equal(a.bids[:C], b.bids[:C])
        assert torch.equal(a.aabb.view(torch.int32), b.aabb.view(torch.int32))


def test_stage_and_span_profiling_leave_results_unchanged(cb):
    # per-stage events, span events (in-order narrowphase) and no events give
    # the same step; spans report exactly the broadphase and narrowphase
    m = S.mixed_slab(100_000, seed=4, extent=(1.0, 1.0, 0.1))
    ref = cb.collide(cb.DeviceScene(m), grid=(16, 16, 16))
    for mode in ("stages", "spans"):
        ctx = cb.Context()
        ctx.set_narrowphase_overlap(False)
        pipe = cb.DevicePipeline(cb.DeviceScene(m), ctx=ctx)
        ctx.set_profiling(True, spans=mode == "spans")
        ctx.reset_stage_times()
        for _ in range(3):
            pipe.run()
            assert torch.equal(pipe.pairs[: pipe.n_pairs], ref["pairs"])
            assert torch.equal(pipe.norm[: pipe.n_contacts], ref["norm"])
        t = ctx.stage_times()
        if mode == "spans":
            assert set(t) == {"broadphase_span", "narrowphase_span"}
        else:
            assert {"count", "pair_test", "mpr"} <= set(t) and "broadphase_span" not in t
        assert all(n >= 3 and ms > 0 for ms, n in t.values()), t  # the first call may redo stages after sizing
        ctx.set_profiling(False)
