"""Serving loop: the arrival stream (CPU), and on the GPU that a scene's
results are the same alone and inside a batched pass, that admission evicts
least-recently-used idle scenes and never exceeds the budget, that the
time-step update is reproducible, and that both serving modes finish a short
stream."""
import numpy as np
import pytest
import torch

from collide_b200 import scenes as S
from collide_b200 import serving as SV


def test_poisson_stream_rate_and_mix():
    st = SV.poisson_stream(rate=2000.0, duration=2.0, resident=100, pool=10, update_frac=0.7, seed=3)
    n = len(st.queries)
    assert abs(n - 4000) < 4 * np.sqrt(4000)
    arr = np.array([q.arrival for q in st.queries])
    assert np.all(np.diff(arr) >= 0) and arr[-1] < 2.0
    frac = np.mean([q.kind == "update" for q in st.queries])
    assert abs(frac - 0.7) < 0.05
    assert all(0 <= q.scene < (100 if q.kind == "update" else 10) for q in st.queries)


def test_scene_bytes_counts_inputs_and_boxes():
    sc = S.mixed_slab(1000, seed=1)
    assert SV.scene_bytes(sc) == sc.nbytes() + 24 * 1000


def test_arena_best_fit_merges_and_never_overlaps():
    # the resident-scene arena's free list on a host buffer: random takes and
    # gives keep the ranges aligned, disjoint, merged with free neighbours,
    # and the free and taken bytes always add up to the arena
    a = SV.Arena(1 << 20, "cpu")
    rng = np.random.default_rng(0)
    live = {}
    for it in range(5000):
        if live and rng.random() < 0.5:
            k = list(live)[int(rng.integers(0, len(live)))]
            a.give(*live.pop(k))
        else:
            size = int(rng.integers(1, 60_000))
            off = a.take(size)
            if off is not None:
                assert off % 256 == 0
                for o, z in live.values():
                    assert off + SV._align(size) <= o or o + SV._align(z) <= off
                live[it] = (off, size)
        fr = a.free
        assert all(fr[i][0] + fr[i][1] < fr[i + 1][0] for i in range(len(fr) - 1))
        assert sum(z for _, z in fr) + sum(SV._align(z) for _, z in live.values()) == a.size
    for off, size in live.values():
        a.give(off, size)
    assert a.free == [(0, a.size)]
    assert a.take(a.size + 1) is None


@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix(cb):
    pool = [S.mixed_slab(n, seed=n, extent=(1.0, 1.0, 0.1)) for n in (3000, 12000, 800, 25000)]
    srv = SV.Server(pool, resident=4, max_batch=16, reserve_bytes=1 << 28)
    sids = list(srv.resident)
    srv.batch.run([srv.resident[s] for s in sids])
    b = srv.batch
    co = b.contact_offsets.astype(np.int64)
    ctx = cb.Context()
    assert b.n_contacts > 0
    for i, s in enumerate(sids):
        alone = cb.DevicePipeline(srv.resident[s], ctx=ctx)
        P, C = alone.run()
        assert int(b.scene_pairs[i]) == P and co[i + 1] - co[i] == C
        sl = slice(co[i], co[i + 1])
        assert torch.equal(b.norm[sl], alone.norm[:C]) and torch.equal(b.depth[sl], alone.depth[:C])
        assert torch.equal(b.cpta[sl], alone.cpta[:C]) and torch.equal(b.cptb[sl], alone.cptb[:C])


@pytest.mark.gpu
def test_admission_evicts_lru_within_budget(cb):
    pool = [S.mixed_slab(1000, seed=i) for i in range(6)]
    one = SV.scene_bytes(pool[0])
    srv = SV.Server(pool, resident=3, budget_bytes=3.5 * one, reserve_bytes=0)
    assert srv.initial == 3 and srv.bytes <= srv.budget
    first = list(srv.resident)[0]
    srv.resident.move_to_end(first)  # used recently: the second-oldest goes first
    second = list(srv.resident)[0]
    sid = srv.admit(srv.pool[4])
    assert sid is not None and second not in srv.resident and first in srv.resident
    assert srv.bytes <= srv.budget
    big = SV.PinnedScene(S.mixed_slab(5000, seed=9))
    assert srv.admit(big) is None and srv.rejected == 1


@pytest.mark.gpu
def test_time_step_update_is_reproducible_and_small(cb):
    sc = S.mixed_slab(20000, seed=4)
    ctx = cb.Context()
    a, b = cb.DeviceScene(sc), cb.DeviceScene(sc)
    SV.perturb_(ctx, a, 123)
    SV.perturb_(ctx, b, 123)
    torch.cuda.synchronize()
    assert torch.equal(a.pos, b.pos) and torch.equal(a.rot, b.rot)
    d = (a.pos.cpu().numpy() - sc.pos).ravel()
    assert abs(d.std() - 1e-4) < 5e-6 and abs(d.mean()) < 5e-6
    q = a.rot.cpu().numpy().astype(np.float64)
    assert np.allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-6)
    # rotation angle of q * conj(q0), from its vector part (well conditioned near 0)
    q0 = sc.rot.astype(np.float64)
    w0, v0 = q0[:, :1], -q0[:, 1:]
    w1, v1 = q[:, :1], q[:, 1:]
    v = w1 * v0 + w0 * v1 + np.cross(v1, v0)
    w = w1 * w0 - np.sum(v1 * v0, axis=1, keepdims=True)
    ang = 2 * np.arctan2(np.linalg.norm(v, axis=1), np.abs(w[:, 0]))
    assert ang.max() <= 1.0e-3 + 1e-6 and ang.mean() > 3e-4


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_serve_short_stream(cb, mode):
    pool = [S.mixed_slab(n, seed=n, extent=(2.0, 2.0, 0.2)) for n in (2000, 5000, 9000, 3000)]
    srv = SV.Server(pool, resident=8, max_batch=32, reserve_bytes=1 << 28)
    st = SV.poisson_stream(rate=400.0, duration=0.25, resident=8, pool=4, seed=1)
    r = srv.serve(st, mode=mode)
    assert r["queries"] == len(st.queries) > 20
    assert all(np.isfinite(q.done) and q.done >= q.arrival for q in st.queries)
    assert r["p99_ms"] >= r["p50_ms"] > 0


@pytest.mark.gpu
def test_batched_updates_equal_one_at_a_time(cb):
    # cc_perturb_scenes (one launch per round of distinct scenes) moves every
    # body exactly as cc_perturb_bodies per update, in order, including a
    # scene updated twice in one list
    scenes = [S.mixed_slab(n, seed=n, extent=(1.0, 1.0, 0.1)) for n in (3000, 12000, 1, 25000)]
    a = [cb.DeviceScene(s) for s in scenes]
    b = [cb.DeviceScene(s) for s in scenes]
    ctx = cb.Context()
    plan = [(0, 11), (1, 12), (3, 13), (1, 14), (2, 15), (1, 16)]
    for k, seed in plan:
        SV.perturb_(ctx, a[k], seed)
    SV.perturb_many(ctx, [(b[k], seed) for k, seed in plan])
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x.pos.view(torch.int32), y.pos.view(torch.int32))
        assert torch.equal(x.rot.view(torch.int32), y.rot.view(torch.int32))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_live_stream_results_equal_solo_calls(cb, mode):
    # queries recorded DURING a Poisson stream (new scenes admitted, updates
    # moving resident scenes, passes overlapping the next admissions): each
    # recorded result equals a solo cc_collide on the same post-update scene
    pool = [S.mixed_slab(n, seed=n, extent=(1.0, 1.0, 0.1)) for n in (3000, 12000, 800, 25000, 6000)]
    srv = SV.Server(pool, resident=6, max_batch=32, reserve_bytes=1 << 28)
    st = SV.poisson_stream(rate=600.0, duration=0.3, resident=6, pool=5, seed=4)
    for q in st.queries[::5]:
        q.record = True
    r = srv.serve(st, mode=mode)
    assert r["queries"] == len(st.queries)
    rec = [q for q in st.queries if q.record and q.result is not None]
    assert len(rec) >= 10 and {q.kind for q in rec} == {"update", "new"}
    ctx = cb.Context()
    for q in rec:
        res = q.result
        ds = cb.DeviceScene.__new__(cb.DeviceScene)
        for k, t in res["scene"].items():
            setattr(ds, k, t)
        ds.n, ds.nb = int(ds.T.shape[0]), int(ds.pos.shape[0])
        solo = cb.collide(ds, grid=srv.grid, ctx=ctx)
        assert solo["n_pairs"] == res["n_pairs"] and solo["n_contacts"] == res["n_contacts"]
        assert torch.equal(solo["contact_pairs"], res["contact_pairs"])
        for k in ("norm", "depth", "cpta", "cptb"):
            assert torch.equal(solo[k].view(torch.int32), res[k].view(torch.int32)), k
