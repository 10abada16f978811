"""Batched scenes (cc_collide_batch) against separate cc_collide calls and the
oracle: every scene's shifted boxes, pair list and contacts must be the ones
a call on that scene alone gives, bit for bit."""
import numpy as np
import pytest
import torch

import oracle as O
from _helpers import gold, scene_of
from collide_b200 import scenes as S

pytestmark = pytest.mark.gpu


def empty_scene():
    z = lambda *s: np.zeros(s, np.float32)  # noqa: E731
    return S.Scene(T=np.zeros(0, np.int32), A=z(0, 3), B=z(0, 3), C=z(0, 3), R=z(0, 4), ID=np.zeros(0, np.uint32),
                   pos=z(0, 3), rot=z(0, 4), active=np.zeros(0, np.uint8))


def local_keys(keys, off):
    a, b = keys >> 32, keys & 0xFFFFFFFF
    return ((a - off) << 32) | (b - off)


def check_batch(cb, scenes, grid=(16, 16, 16), precision="exact"):
    db = cb.DeviceBatch(scenes)
    ctx = cb.Context()
    ctx.set_narrowphase_precision(precision)
    out = cb.collide_batch(db, grid=grid, ctx=ctx)
    so, bo = db.shape_offsets.astype(np.int64), db.body_offsets.astype(np.int64)
    n = db.n
    aabb = out["aabb"].cpu().numpy()
    allp = torch.cat([out["pairs"]]).cpu().numpy()
    cp = out["contact_pairs"].cpu().numpy()
    norm, depth = out["norm"].cpu().numpy(), out["depth"].cpu().numpy()
    cpa, bids = out["cpta"].cpu().numpy(), out["bids"].cpu().numpy()
    coff = out["contact_offsets"].astype(np.int64)
    assert out["n_pairs"] == int(out["scene_pairs"].sum())
    for s, sc in enumerate(scenes):
        a0, a1 = so[s], so[s + 1]
        if sc.n == 0:
            assert out["scene_pairs"][s] == 0 and coff[s + 1] == coff[s]
            continue
        ref = cb.collide(cb.DeviceScene(sc), grid=grid, ctx=ctx)
        ra = ref["aabb"].cpu().numpy()
        assert np.array_equal(aabb[a0:a1].view(np.uint32), ra[: sc.n].view(np.uint32)), s
        assert np.array_equal(aabb[n + a0:n + a1].view(np.uint32), ra[sc.n:].view(np.uint32)), s
        mine = allp[((allp >> 32) >= a0) & ((allp >> 32) < a1)]
        assert np.array_equal(np.sort(local_keys(mine, a0)), np.sort(ref["pairs"].cpu().numpy())), s
        assert out["scene_pairs"][s] == ref["n_pairs"]
        c0, c1 = coff[s], coff[s + 1]
        assert c1 - c0 == ref["n_contacts"], s
        assert np.array_equal(local_keys(cp[c0:c1], a0), ref["contact_pairs"].cpu().numpy())
        assert np.array_equal(norm[c0:c1].view(np.uint32), ref["norm"].cpu().numpy().view(np.uint32))
        assert np.array_equal(depth[c0:c1].view(np.uint32), ref["depth"].cpu().numpy().view(np.uint32))
        assert np.array_equal(cpa[c0:c1].view(np.uint32), ref["cpta"].cpu().numpy().view(np.uint32))
        assert np.array_equal(bids[c0:c1] - bo[s], ref["bids"].cpu().numpy())
    return out


def test_batch_equals_separate_calls(cb):
    scenes = [S.mixed_slab(n, seed=10 + i, extent=(1.0, 1.0, t))
              for i, (n, t) in enumerate([(1000, 0.1), (20_000, 0.05), (3000, 0.5), (50_000, 0.2)])]
    scenes.insert(2, S.spheres_uniform(4096, seed=3, rmin=0.005, rmax=0.02))
    out = check_batch(cb, scenes)
    assert out["n_contacts"] > 1000


def test_batch_with_empty_and_single_shape_scenes(cb):
    one = S.mixed_slab(1, seed=1, extent=(1.0, 1.0, 1.0))
    scenes = [empty_scene(), S.mixed_slab(5000, seed=4, extent=(1.0, 1.0, 0.1)), empty_scene(), one,
              S.mixed_slab(2000, seed=5, extent=(0.5, 0.5, 0.05)), empty_scene()]
    check_batch(cb, scenes)


def test_batch_fast_precision_and_pinned_grid(cb):
    scenes = [S.mixed_slab(n, seed=20 + n, extent=(1.0, 1.0, 0.1)) for n in (4000, 9000, 1500)]
    check_batch(cb, scenes, grid=(8, 8, 8), precision="fp64")


def test_batch_matches_oracle_goldens(cb):
    gs, gm = gold("spheres"), gold("mixed")
    scenes = [scene_of(gm), scene_of(gs)]
    db = cb.DeviceBatch(scenes)
    out = cb.collide_batch(db, grid=(16, 16, 16))
    so = db.shape_offsets.astype(np.int64)
    allp = out["pairs"].cpu().numpy()
    for s, g in enumerate((gm, gs)):
        mine = allp[((allp >> 32) >= so[s]) & ((allp >> 32) < so[s + 1])]
        assert np.array_equal(np.sort(local_keys(mine, so[s])), g["pairs"])
    n = db.n
    a = out["aabb"].cpu().numpy()
    ns = scenes[0].n
    sh = np.concatenate([a[:ns], a[n:n + ns]])
    assert np.array_equal(sh.view(np.uint32), g_shifted(gm).view(np.uint32))


def g_shifted(g):
    return O.broadphase(O.aabb(scene_of(g)), (16, 16, 16))[0]


def test_batch_bad_local_body_id_is_rejected(cb):
    a, b = S.mixed_slab(100, seed=1), S.mixed_slab(100, seed=2)
    b.ID = b.ID.copy()
    b.ID[5] = 100  # valid globally (scene a has 100 bodies) but not inside scene b
    db = cb.DeviceBatch([a, b])
    with pytest.raises(cb.CollideError):
        cb.collide_batch(db)
