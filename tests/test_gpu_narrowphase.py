"""GPU narrowphase against the FP64 MPR oracle (the reference's
CollideAndFindPoint restated in double) and the pipeline entry points.

Tolerances (written here, measured on B200): on pairs both report as
contacts, unit normals agree to NORMAL_TOL (max) / NORMAL_P99 (99th pct),
depths and contact points to DEPTH_TOL / POINT_TOL in units of the pair's
length scale (the larger shape size). Contacts reported by only one side
must be grazing (|depth| below GRAZE of the length scale)."""
import numpy as np
import pytest
import torch

import oracle as O
from _helpers import contact_errors, gold, scene_of
from collide_b200 import scenes as S

pytestmark = pytest.mark.gpu

NORMAL_TOL, NORMAL_P99 = 1e-3, 1e-5
DEPTH_TOL, POINT_TOL = 1e-3, 1e-3
DEPTH_P99, POINT_P99 = 1e-5, 1e-5
GRAZE = 1e-4


def run_np(cb, scene, pairs, envelope=0.0):
    ds = cb.DeviceScene(scene)
    pk = torch.from_numpy(np.ascontiguousarray(pairs, np.int64)).cuda()
    npc = cb.Narrowphase()
    npc.SetCollisionEnvelope(envelope)
    norm, ca, cb_, d, ids, k = npc.DoNarrowphase(ds.T, ds.A, ds.B, ds.C, ds.R, ds.ID, ds.active, ds.pos, ds.rot, pk)
    return dict(norm=norm.cpu().numpy(), cpta=ca.cpu().numpy(), cptb=cb_.cpu().numpy(), depth=d.cpu().numpy(),
                bids=ids.cpu().numpy(), n=k, pairs=pk.cpu().numpy(), contact_pairs=pk[:k].cpu().numpy())


def check_errors(err, depth_ref_only, depth_gpu_only):
    assert err["n_common"] > 0
    assert err["normal"].max() <= NORMAL_TOL, err["normal"].max()
    assert np.quantile(err["normal"], 0.99) <= NORMAL_P99
    assert err["depth"].max() <= DEPTH_TOL
    assert np.quantile(err["depth"], 0.99) <= DEPTH_P99
    assert err["point"].max() <= POINT_TOL
    assert np.quantile(err["point"], 0.99) <= POINT_P99
    assert np.all(np.abs(depth_ref_only) <= GRAZE) and np.all(np.abs(depth_gpu_only) <= GRAZE)


def scale_of(scene):
    return float(np.max(scene.B))


@pytest.mark.parametrize("name", ["spheres", "mixed"])
def test_narrowphase_vs_fp64_golden(cb, name):
    g = gold(name)
    s = scene_of(g)
    r = run_np(cb, s, g["pairs"])
    ref = dict(n=len(g["np_f64_depth"]), pairs=g["np_f64_pairs"], norm=g["np_f64_norm"], depth=g["np_f64_depth"],
               cpta=g["np_f64_cpta"], cptb=g["np_f64_cptb"])
    err = contact_errors(r, ref, scale_of(s))
    ro = np.isin(ref["pairs"][: ref["n"]], err["only_ref"])
    go = np.isin(r["contact_pairs"], err["only_gpu"])
    check_errors(err, ref["depth"][ro] / scale_of(s), r["depth"][go] / scale_of(s))


def test_narrowphase_1m_mixed_vs_fp64(cb):
    m = S.mixed_slab(1 << 20, seed=0)
    _, p = O.broadphase(O.aabb(m), (200, 200, 10))
    r = run_np(cb, m, p)
    ref = O.narrowphase(m, p, 0.0, "f64")
    err = contact_errors(r, ref, scale_of(m))
    ro = np.isin(ref["pairs"][: ref["n"]], err["only_ref"])
    go = np.isin(r["contact_pairs"], err["only_gpu"])
    check_errors(err, ref["depth"][ro] / scale_of(m), r["depth"][go] / scale_of(m))


def test_contacts_come_first_in_pair_order(cb):
    g = gold("mixed")
    s = scene_of(g)
    r = run_np(cb, s, g["pairs"])
    k = r["n"]
    hits, misses = r["pairs"][:k], r["pairs"][k:]
    assert np.all(np.diff(hits) > 0) and np.all(np.diff(misses) > 0)  # stable: input was sorted
    assert np.array_equal(np.sort(r["pairs"]), g["pairs"])
    # bids are the bodies of the pair's shapes (one shape per body here)
    assert np.array_equal(r["bids"][:, 0], hits >> 32) and np.array_equal(r["bids"][:, 1], hits & 0xFFFFFFFF)


def test_envelope_moves_points_and_depth(cb):
    g = gold("spheres")
    s = scene_of(g)
    r0 = run_np(cb, s, g["pairs"], 0.0)
    r1 = run_np(cb, s, g["pairs"], 0.001)
    assert r0["n"] == r1["n"]
    # Narrowphase.cu:412-415: p1 -= N*env, p2 += N*env, depth = N.(p2 - p1)
    assert np.allclose(r1["depth"], r0["depth"] + 0.002, atol=1e-6)
    assert np.allclose(r1["cpta"], r0["cpta"] - 0.001 * r0["norm"], atol=1e-6)


def test_inactive_and_same_body_pairs_are_skipped(cb):
    g = gold("spheres")
    s = scene_of(g)
    r_all = run_np(cb, s, g["pairs"])
    s2 = scene_of(g)
    s2.active = s2.active.copy()
    a = (r_all["contact_pairs"][0] >> 32)
    b = (r_all["contact_pairs"][0] & 0xFFFFFFFF)
    s2.active[[a, b]] = 0
    r2 = run_np(cb, s2, g["pairs"])
    assert r_all["contact_pairs"][0] not in r2["contact_pairs"]
    # one shape per body -> same-body pairs only if ID maps two shapes to one body
    s3 = scene_of(g)
    s3.ID = s3.ID.copy()
    s3.ID[b] = s3.ID[a]
    r3 = run_np(cb, s3, g["pairs"])
    assert r_all["contact_pairs"][0] not in r3["contact_pairs"]


def test_pipeline_equals_stages(cb):
    m = S.mixed_slab(200_000, seed=2, extent=(3.0, 3.0, 0.3))
    ds = cb.DeviceScene(m)
    out = cb.collide(ds, grid=(16, 16, 16))
    a = cb.AABBGenerator().GenerateAABB(*ds.arrays())
    bp = cb.Broadphase()
    p = bp.detectPossibleCollisions(a)
    assert torch.equal(a, out["aabb"])
    assert torch.equal(p, out["pairs"].sort().values)
    st = run_np(cb, m, p.cpu().numpy())
    assert out["n_contacts"] == st["n"]
    assert np.array_equal(out["contact_pairs"].cpu().numpy(), st["contact_pairs"])
    assert np.array_equal(out["norm"].cpu().numpy(), st["norm"])
    assert np.array_equal(out["depth"].cpu().numpy(), st["depth"])


def test_host_entry_point_equals_device(cb):
    m = S.mixed_slab(100_000, seed=9, extent=(2.0, 2.0, 0.2))
    h = cb.collide_host(m, grid=(16, 16, 16))
    d = cb.collide(cb.DeviceScene(m), grid=(16, 16, 16))
    assert h["n_pairs"] == d["n_pairs"] and h["n_contacts"] == d["n_contacts"]
    assert np.array_equal(h["pairs"], d["pairs"].cpu().numpy())
    assert np.array_equal(h["norm"], d["norm"].cpu().numpy())
    assert np.array_equal(h["aabb"], d["aabb"].cpu().numpy())
