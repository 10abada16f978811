"""GPU narrowphase against the FP64 MPR oracle (the reference's
CollideAndFindPoint restated in double) and the pipeline entry points.

Errors are measured on the pairs both report as contacts: unit-normal
difference, depth difference in units of the scene's largest shape size,
contact-point difference relative to the point's magnitude (the outputs are
float32 world coordinates).

* exact mode (default): the contact set must be identical and every error at
  float32 output rounding (EXACT_TOL).
* fp64 / mixed modes: max and p99 bounds measured on B200 at the 1M scene,
  with margin (FAST_BOUNDS)."""
import numpy as np
import pytest
import torch

import oracle as O
from _helpers import contact_errors, gold, scene_of
from collide_b200 import scenes as S

pytestmark = pytest.mark.gpu

EXACT_TOL = dict(normal=1e-6, depth=1e-6, point=1e-6)
FAST_BOUNDS = {  # (max, p99)
    "fp64": dict(normal=(2e-2, 5e-5), depth=(5e-3, 5e-6), point=(1e-5, 1e-6)),
    "mixed": dict(normal=(5e-2, 2e-3), depth=(5e-3, 2e-4), point=(1e-4, 1e-6)),
}


def run_np(cb, scene, pairs, envelope=0.0, precision="exact"):
    ds = cb.DeviceScene(scene)
    pk = torch.from_numpy(np.ascontiguousarray(pairs, np.int64)).cuda()
    ctx = cb.Context()
    ctx.set_narrowphase_precision(precision)
    npc = cb.Narrowphase(ctx)
    npc.SetCollisionEnvelope(envelope)
    norm, ca, cb_, d, ids, k = npc.DoNarrowphase(ds.T, ds.A, ds.B, ds.C, ds.R, ds.ID, ds.active, ds.pos, ds.rot, pk)
    return dict(norm=norm.cpu().numpy(), cpta=ca.cpu().numpy(), cptb=cb_.cpu().numpy(), depth=d.cpu().numpy(),
                bids=ids.cpu().numpy(), n=k, pairs=pk.cpu().numpy(), contact_pairs=pk[:k].cpu().numpy())


def check_exact(err):
    assert err["n_common"] > 0
    assert len(err["only_gpu"]) == 0 and len(err["only_ref"]) == 0, (err["only_gpu"], err["only_ref"])
    for k, tol in EXACT_TOL.items():
        assert err[k].max() <= tol, (k, err[k].max())


def scale_of(scene):
    return float(np.max(scene.B))


@pytest.mark.parametrize("name", ["spheres", "mixed"])
def test_narrowphase_vs_fp64_golden(cb, name):
    g = gold(name)
    s = scene_of(g)
    r = run_np(cb, s, g["pairs"])
    ref = dict(n=len(g["np_f64_depth"]), pairs=g["np_f64_pairs"], norm=g["np_f64_norm"], depth=g["np_f64_depth"],
               cpta=g["np_f64_cpta"], cptb=g["np_f64_cptb"])
    check_exact(contact_errors(r, ref, scale_of(s)))


@pytest.fixture(scope="module")
def scene_1m():
    m = S.mixed_slab(1 << 20, seed=0)
    _, p = O.broadphase(O.aabb(m), (200, 200, 10))
    return m, p, O.narrowphase(m, p, 0.0, "f64")


def test_narrowphase_1m_exact_equals_fp64_oracle(cb, scene_1m):
    m, p, ref = scene_1m
    check_exact(contact_errors(run_np(cb, m, p), ref, scale_of(m)))


def test_narrowphase_more_pairs_than_lanes_exact(cb):
    """66,705 pairs, more than the exact kernel's resident lanes (~38K on
    B200): early lanes finish their pairs in place and take more from the
    queue, later ones park their finished refinements until the warp is done.
    Both ways must give the oracle's contacts."""
    m = S.mixed_slab(1 << 18, seed=3, extent=(1.6, 1.6, 0.5))
    _, p = O.broadphase(O.aabb(m), (80, 80, 25))
    assert len(p) > 60_000
    check_exact(contact_errors(run_np(cb, m, p), O.narrowphase(m, p, 0.0, "f64"), scale_of(m)))


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_narrowphase_1m_fast_modes_within_bounds(cb, scene_1m, mode):
    m, p, ref = scene_1m
    err = contact_errors(run_np(cb, m, p, precision=mode), ref, scale_of(m))
    assert err["n_common"] >= 0.999 * ref["n"]
    for k, (mx, p99) in FAST_BOUNDS[mode].items():
        assert err[k].max() <= mx and np.quantile(err[k], 0.99) <= p99, (k, err[k].max(), np.quantile(err[k], .99))


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
