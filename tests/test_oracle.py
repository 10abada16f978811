"""CPU tests: the oracle restatement (oracle/cc_oracle.c) pinned against

* golden vectors produced by the reference's own sources compiled in host mode
  (tests/golden/make_golden.py, committed .npz files),
* the reference's own known-answer tests (test/test1.cu, test/binTest_Broadphase.cu,
  test/nSquared_Broadphase.cu),
* the compiled reference itself (oracle/_ref) when it is present,
* the property that pair lists do not depend on the grid.
"""
import os

import numpy as np
import pytest

import oracle as O
from collide_b200 import scenes as S

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return dict(np.load(os.path.join(GOLD, f"{name}.npz")))


def scene_of(g):
    return S.Scene(T=g["T"], A=g["A"], B=g["B"], C=g["C"], R=g["R"], ID=g["ID"], pos=g["pos"], rot=g["rot"],
                   active=g["active"])


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("name", ["spheres", "mixed"])
def test_oracle_aabb_matches_reference_golden(name):
    g = gold(name)
    assert np.array_equal(bits(O.aabb(scene_of(g))), bits(g["aabb"]))


def test_oracle_aabb_all_shape_types_golden():
    g = gold("all_types")
    a = O.aabb(scene_of(g), init=g["aabb_init"])
    assert np.array_equal(bits(a), bits(g["aabb"]))
    # RECT (4) and TRIANGLEMESH (6) are skipped by the reference: untouched
    skipped = np.isin(g["T"], [4, 6])
    n = g["T"].shape[0]
    assert np.all(a[:n][skipped] == 7.0) and np.all(a[n:][skipped] == 7.0)


@pytest.mark.parametrize("name", ["spheres", "mixed", "test1", "lattice", "planar"])
def test_oracle_bins_and_pairs_match_reference_golden(name):
    g = gold(name)
    grid = tuple(int(v) for v in g["grid"])
    b = O.bins(g["aabb"], grid)
    assert np.array_equal(b["bins"], g["bins"])
    assert np.array_equal(b["bodies"], g["bodies"])
    assert np.array_equal(b["active"], g["active_bins"])
    assert np.array_equal(b["bin_end"], g["bin_end"])
    sh, p = O.broadphase(g["aabb"], grid)
    assert np.array_equal(bits(sh), bits(g["shifted"]))
    assert np.array_equal(p, g["pairs"])


def test_known_answer_test1():
    """test/test1.cu:9-33: n identical unit boxes in a 1x1x1 grid -> n(n-1)/2."""
    for n in (1, 2, 10, 57):
        _, p = O.broadphase(S.unit_boxes(n), (1, 1, 1))
        assert len(p) == n * (n - 1) // 2


@pytest.mark.parametrize("m,bpa", [(10, 10), (7, 3), (5, 16), (4, 1)])
def test_known_answer_bintest(m, bpa):
    """test/binTest_Broadphase.cu:13-43, 85-89: duplicated lattice -> m^3 pairs for any bins per axis."""
    _, p = O.broadphase(S.lattice_pairs(m), (bpa, bpa, bpa))
    assert len(p) == m ** 3
    assert np.all((p >> 32) + 1 == (p & 0xFFFFFFFF))


def test_known_answer_nsquared_superset():
    """test/nSquared_Broadphase.cu:99-133: every true sphere overlap (strict, double) is a pair."""
    s = S.random_spheres_cube(3000, seed=3)
    _, p = O.broadphase(S.sphere_aabbs(s), (30, 30, 30))
    c = s.pos.astype(np.float64)
    r = s.B[:, 0].astype(np.float64)
    d2 = ((c[:, None, :] - c[None, :, :]) ** 2).sum(-1)
    iu = np.triu_indices(s.n, 1)
    hit = d2[iu] < (r[iu[0]] + r[iu[1]]) ** 2
    true_keys = (iu[0][hit].astype(np.int64) << 32) | iu[1][hit]
    assert len(true_keys) > 0
    assert np.all(np.isin(true_keys, p))


def test_pairs_are_grid_invariant_and_equal_bruteforce():
    s = S.spheres_uniform(4000, seed=9, rmin=0.005, rmax=0.02)
    a = O.aabb(s)
    ref = None
    for g in [(1, 1, 1), (4, 4, 4), (16, 16, 16), (37, 5, 64), (128, 128, 128)]:
        sh, p = O.broadphase(a, g)
        if ref is None:
            ref = p
            assert np.array_equal(O.pairs_bruteforce(sh), p)
        assert np.array_equal(p, ref)


def test_oracle_narrowphase_golden():
    for name in ("spheres", "mixed"):
        g = gold(name)
        r = O.narrowphase(scene_of(g), g["pairs"], 0.0, "f64")
        assert r["n"] == len(g["np_f64_depth"])
        assert np.array_equal(r["pairs"], g["np_f64_pairs"])
        for k in ("norm", "depth", "cpta", "cptb"):
            assert np.array_equal(r[k], g["np_f64_" + k]), k
        assert np.array_equal(r["ids"], g["np_f64_ids"])


needs_ref = pytest.mark.skipif(not (O.ref_available("f32") and O.ref_available("f64")),
                               reason="oracle/_ref not built (needs the reference checkout)")


@needs_ref
def test_oracle_equals_compiled_reference_mixed():
    m = S.mixed_slab(20000, seed=21, extent=(1.0, 1.0, 0.05))
    a, ar = O.aabb(m), O.ref_aabb(m)
    assert np.array_equal(bits(a), bits(ar))
    for g in [(16, 16, 16), (20, 20, 2)]:
        sh, p = O.broadphase(a, g)
        shr, pr = O.ref_broadphase(ar, g)
        assert np.array_equal(p, pr) and np.array_equal(bits(sh), bits(shr))
        b, br = O.bins(a, g), O.ref_bins(ar, g)
        for k in ("bins", "bodies", "active", "bin_end"):
            assert np.array_equal(b[k], br[k])
    for prec in ("f32", "f64"):
        r, rr = O.narrowphase(m, p, 0.001, prec), O.ref_narrowphase(m, p, 0.001, prec)
        for k in ("norm", "cpta", "cptb", "depth", "ids", "pairs"):
            assert np.array_equal(r[k], rr[k]), (prec, k)


@needs_ref
def test_oracle_equals_compiled_reference_edge_cases():
    rng = np.random.default_rng(4)
    cases = []
    # negative minimum, positive minimum (origin quirk: fabs(min) is ADDED)
    for lo, hi in [(-5.0, -1.0), (3.0, 9.0), (-1.0, 1.0)]:
        c = rng.uniform(lo, hi, size=(500, 3)).astype(np.float32)
        r = rng.uniform(0.05, 0.3, size=(500, 1)).astype(np.float32)
        cases.append(np.concatenate([c - r, c + r]).astype(np.float32))
    # coordinates exactly on cell boundaries
    c = rng.integers(0, 8, size=(400, 3)).astype(np.float32) * 0.125
    cases.append(np.concatenate([c, c + 0.125]).astype(np.float32))
    # all coincident points
    z = np.zeros((50, 3), np.float32)
    cases.append(np.concatenate([z, z]))
    # a single box
    cases.append(np.array([[0, 0, 0], [1, 2, 3]], np.float32))
    for a in cases:
        for g in [(1, 1, 1), (8, 8, 8), (3, 7, 5)]:
            sh, p = O.broadphase(a, g)
            shr, pr = O.ref_broadphase(a, g)
            assert np.array_equal(p, pr) and np.array_equal(bits(sh), bits(shr))
            b, br = O.bins(a, g), O.ref_bins(a, g)
            for k in ("bins", "bodies", "active", "bin_end"):
                assert np.array_equal(b[k], br[k])


@needs_ref
def test_reference_thread_flags_do_not_change_pairs():
    """setParallelConfiguration (Broadphase.cu:69-90) only picks OpenMP vs sequential Thrust."""
    s = S.spheres_uniform(3000, seed=2, rmin=0.005, rmax=0.02)
    a = O.ref_aabb(s)
    _, p0 = O.ref_broadphase(a, (16, 16, 16), par=[0] * 10)
    _, p1 = O.ref_broadphase(a, (16, 16, 16), par=[1] * 10)
    assert np.array_equal(p0, p1)


def test_mpr_iteration_counts_per_class():
    """The FP64 oracle's iteration record covers every MPR call (early exits
    included) and stays within the reference's 35-iteration caps
    (Narrowphase.cu:201-205, 253)."""
    m = S.mixed_slab(20_000, seed=4, extent=(0.6, 0.6, 0.1))
    a = O.aabb(m)
    _, p = O.broadphase(a, (16, 16, 16))
    it = O.mpr_iterations(m, p)  # asserts one record per MPR call
    assert sum(v["pairs"] for v in it.values()) > 500
    assert ("sphere", "sphere") not in it  # analytic, no MPR
    for v in it.values():
        assert 0 <= v["discovery_mean"] <= v["discovery_max"] <= 35
        assert 0 <= v["refinement_mean"] <= v["refinement_max"] <= 35
