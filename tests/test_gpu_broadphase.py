"""GPU parity of AABB generation and the broadphase against the reference
(golden vectors) and the oracle. Everything here is bit-exact: AABBs, the
in-place shift, the sorted bin list and the sorted unique pair list."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from _helpers import bits, gold, pair_set_diff, same_bits, scene_of
from collide_b200 import scenes as S

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda").to(dtype) if dtype is not None else \
        torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def gpu_aabb(cb, scene, init=None):
    ds = cb.DeviceScene(scene)
    out = None if init is None else torch.from_numpy(np.ascontiguousarray(init, np.float32)).cuda()
    a = cb.AABBGenerator().GenerateAABB(ds.T, ds.A, ds.B, ds.C, ds.R, ds.ID, ds.pos, ds.rot, out)
    return a.cpu().numpy()


def gpu_broadphase(cb, aabb, grid, ctx=None):
    t = torch.from_numpy(np.ascontiguousarray(aabb, np.float32)).cuda()
    bp = cb.Broadphase(ctx)
    bp.setBinsPerAxis(grid)
    p = bp.detectPossibleCollisions(t)
    assert bp.getNumPossibleContacts() == len(p)
    return t.cpu().numpy(), p.cpu().numpy()


def gpu_bins(cb, aabb, grid):
    t = torch.from_numpy(np.ascontiguousarray(aabb, np.float32)).cuda()
    bp = cb.Broadphase()
    bp.setBinsPerAxis(grid)
    b = bp.bins(t)
    return {k: v.cpu().numpy().view(np.uint32) for k, v in b.items()}, t.cpu().numpy()


# ------------------------------------------------------------------ AABB
@pytest.mark.parametrize("name", ["spheres", "mixed"])
def test_aabb_bitexact_golden(cb, name):
    g = gold(name)
    assert same_bits(gpu_aabb(cb, scene_of(g)), g["aabb"])


def test_aabb_all_shape_types_golden(cb):
    g = gold("all_types")
    a = gpu_aabb(cb, scene_of(g), init=g["aabb_init"])
    assert same_bits(a, g["aabb"])


def test_aabb_bitexact_large_mixed(cb):
    m = S.mixed_slab(300_000, seed=5)
    assert same_bits(gpu_aabb(cb, m), O.aabb(m))


# ------------------------------------------------------------------ pairs + bins vs the reference's own outputs
@pytest.mark.parametrize("name", ["spheres", "mixed", "test1", "lattice", "planar"])
def test_broadphase_bitexact_golden(cb, name):
    g = gold(name)
    grid = tuple(int(v) for v in g["grid"])
    sh, p = gpu_broadphase(cb, g["aabb"], grid)
    assert same_bits(sh, g["shifted"])
    assert np.array_equal(p, g["pairs"])


@pytest.mark.parametrize("name", ["spheres", "mixed", "test1", "lattice", "planar"])
def test_bin_list_bitexact_golden(cb, name):
    g = gold(name)
    grid = tuple(int(v) for v in g["grid"])
    b, sh = gpu_bins(cb, g["aabb"], grid)
    assert same_bits(sh, g["shifted"])
    assert np.array_equal(b["bin_number"], g["bins"])
    assert np.array_equal(b["body_number"], g["bodies"])
    assert np.array_equal(b["active_bins"], g["active_bins"])
    assert np.array_equal(b["bin_end"], g["bin_end"])


# ------------------------------------------------------------------ the benchmark workloads
def test_plain_16k_spheres_default_grid(cb):
    """16,384 spheres, U[0,1]^3, r U[0.002,0.006], the reference's default 16^3."""
    s = S.spheres_uniform(16384, seed=0)
    a = O.aabb(s)
    sh, p = gpu_broadphase(cb, a, (16, 16, 16))
    sho, po = O.broadphase(a, (16, 16, 16))
    assert same_bits(sh, sho) and np.array_equal(p, po)
    b, _ = gpu_bins(cb, a, (16, 16, 16))
    bo = O.bins(a, (16, 16, 16))
    assert np.array_equal(b["bin_number"], bo["bins"]) and np.array_equal(b["body_number"], bo["bodies"])
    assert np.array_equal(b["active_bins"], bo["active"]) and np.array_equal(b["bin_end"], bo["bin_end"])


def test_full_1m_mixed_shapes(cb):
    """1,048,576 mixed shapes in the [0,10]x[0,10]x[0,0.5] slab: full-size parity."""
    m = S.mixed_slab(1 << 20, seed=0)
    a = gpu_aabb(cb, m)
    ao = O.aabb(m)
    assert same_bits(a, ao)
    sh, p = gpu_broadphase(cb, a, (16, 16, 16))
    sho, po = O.broadphase(ao, (200, 200, 10))  # pairs and the shift do not depend on the grid
    assert same_bits(sh, sho)
    assert np.array_equal(p, po)
    # size-independent properties
    assert np.all(np.diff(p) > 0)  # sorted, unique
    assert np.all((p >> 32) < (p & 0xFFFFFFFF))


@pytest.mark.parametrize("dims", [(0, 0, 0), (1, 1, 1), (7, 3, 2), (64, 64, 4), (1000, 1000, 50)])
def test_search_grid_does_not_change_pairs(cb, dims):
    m = S.mixed_slab(100_000, seed=3, extent=(2.0, 2.0, 0.2))
    a = O.aabb(m)
    _, po = O.broadphase(a, (16, 16, 16))
    ctx = cb.Context()
    ctx.set_search_grid(dims)
    _, p = gpu_broadphase(cb, a, (16, 16, 16), ctx)
    assert np.array_equal(p, po), pair_set_diff(p, po)


def test_dense_kernel_skipped_after_sparse_calls(cb):
    """A context whose last call found no dense cell launches no dense-cell
    kernel; a dense scene then is tested by the lane-per-entry kernel alone
    (same pairs) and turns the dense-cell kernel back on for the next call."""
    sparse = O.aabb(S.spheres_uniform(16384, seed=0))
    _, ps = O.broadphase(sparse, (16, 16, 16))
    dense = O.aabb(S.clustered_spheres(60_000, seed=2, clusters=2, sigma=0.01, background=0.05))
    _, pd = O.broadphase(dense, (64, 64, 64))
    ctx = cb.Context()
    launches = []
    for a, want in ((sparse, ps), (sparse, ps), (dense, pd), (dense, pd), (sparse, ps)):
        _, p = gpu_broadphase(cb, a, (16, 16, 16), ctx)
        assert np.array_equal(p, want), pair_set_diff(p, want)
        launches.append(ctx.launches())
    assert launches[1] == launches[0] - 1  # no dense cell in the first call: none launched in the second
    # the dense scene's first call skipped it but counted its dense cells, so the
    # next call runs as on a context that saw the dense scene from the start
    fresh = cb.Context()
    for _ in range(2):
        gpu_broadphase(cb, dense, (16, 16, 16), fresh)
    assert launches[3] == fresh.launches()


@pytest.mark.parametrize("target,ratio", [(1.0, 1.0), (4.0, 2.0), (32.0, 0.5), (0.25, 8.0)])
def test_tuning_does_not_change_pairs(cb, target, ratio):
    s = S.clustered_spheres(200_000, seed=1)
    a = O.aabb(s)
    _, po = O.broadphase(a, (64, 64, 64))
    ctx = cb.Context()
    ctx.set_tuning(target, ratio)
    _, p = gpu_broadphase(cb, a, (16, 16, 16), ctx)
    assert np.array_equal(p, po), pair_set_diff(p, po)


def test_dense_cells_match_oracle(cb):
    # two tight clusters: cells of the search grid hold hundreds of entries, so
    # their tests run in the tiled dense-cell kernel (the background in the
    # lane-per-entry kernel); a coarse pinned grid makes nearly every cell dense
    s = S.clustered_spheres(60_000, seed=2, clusters=2, sigma=0.01, background=0.05)
    a = O.aabb(s)
    _, po = O.broadphase(a, (64, 64, 64))
    assert len(po) > 1_000_000
    for dims in ((0, 0, 0), (20, 20, 20)):
        for dense in (0, 128, 512):  # 0: every cell in the lane-per-entry kernel
            ctx = cb.Context()
            ctx.set_search_grid(dims)
            ctx.set_dense_cell(dense)
            _, p = gpu_broadphase(cb, a, (16, 16, 16), ctx)
            assert np.array_equal(p, po), (dims, dense, pair_set_diff(p, po))


def test_tuner_picks_a_setting_and_pairs_do_not_change(cb):
    from collide_b200 import tuner
    s = S.clustered_spheres(100_000, seed=4)
    ds = cb.DeviceScene(s)
    a0 = cb.AABBGenerator().GenerateAABB(*ds.arrays())
    ctx = cb.Context()
    bp = cb.Broadphase(ctx)
    out = {}

    def run():
        a = a0.clone()
        out["p"] = bp.detectPossibleCollisions(a)

    run()
    before = out["p"].clone()
    best, table = tuner.tune(ctx, run, grid_candidates=((4.0, 2.0), (1.0, 1.0)), dense_candidates=(128, 0),
                             shape_candidates=((96, 8), (64, 16), (128, 5)))
    assert len(table) == 6 and best in [c for c, _ in table]  # (96, 8) is the default shape: timed once
    run()
    assert torch.equal(out["p"], before)
    for cand, _ in table:  # every candidate gives the same list
        tuner.apply(ctx, cand)
        run()
        assert torch.equal(out["p"], before), cand


def test_clustered_4m_sorted_unique_and_subboxes(cb):
    # 4,194,304 clustered spheres (about 2.5e8 pairs): the list is strictly
    # increasing (sorted, no duplicates) and, restricted to the bodies meeting
    # a box in a cluster core, equals the brute-force oracle there
    s = S.clustered_spheres(1 << 22, seed=0)
    ds = cb.DeviceScene(s)
    a = cb.AABBGenerator().GenerateAABB(*ds.arrays())
    p = cb.Broadphase(cb.Context()).detectPossibleCollisions(a)
    P = p.numel()
    assert P > 200_000_000
    for s0 in range(0, P - 1, 1 << 27):
        c = p[s0:min(P, s0 + (1 << 27) + 1)]
        assert bool((c[1:] > c[:-1]).all())
    an = a.cpu().numpy()
    n = s.n
    mn, mx = an[:n], an[n:]
    rng = np.random.default_rng(5)
    for _ in range(3):
        c0 = mn[rng.integers(0, n)]  # a random body's corner: 90% of them lie in a cluster
        half = 0.004
        while True:
            sel = np.nonzero(np.all(mn <= c0 + half, 1) & np.all(mx >= c0 - half, 1))[0]
            if len(sel) <= 15000:
                break
            half /= 1.3
        ref = O.pairs_bruteforce(np.concatenate([mn[sel], mx[sel]]))
        ref = (sel[ref >> 32].astype(np.int64) << 32) | sel[ref & 0xFFFFFFFF].astype(np.int64)
        mask = torch.zeros(n, dtype=torch.bool, device=p.device)
        mask[torch.from_numpy(sel).to(p.device)] = True
        got = torch.cat([c[mask[c >> 32] & mask[c & 0xFFFFFFFF]].cpu() for c in torch.split(p, 1 << 26)]).numpy()
        assert np.array_equal(got, np.sort(ref)), (len(sel), len(got), len(ref))


# ------------------------------------------------------------------ the reference's own tests
@pytest.mark.parametrize("n", [1, 2, 10, 33, 100, 4097, 6000])
def test_reference_test1_single_bin(cb, n):
    """test/test1.cu: n identical unit boxes -> n(n-1)/2 pairs. n > 4097 puts
    more than 4096 pairs on one owner (the whole-list sort path)."""
    sh, p = gpu_broadphase(cb, S.unit_boxes(n), (1, 1, 1))
    assert len(p) == n * (n - 1) // 2
    a = np.arange(n, dtype=np.int64)
    iu = np.triu_indices(n, 1)
    assert np.array_equal(p, (a[iu[0]] << 32) | a[iu[1]])


@pytest.mark.parametrize("m,bpa", [(10, 10), (20, 20), (7, 3), (5, 16)])
def test_reference_bintest_lattice(cb, m, bpa):
    """test/binTest_Broadphase.cu: duplicated lattice -> exactly m^3 pairs."""
    _, p = gpu_broadphase(cb, S.lattice_pairs(m), (bpa, bpa, bpa))
    assert len(p) == m ** 3


def test_reference_nsquared_superset(cb):
    """test/nSquared_Broadphase.cu: every true sphere overlap is a pair (N=20,000)."""
    s = S.random_spheres_cube(20000, seed=4)
    a = S.sphere_aabbs(s)
    _, p = gpu_broadphase(cb, a, (30, 30, 30))
    c = torch.from_numpy(s.pos.astype(np.float64)).cuda()
    r = torch.from_numpy(s.B[:, 0].astype(np.float64)).cuda()
    d2 = torch.cdist(c, c) ** 2
    hit = torch.triu(d2 < (r[:, None] + r[None, :]) ** 2, diagonal=1)
    ii, jj = torch.nonzero(hit, as_tuple=True)
    true_keys = ((ii.cpu().numpy().astype(np.int64) << 32) | jj.cpu().numpy())
    assert len(true_keys) > 0 and np.all(np.isin(true_keys, p))
    _, po = O.broadphase(a, (30, 30, 30))
    assert np.array_equal(p, po)


# ------------------------------------------------------------------ edge cases
def edge_cases():
    rng = np.random.default_rng(4)
    out = {}
    for lo, hi in [(-5.0, -1.0), (3.0, 9.0), (-1.0, 1.0)]:
        c = rng.uniform(lo, hi, size=(500, 3)).astype(np.float32)
        r = rng.uniform(0.05, 0.3, size=(500, 1)).astype(np.float32)
        out[f"range_{lo}_{hi}"] = np.concatenate([c - r, c + r]).astype(np.float32)
    c = rng.integers(0, 8, size=(400, 3)).astype(np.float32) * 0.125
    out["cell_boundaries"] = np.concatenate([c, c + 0.125]).astype(np.float32)
    z = np.zeros((50, 3), np.float32)
    out["coincident_points"] = np.concatenate([z, z])
    out["single_box"] = np.array([[0, 0, 0], [1, 2, 3]], np.float32)
    out["touching_faces"] = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 1], [2, 1, 1]], np.float32)
    t = np.linspace(-3, 3, 64, dtype=np.float32)
    out["line_x"] = np.concatenate([np.stack([t, 0 * t, 0 * t], 1), np.stack([t + 0.1, 0 * t, 0 * t], 1)])
    return out


@pytest.mark.parametrize("case", sorted(edge_cases()))
@pytest.mark.parametrize("grid", [(1, 1, 1), (8, 8, 8), (3, 7, 5)])
def test_edge_cases_match_oracle(cb, case, grid):
    a = edge_cases()[case]
    sh, p = gpu_broadphase(cb, a, grid)
    sho, po = O.broadphase(a, grid)
    assert same_bits(sh, sho)
    assert np.array_equal(p, po)
    b, _ = gpu_bins(cb, a, grid)
    bo = O.bins(a, grid)
    for k, ko in (("bin_number", "bins"), ("body_number", "bodies"), ("active_bins", "active"),
                  ("bin_end", "bin_end")):
        assert np.array_equal(b[k], bo[ko]), k


def test_empty_input(cb):
    sh, p = gpu_broadphase(cb, np.zeros((0, 3), np.float32), (16, 16, 16))
    assert len(p) == 0


@pytest.mark.parametrize("bad", ["nan", "inf", "inverted"])
def test_invalid_input_is_rejected_and_untouched(cb, bad):
    a = S.sphere_aabbs(S.spheres_uniform(1000, seed=1))
    if bad == "nan":
        a[17, 1] = np.nan
    elif bad == "inf":
        a[1000 + 5, 2] = np.inf
    else:
        a[3, 0] = a[1003, 0] + 1.0
    t = torch.from_numpy(a.copy()).cuda()
    with pytest.raises(cb.CollideError) as e:
        cb.Broadphase().detectPossibleCollisions(t)
    assert e.value.status == 2  # CC_ERR_INVALID_INPUT
    assert same_bits(t.cpu().numpy(), a)


def test_capacity_then_fetch(cb):
    from collide_b200 import _lib
    s = S.spheres_uniform(20000, seed=8, rmin=0.01, rmax=0.02)
    a = O.aabb(s)
    _, po = O.broadphase(a, (16, 16, 16))
    ctx = cb.Context()
    t = torch.from_numpy(a).cuda()
    small = torch.empty(10, dtype=torch.int64, device="cuda")
    n = ctypes.c_uint64()
    st = _lib.lib.cc_broadphase(ctx.h, s.n, ctypes.c_void_p(t.data_ptr()), 16, 16, 16,
                                ctypes.c_void_p(small.data_ptr()), 10, ctypes.byref(n), None)
    assert st == 3 and n.value == len(po)
    out = torch.empty(n.value, dtype=torch.int64, device="cuda")
    assert _lib.lib.cc_broadphase_fetch(ctx.h, ctypes.c_void_p(out.data_ptr()), n.value, None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), po)
    # the retained result is handed out once
    assert _lib.lib.cc_broadphase_fetch(ctx.h, ctypes.c_void_p(out.data_ptr()), n.value, None) == 7


def test_repeated_calls_are_deterministic(cb):
    m = S.mixed_slab(200_000, seed=6)
    a = O.aabb(m)
    ctx = cb.Context()
    first = None
    for _ in range(3):
        _, p = gpu_broadphase(cb, a, (16, 16, 16), ctx)
        if first is None:
            first = p
        assert np.array_equal(p, first)


def test_owner_buckets_follow_the_pair_density(cb):
    # One context, one body count, scenes of rising density: each call buckets
    # pair owners by the previous call's pairs per body, so the dense calls
    # meet buckets of hundreds to thousands of keys sorted on packed 32-bit
    # keys (warp, warp-pair and block tiers) before the bucket size adapts.
    ctx = cb.Context()
    n = 65536
    rng = np.random.default_rng(11)
    # (pairs per body 0.001 .. 7.4): with 4,096 owners per bucket after a
    # sparse call, the 0.0056 scene fills warp, warp-pair and block tiers,
    # 0.008 the block tier, and 0.0155 exceeds 16,384 keys in a bucket (the
    # whole-list sort takes over)
    for half in (0.0008, 0.0008, 0.0056, 0.0008, 0.0008, 0.008, 0.0008, 0.0008, 0.0155, 0.0008):
        lo = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
        a = np.ascontiguousarray(np.concatenate([lo, lo + np.float32(2 * half)]).astype(np.float32))
        sh, p = gpu_broadphase(cb, a, (16, 16, 16), ctx=ctx)
        sh_ref, p_ref = O.broadphase(a, (16, 16, 16))
        assert same_bits(sh, sh_ref)
        assert np.array_equal(p, p_ref), (half, len(p), len(p_ref), pair_set_diff(p, p_ref))
