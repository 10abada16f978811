"""Writes tests/golden/*.npz: seeded inputs and the outputs of the
REFERENCE ITSELF (its own AABBGenerator.cu / Broadphase.cu / Narrowphase.cu
compiled in host mode by oracle/Makefile into oracle/_ref/), so the oracle
restatement and the GPU path can be checked against them without the
reference checkout.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "collision-detection_b200"))

import oracle as O  # noqa: E402
from collide_b200 import scenes as S  # noqa: E402


def scene_dict(s):
    return dict(T=s.T, A=s.A, B=s.B, C=s.C, R=s.R, ID=s.ID, pos=s.pos, rot=s.rot, active=s.active)


def all_types_scene(n=512, seed=7):
    """Every shape type, several shapes per body, local offsets and rotations."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nb = n // 2
    T = rng.integers(0, 7, size=n).astype(np.int32)
    A = rng.uniform(-0.02, 0.02, size=(n, 3))
    B = rng.uniform(0.01, 0.05, size=(n, 3))
    C = rng.uniform(-0.05, 0.05, size=(n, 3))
    R = S.random_quaternions(rng, n)
    ID = rng.integers(0, nb, size=n).astype(np.uint32)
    pos = rng.uniform(-0.5, 0.5, size=(nb, 3))
    rot = S.random_quaternions(rng, nb)
    return S.Scene(T=T, A=A.astype(np.float32), B=B.astype(np.float32), C=C.astype(np.float32),
                   R=R.astype(np.float32), ID=ID, pos=pos.astype(np.float32), rot=rot.astype(np.float32),
                   active=np.ones(nb, np.uint8), name="all_types")


def main():
    out = {}
    # 1. spheres: AABBs, bin list on the default 16^3 grid, pairs, contacts
    s = S.spheres_uniform(2048, seed=11, rmin=0.005, rmax=0.02)
    a = O.ref_aabb(s)
    b = O.ref_bins(a, (16, 16, 16))
    sh, p = O.ref_broadphase(a, (16, 16, 16))
    np32 = O.ref_narrowphase(s, p, 0.0, "f32")
    np64 = O.ref_narrowphase(s, p, 0.0, "f64")
    out["spheres"] = dict(scene_dict(s), aabb=a, shifted=sh, pairs=p, bins=b["bins"], bodies=b["bodies"],
                          active_bins=b["active"], bin_end=b["bin_end"], grid=np.array([16, 16, 16], np.int32),
                          np_f64_norm=np64["norm"], np_f64_depth=np64["depth"], np_f64_cpta=np64["cpta"],
                          np_f64_cptb=np64["cptb"], np_f64_ids=np64["ids"], np_f64_pairs=np64["pairs"],
                          np_f32_n=np.array([np32["n"]]))
    # 2. mixed convex shapes: AABBs, pairs on an 8x8x4 grid, FP64 contacts
    m = S.mixed_slab(2048, seed=12, extent=(0.3, 0.3, 0.05))
    a = O.ref_aabb(m)
    b = O.ref_bins(a, (8, 8, 4))
    sh, p = O.ref_broadphase(a, (8, 8, 4))
    np64 = O.ref_narrowphase(m, p, 0.0, "f64")
    out["mixed"] = dict(scene_dict(m), aabb=a, shifted=sh, pairs=p, bins=b["bins"], bodies=b["bodies"],
                        active_bins=b["active"], bin_end=b["bin_end"], grid=np.array([8, 8, 4], np.int32),
                        np_f64_norm=np64["norm"], np_f64_depth=np64["depth"], np_f64_cpta=np64["cpta"],
                        np_f64_cptb=np64["cptb"], np_f64_ids=np64["ids"], np_f64_pairs=np64["pairs"])
    # 3. every shape type (AABB generation incl. the type-5 triangle quirk)
    t = all_types_scene()
    init = np.full((2 * t.n, 3), 7.0, np.float32)  # skipped shapes keep these
    a = O.ref_aabb(t, init=init)
    out["all_types"] = dict(scene_dict(t), aabb_init=init, aabb=a)
    # 4. the reference's own known-answer tests (test1.cu, binTest_Broadphase.cu)
    ub = S.unit_boxes(10)
    sh, p = O.ref_broadphase(ub, (1, 1, 1))
    b = O.ref_bins(ub, (1, 1, 1))
    out["test1"] = dict(aabb=ub, shifted=sh, pairs=p, bins=b["bins"], bodies=b["bodies"], active_bins=b["active"],
                        bin_end=b["bin_end"], grid=np.array([1, 1, 1], np.int32))
    lp = S.lattice_pairs(6)
    sh, p = O.ref_broadphase(lp, (10, 10, 10))
    b = O.ref_bins(lp, (10, 10, 10))
    out["lattice"] = dict(aabb=lp, shifted=sh, pairs=p, bins=b["bins"], bodies=b["bodies"], active_bins=b["active"],
                          bin_end=b["bin_end"], grid=np.array([10, 10, 10], np.int32))
    # 5. a planar scene (all z == 0): the reference's bin scale is 0/0 on z
    rng = np.random.Generator(np.random.PCG64(5))
    c = rng.uniform(-1, 1, size=(300, 3)).astype(np.float32)
    c[:, 2] = 0
    r = rng.uniform(0.02, 0.08, size=(300, 1)).astype(np.float32)
    lo, hi = c - r, c + r
    lo[:, 2] = 0
    hi[:, 2] = 0
    pl = np.concatenate([lo, hi]).astype(np.float32)
    sh, p = O.ref_broadphase(pl, (8, 8, 8))
    b = O.ref_bins(pl, (8, 8, 8))
    out["planar"] = dict(aabb=pl, shifted=sh, pairs=p, bins=b["bins"], bodies=b["bodies"], active_bins=b["active"],
                         bin_end=b["bin_end"], grid=np.array([8, 8, 8], np.int32))
    for k, v in out.items():
        np.savez_compressed(os.path.join(HERE, f"{k}.npz"), **v)
        print(k, {kk: vv.shape for kk, vv in v.items()})


if __name__ == "__main__":
    main()
