"""Narrowphase of every shape type the reference's support maps cover,
including CONE, RECT and TRIANGLEMESH (SupportFunctions.cuh:14-99), against
the FP64 MPR oracle: pairs are given directly (the reference's AABB stage
bounds no RECT/TRIANGLEMESH shape and bounds CONE as a triangle), and the
exact mode must return the oracle's contacts to float rounding."""
import numpy as np
import pytest

import oracle as O
from collide_b200 import scenes as S

from test_gpu_narrowphase import check_exact, run_np
from _helpers import contact_errors

pytestmark = pytest.mark.gpu


def all_types_scene(n=3000, seed=0, box=0.3):
    rng = np.random.Generator(np.random.PCG64(seed))
    T = rng.integers(0, 7, size=n).astype(np.int32)
    h = rng.uniform(0.01, 0.04, size=(n, 3))
    B = h.copy()
    B[T == S.SPHERE, 1:] = 0.0
    B[T == S.CYLINDER, 2] = B[T == S.CYLINDER, 0]
    B[T == S.RECT, 2] = 0.0
    A = np.zeros((n, 3))
    C = np.zeros((n, 3))
    tri = T == S.TRIANGLEMESH  # vertices in A, B, C
    A[tri] = rng.uniform(-0.04, 0.04, size=(tri.sum(), 3))
    B[tri] = rng.uniform(-0.04, 0.04, size=(tri.sum(), 3))
    C[tri] = rng.uniform(-0.04, 0.04, size=(tri.sum(), 3))
    c = rng.random((n, 3)) * box
    q = S.random_quaternions(rng, n)
    sc = S._one_shape_per_body(T, B, c, q, f"all_types_{n}")
    sc.A = A.astype(np.float32)
    sc.C = C.astype(np.float32)
    return sc


def close_pairs(sc, r=0.06):
    p = sc.pos.astype(np.float64)
    n = len(p)
    out = []
    for i in range(n):
        d = np.linalg.norm(p[i + 1:] - p[i], axis=1)
        j = np.nonzero(d < r)[0] + i + 1
        out.append((np.int64(i) << 32) | j.astype(np.int64))
    return np.concatenate(out)


@pytest.mark.parametrize("seed", [0, 1])
def test_every_shape_type_matches_fp64_oracle(cb, seed):
    sc = all_types_scene(seed=seed)
    pairs = close_pairs(sc)
    tt = sc.T[pairs >> 32] * 7 + sc.T[pairs & 0xFFFFFFFF]
    assert len(np.unique(tt)) >= 40  # nearly every (type, type) combination is present
    ref = O.narrowphase(sc, pairs, 0.0, "f64")
    got = run_np(cb, sc, pairs)
    err = contact_errors(got, ref, float(np.abs(sc.B).max()))
    assert err["n_ref"] > 500
    check_exact(err)
