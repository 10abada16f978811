"""Seeded synthetic scenes in the reference's shape-array layout.

A scene is the argument list of the reference's ``AABBGenerator::GenerateAABB``
and ``Narrowphase::DoNarrowphase`` (src/aabb/AABBGenerator.cuh:21-30,
src/narrowphase/Narrowphase.cuh:19-34) as host numpy arrays:

==========  =========  ======================================================
field       dtype      meaning (src/aabb/AABBGenerator.cuh:53-75)
==========  =========  ======================================================
T           int32[n]   shape_type: SPHERE 0, ELLIPSOID 1, BOX 2, CYLINDER 3,
                       RECT 4, CONE 5, TRIANGLEMESH 6
A           f32[n,3]   local position of the shape in its body
B           f32[n,3]   radius (r,0,0) / half extents / cylinder (r, h, r)
C           f32[n,3]   unused for convex shapes
R           f32[n,4]   local rotation quaternion (w, x, y, z)
ID          u32[n]     body of each shape
pos         f32[nb,3]  body position
rot         f32[nb,4]  body rotation quaternion (w, x, y, z)
active      u8[nb]     body active flag (narrowphase only)
==========  =========  ======================================================

Every value is drawn in double from ``numpy.random.Generator(PCG64(seed))``
and stored as float32. All scenes put one shape per body (``ID[i] = i``,
``A = C = 0``, ``R = identity``): the body pose carries the placement.
"""
from __future__ import annotations

import dataclasses

import numpy as np

SPHERE, ELLIPSOID, BOX, CYLINDER, RECT, CONE, TRIANGLEMESH = range(7)


@dataclasses.dataclass
class Scene:
    T: np.ndarray
    A: np.ndarray
    B: np.ndarray
    C: np.ndarray
    R: np.ndarray
    ID: np.ndarray
    pos: np.ndarray
    rot: np.ndarray
    active: np.ndarray
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.T.shape[0])

    @property
    def nb(self) -> int:
        return int(self.pos.shape[0])

    def arrays(self):
        return (self.T, self.A, self.B, self.C, self.R, self.ID, self.pos, self.rot, self.active)

    def nbytes(self) -> int:
        return int(sum(a.nbytes for a in self.arrays()))


def _identity_quats(n):
    q = np.zeros((n, 4), dtype=np.float32)
    q[:, 0] = 1.0
    return q


def random_quaternions(rng, n):
    """Uniform random unit quaternions (w, x, y, z) by Shoemake's method."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    x = a * np.sin(2 * np.pi * u2)
    y = a * np.cos(2 * np.pi * u2)
    z = b * np.sin(2 * np.pi * u3)
    w = b * np.cos(2 * np.pi * u3)
    return np.stack([w, x, y, z], axis=1)


def _one_shape_per_body(T, B, centers, quats, name):
    n = T.shape[0]
    zeros3 = np.zeros((n, 3), dtype=np.float32)
    return Scene(
        T=np.ascontiguousarray(T, dtype=np.int32),
        A=zeros3.copy(),
        B=np.ascontiguousarray(B, dtype=np.float32),
        C=zeros3.copy(),
        R=_identity_quats(n),
        ID=np.arange(n, dtype=np.uint32),
        pos=np.ascontiguousarray(centers, dtype=np.float32),
        rot=np.ascontiguousarray(quats, dtype=np.float32),
        active=np.ones(n, dtype=np.uint8),
        name=name,
    )


def spheres_uniform(n=16384, seed=0, lo=0.0, hi=1.0, rmin=0.002, rmax=0.006):
    """Spheres with centres U[lo,hi]^3 and radii U[rmin,rmax], identity pose.

    Defaults are the 16,384-sphere plain-method workload (its grid is the
    reference's default 16^3, src/broadphase/Broadphase.cu:37).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    c = rng.uniform(lo, hi, size=(n, 3))
    r = rng.uniform(rmin, rmax, size=n)
    B = np.zeros((n, 3))
    B[:, 0] = r
    return _one_shape_per_body(np.full(n, SPHERE), B, c, _identity_quats(n), f"spheres_uniform_{n}")


def mixed_slab(n=1 << 20, seed=0, extent=(10.0, 10.0, 0.5), hmin=0.001, hmax=0.004,
               mix=(0.40, 0.30, 0.15, 0.15)):
    """Mixed convex shapes in a slab.

    Defaults are the 1,048,576-shape workload: 40% spheres, 30% boxes, 15%
    ellipsoids, 15% cylinders (assigned by a seeded shuffle); half extents /
    radii U[0.001, 0.004]; uniform random orientations; centres uniform in
    [0,10] x [0,10] x [0,0.5]. Cylinders store (r, h, r): radius in x and z,
    half height in y (src/SupportFunctions.cuh:52-64), because the AABB stage
    uses B as box half extents (src/aabb/AABBGenerator.cu:108-109).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = [int(round(f * n)) for f in mix]
    counts[0] += n - sum(counts)
    T = np.concatenate([np.full(k, t) for k, t in zip(counts, (SPHERE, BOX, ELLIPSOID, CYLINDER))])
    rng.shuffle(T)
    h = rng.uniform(hmin, hmax, size=(n, 3))
    B = h.copy()
    sph = T == SPHERE
    B[sph, 1:] = 0.0
    cyl = T == CYLINDER
    B[cyl, 2] = B[cyl, 0]
    c = rng.random((n, 3)) * np.asarray(extent)
    q = random_quaternions(rng, n)
    return _one_shape_per_body(T, B, c, q, f"mixed_slab_{n}")


def batched_mixed(num_scenes=512, seed=0, nmin=1000, nmax=200_000, dmin=0.2, dmax=1.0):
    """Independent scenes of uneven size for the batched path.

    Defaults are the 512-scene workload: body counts log-uniform in
    [1,000, 200,000] (mean about 37.6k, about 19M in total), each scene a
    mixed_slab (the 1M workload's shape mix, sizes and orientations) with its
    own fill density d ~ U[0.2, 1.0] read as slab thickness 0.5 / d over the
    10 x 10 footprint. Returns a list of Scene.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=num_scenes)).round().astype(np.int64)
    dens = rng.uniform(dmin, dmax, size=num_scenes)
    return [mixed_slab(int(n), seed=seed * 1_000_003 + 1 + i, extent=(10.0, 10.0, 0.5 / d))
            for i, (n, d) in enumerate(zip(sizes, dens))]


def concat(scenes):
    """Concatenates scenes for the batched entry point: returns (scene,
    shape_offsets, body_offsets). ID stays local to each scene."""
    so = np.zeros(len(scenes) + 1, np.uint64)
    bo = np.zeros(len(scenes) + 1, np.uint64)
    so[1:] = np.cumsum([s.n for s in scenes])
    bo[1:] = np.cumsum([s.nb for s in scenes])
    cat = lambda f: np.ascontiguousarray(np.concatenate([getattr(s, f) for s in scenes]))
    sc = Scene(T=cat("T"), A=cat("A"), B=cat("B"), C=cat("C"), R=cat("R"), ID=cat("ID"), pos=cat("pos"),
               rot=cat("rot"), active=cat("active"), name=f"batch_{len(scenes)}")
    return sc, so, bo


def clustered_spheres(n=1 << 24, seed=0, clusters=64, sigma=0.02, background=0.10,
                      rmin=0.0005, rmax=0.005):
    """Load-imbalanced spheres.

    Defaults are the 16,777,216-sphere workload: radii log-uniform
    [0.0005, 0.005]; 90% of centres from 64 isotropic Gaussians (sigma 0.02)
    whose means are U[0,1]^3, 10% uniform in [0,1]^3.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    nbg = int(round(background * n))
    ncl = n - nbg
    means = rng.random((clusters, 3))
    lab = rng.integers(0, clusters, size=ncl)
    c = np.empty((n, 3))
    c[:ncl] = means[lab] + rng.normal(0.0, sigma, size=(ncl, 3))
    c[ncl:] = rng.random((nbg, 3))
    perm = rng.permutation(n)
    c = c[perm]
    r = np.exp(rng.uniform(np.log(rmin), np.log(rmax), size=n))
    B = np.zeros((n, 3))
    B[:, 0] = r
    return _one_shape_per_body(np.full(n, SPHERE), B, c, _identity_quats(n), f"clustered_spheres_{n}")


def lattice_pairs(m=10, spacing=1.0, radius=0.25):
    """AABB corners of the reference's lattice test (test/binTest_Broadphase.cu:
    13-43): an m^3 lattice with every sphere listed twice, mins then maxs.
    Returns a (2N, 3) float32 array; the known answer is m^3 pairs."""
    idx = np.array([(i, j, k) for k in range(m) for j in range(m) for i in range(m)], dtype=np.float64)
    c = np.repeat(idx * spacing, 2, axis=0).astype(np.float32)
    r = np.float32(radius)
    return np.concatenate([c - r, c + r]).astype(np.float32)


def unit_boxes(n=10):
    """The reference's single-bin test (test/test1.cu:9-33): n identical unit
    boxes [0,1]^3 as (2N, 3) corners; known answer n(n-1)/2 pairs."""
    return np.concatenate([np.zeros((n, 3)), np.ones((n, 3))]).astype(np.float32)


def random_spheres_cube(n, seed=0, lo=-30.0, hi=30.0, rmin=0.1, rmax=1.0):
    """Spheres with the distribution of the reference's completeness and
    timing tests (test/nSquared_Broadphase.cu:30-53): centres U[-30,30]^3,
    radii U[0.1,1], drawn from PCG64 instead of libc rand()."""
    return spheres_uniform(n, seed=seed, lo=lo, hi=hi, rmin=rmin, rmax=rmax)


def sphere_aabbs(scene: Scene) -> np.ndarray:
    """(2N,3) AABBs of a sphere scene the way the reference's tests build
    them: min = c - r, max = c + r in float (test/nSquared_Broadphase.cu:59-72)."""
    c = scene.pos.astype(np.float32)
    r = scene.B[:, :1].astype(np.float32)
    return np.concatenate([c - r, c + r]).astype(np.float32)
