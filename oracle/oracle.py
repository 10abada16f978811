"""ORACLE — test infrastructure only.

numpy front end for the CPU checker:

* ``build/liboracle.so``: the plain-C restatement of the reference path
  (cc_oracle.c). Always available once ``make -C oracle`` ran.
* ``_ref/libccref_f32.so`` / ``_ref/libccref_f64.so``: the reference's own
  sources compiled in host/OpenMP mode against the gpu_math stand-in
  (ref_capi.cu). Built where the reference checkout exists; the built files
  travel with the repository.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may
import this module. The product library never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
P = ctypes.c_void_p
U64 = ctypes.c_uint64
I64 = ctypes.c_int64

_lib = None
_ref = {}


def _p(a):
    return None if a is None else a.ctypes.data_as(P)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "build", "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = ctypes.CDLL(path)
        for f in ("cco_bins", "cco_broadphase", "cco_pairs_bruteforce", "cco_narrowphase_f32_api",
                  "cco_narrowphase_f64_api"):
            getattr(L, f).restype = I64
        _lib = L
    return _lib


def ref_available(prec="f32"):
    return os.path.exists(os.path.join(HERE, "_ref", f"libccref_{prec}.so"))


def ref(prec="f32"):
    if prec not in _ref:
        path = os.path.join(HERE, "_ref", f"libccref_{prec}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference is present")
        L = ctypes.CDLL(path)
        for f in ("ccref_broadphase", "ccref_bins", "ccref_narrowphase"):
            if hasattr(L, f):
                getattr(L, f).restype = I64
        if hasattr(L, "ccref_session_create"):
            L.ccref_session_create.restype = P
        _ref[prec] = L
    return _ref[prec]


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _scene_args(s):
    return (_c(s.T, np.int32), _c(s.A, np.float32), _c(s.B, np.float32), _c(s.C, np.float32),
            _c(s.R, np.float32), _c(s.ID, np.uint32), _c(s.pos, np.float32), _c(s.rot, np.float32),
            _c(s.active, np.uint8))


# ----------------------------------------------------------------------------- AABB
def aabb(scene, init=None):
    """Restated GenerateAABB: (2N,3) float32, mins then maxs."""
    T, A, B, C, R, ID, pos, rot, _ = _scene_args(scene)
    n = T.shape[0]
    out = np.zeros((2 * n, 3), np.float32) if init is None else _c(init, np.float32).copy()
    lib().cco_aabb(U64(n), _p(T), _p(A), _p(B), _p(C), _p(R), _p(ID), _p(pos), _p(rot), _p(out))
    return out


def ref_aabb(scene, init=None):
    """The reference's own GenerateAABB (host build)."""
    T, A, B, C, R, ID, pos, rot, _ = _scene_args(scene)
    n = T.shape[0]
    out = np.zeros((2 * n, 3), np.float32) if init is None else _c(init, np.float32).copy()
    ref().ccref_generate_aabb(U64(n), _p(T), _p(A), _p(B), _p(C), _p(R), _p(ID), U64(pos.shape[0]), _p(pos),
                              _p(rot), _p(out))
    return out


# ----------------------------------------------------------------------------- broadphase
def bounds_shift(aabb_in, grid):
    """Returns (shifted copy, origin[3], inverse bin size[3])."""
    a = _c(aabb_in, np.float32).copy()
    g = _c(grid, np.int32)
    o = np.zeros(3, np.float32)
    s = np.zeros(3, np.float32)
    lib().cco_bounds_shift(U64(a.shape[0] // 2), _p(a), _p(g), _p(o), _p(s))
    return a, o, s


def bins(aabb_in, grid):
    """Restated sorted bin list at `grid`: dict(bins, bodies, active, bin_end,
    shifted)."""
    a, _, s = bounds_shift(aabb_in, grid)
    n = a.shape[0] // 2
    g = _c(grid, np.int32)
    na = U64(0)
    if n == 0:
        e = np.zeros(0, np.uint32)
        return dict(bins=e, bodies=e, active=e, bin_end=e, shifted=a)
    E = lib().cco_bins(U64(n), _p(a), _p(s), _p(g), None, None, None, None, ctypes.byref(na))
    bn = np.zeros(E, np.uint32)
    bd = np.zeros(E, np.uint32)
    ac = np.zeros(na.value, np.uint32)
    be = np.zeros(na.value, np.uint32)
    lib().cco_bins(U64(n), _p(a), _p(s), _p(g), _p(bn), _p(bd), _p(ac), _p(be), ctypes.byref(na))
    return dict(bins=bn, bodies=bd, active=ac, bin_end=be, shifted=a)


def ref_bins(aabb_in, grid):
    """The reference's own sorted bin list (ccref_bins)."""
    a = _c(aabb_in, np.float32).copy()
    n = a.shape[0] // 2
    if n == 0:
        e = np.zeros(0, np.uint32)
        return dict(bins=e, bodies=e, active=e, bin_end=e, shifted=a)
    cap = 1 << 16
    while True:
        b = a.copy()
        bn = np.zeros(cap, np.uint32)
        bd = np.zeros(cap, np.uint32)
        ac = np.zeros(cap, np.uint32)
        be = np.zeros(cap, np.uint32)
        na = U64(0)
        E = ref().ccref_bins(U64(n), _p(b), int(grid[0]), int(grid[1]), int(grid[2]), _p(bn), _p(bd), U64(cap),
                             _p(ac), _p(be), U64(cap), ctypes.byref(na))
        if E <= cap and na.value <= cap:
            return dict(bins=bn[:E], bodies=bd[:E], active=ac[:na.value], bin_end=be[:na.value], shifted=b)
        cap = max(E, na.value)


def broadphase(aabb_in, grid, cap=None):
    """Restated detectPossibleCollisions: (shifted copy, sorted unique int64 keys)."""
    a = _c(aabb_in, np.float32).copy()
    g = _c(grid, np.int32)
    n = a.shape[0] // 2
    cap = cap or max(16, 4 * n)
    while True:
        b = a.copy()
        out = np.zeros(cap, np.int64)
        Pn = lib().cco_broadphase(U64(n), _p(b), _p(g), _p(out), U64(cap))
        if Pn <= cap:
            return b, out[:Pn]
        cap = Pn


def ref_broadphase(aabb_in, grid, par=None, cap=None):
    """The reference's own detectPossibleCollisions: (shifted, keys)."""
    a = _c(aabb_in, np.float32).copy()
    n = a.shape[0] // 2
    cap = cap or max(16, 4 * n)
    pa = None if par is None else _c(par, np.int32)
    while True:
        b = a.copy()
        out = np.zeros(cap, np.int64)
        Pn = ref().ccref_broadphase(U64(n), _p(b), int(grid[0]), int(grid[1]), int(grid[2]), _p(pa), _p(out),
                                    U64(cap))
        if Pn <= cap:
            return b, out[:Pn]
        cap = Pn


def pairs_bruteforce(shifted):
    """All-pairs closed overlap on already-shifted AABBs (small n)."""
    a = _c(shifted, np.float32)
    n = a.shape[0] // 2
    cap = max(16, 4 * n)
    while True:
        out = np.zeros(cap, np.int64)
        Pn = lib().cco_pairs_bruteforce(U64(n), _p(a), _p(out), U64(cap))
        if Pn <= cap:
            return out[:Pn]
        cap = Pn


# ----------------------------------------------------------------------------- narrowphase
def _np_call(fn, scene, pairs, envelope):
    T, A, B, C, R, ID, pos, rot, act = _scene_args(scene)
    pr = _c(pairs, np.int64).copy()
    P_ = pr.shape[0]
    norm = np.zeros((P_, 3))
    ca = np.zeros((P_, 3))
    cb = np.zeros((P_, 3))
    d = np.zeros(P_)
    ids = np.zeros((P_, 2), np.int32)
    nc = fn(U64(T.shape[0]), _p(T), _p(A), _p(B), _p(C), _p(R), _p(ID), U64(pos.shape[0]), _p(act), _p(pos),
            _p(rot), ctypes.c_float(envelope), _p(pr), U64(P_), _p(norm), _p(ca), _p(cb), _p(d), _p(ids))
    return dict(n=int(nc), norm=norm[:nc], cpta=ca[:nc], cptb=cb[:nc], depth=d[:nc], ids=ids[:nc], pairs=pr)


def narrowphase(scene, pairs, envelope=0.0, prec="f64"):
    """Restated DoNarrowphase in float ("f32") or double ("f64", the FP64 MPR
    oracle). Returns dict(n, norm, cpta, cptb, depth, ids, pairs-permuted)."""
    fn = lib().cco_narrowphase_f64_api if prec == "f64" else lib().cco_narrowphase_f32_api
    return _np_call(fn, scene, pairs, envelope)


TYPE_NAMES = ("sphere", "ellipsoid", "box", "cylinder", "rect", "cone", "trianglemesh")


def mpr_iterations(scene, pairs, prec="f64"):
    """Portal discovery and refinement iterations of every MPR call of the
    restated DoNarrowphase (CollideAndFindPoint, Narrowphase.cu:122-314), per
    shape-type class. Pairs that reach MPR are those not skipped by the
    active / same-body filters (:344-349) and not sphere-sphere (:382-397),
    evaluated in list order, so the record of call k belongs to the k-th of
    them. Returns {(type_a, type_b): dict(pairs, discovery_mean, discovery_max,
    refinement_mean, refinement_max)} with type_a <= type_b."""
    L = lib()
    T, A, B, C, R, ID, pos, rot, act = _scene_args(scene)
    pr = _c(pairs, np.int64)
    a, b = (pr >> 32).astype(np.int64), (pr & 0xFFFFFFFF).astype(np.int64)
    ida, idb = ID.astype(np.int64)[a], ID.astype(np.int64)[b]
    ta, tb = T[a], T[b]
    live = (act[ida] != 0) | (act[idb] != 0)
    mpr = live & (ida != idb) & ~((ta == 0) & (tb == 0))
    sink = np.zeros(max(int(mpr.sum()), 1), np.int32)
    getattr(L, f"cco_iter_sink_{prec}")(_p(sink))
    try:
        _np_call(getattr(L, f"cco_narrowphase_{prec}_api"), scene, pr, 0.0)
        cnt = getattr(L, f"cco_iter_count_{prec}")
        cnt.restype = U64
        got = int(cnt())
    finally:
        getattr(L, f"cco_iter_sink_{prec}")(None)
    assert got == int(mpr.sum()), (got, int(mpr.sum()))
    rec = sink[:got]
    p1, p2 = rec // 1000, rec % 1000
    lo, hi = np.minimum(ta[mpr], tb[mpr]), np.maximum(ta[mpr], tb[mpr])
    out = {}
    for x, y in sorted(set(zip(lo.tolist(), hi.tolist()))):
        m = (lo == x) & (hi == y)
        out[(TYPE_NAMES[x], TYPE_NAMES[y])] = dict(
            pairs=int(m.sum()), discovery_mean=float(p1[m].mean()), discovery_max=int(p1[m].max()),
            refinement_mean=float(p2[m].mean()), refinement_max=int(p2[m].max()))
    return out


def ref_narrowphase(scene, pairs, envelope=0.0, prec="f32"):
    """The reference's own DoNarrowphase in real=float or real=double."""
    return _np_call(ref(prec).ccref_narrowphase, scene, pairs, envelope)


# ----------------------------------------------------------------------------- CPU baseline
class RefSession:
    """The reference's CPU path on a resident scene (host vectors built once).
    run() executes GenerateAABB + detectPossibleCollisions + DoNarrowphase and
    returns (seconds per stage [3], pairs, contacts)."""

    def __init__(self, scene, grid, threads=0, all_parallel=True):
        L = ref()
        if threads:
            L.ccref_set_threads(int(threads))
        self.threads = int(L.ccref_max_threads())
        T, A, B, C, R, ID, pos, rot, act = _scene_args(scene)
        self._keep = (T, A, B, C, R, ID, pos, rot, act)
        self.h = L.ccref_session_create(U64(T.shape[0]), _p(T), _p(A), _p(B), _p(C), _p(R), _p(ID),
                                        U64(pos.shape[0]), _p(act), _p(pos), _p(rot), int(grid[0]), int(grid[1]),
                                        int(grid[2]), int(bool(all_parallel)))

    def run(self):
        t = np.zeros(3)
        c = np.zeros(2, np.uint64)
        ref().ccref_session_run(P(self.h), _p(t), _p(c))
        return t, int(c[0]), int(c[1])

    def close(self):
        if self.h:
            ref().ccref_session_destroy(P(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
