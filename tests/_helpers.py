"""Shared helpers of the GPU tests (not collected: no test_ prefix)."""
import os

import numpy as np

from collide_b200 import scenes as S

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return dict(np.load(os.path.join(GOLD, f"{name}.npz")))


def scene_of(g):
    return S.Scene(T=g["T"], A=g["A"], B=g["B"], C=g["C"], R=g["R"], ID=g["ID"], pos=g["pos"], rot=g["rot"],
                   active=g["active"])


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def same_bits(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and np.array_equal(bits(a), bits(b))


def pair_set_diff(a, b):
    a, b = set(np.asarray(a).tolist()), set(np.asarray(b).tolist())
    return len(a - b), len(b - a)


def contact_errors(gpu, ref, scale):
    """Per-contact errors of the GPU narrowphase against the FP64 oracle on the
    pairs both report as contacts. gpu/ref: dicts with contact_pairs/pairs,
    norm, cpta, cptb, depth. scale: length scale for relative errors."""
    gk = np.asarray(gpu["contact_pairs"])
    rk = np.asarray(ref["pairs"][: ref["n"]])
    common, gi, ri = np.intersect1d(gk, rk, return_indices=True)
    out = dict(n_gpu=len(gk), n_ref=len(rk), n_common=len(common))
    if len(common) == 0:
        return out
    gn, rn = np.asarray(gpu["norm"], np.float64)[gi], ref["norm"][ri]
    out["normal"] = np.linalg.norm(gn - rn, axis=1)
    out["depth"] = np.abs(np.asarray(gpu["depth"], np.float64)[gi] - ref["depth"][ri]) / scale
    # contact points are float32 world coordinates: errors relative to the
    # point's magnitude (what a float32 output can resolve), at least `scale`
    pa = np.linalg.norm(np.asarray(gpu["cpta"], np.float64)[gi] - ref["cpta"][ri], axis=1)
    pb = np.linalg.norm(np.asarray(gpu["cptb"], np.float64)[gi] - ref["cptb"][ri], axis=1)
    mag = np.maximum(np.maximum(np.linalg.norm(ref["cpta"][ri], axis=1), np.linalg.norm(ref["cptb"][ri], axis=1)),
                     scale)
    out["point"] = np.maximum(pa, pb) / mag
    out["only_gpu"] = np.setdiff1d(gk, rk)
    out["only_ref"] = np.setdiff1d(rk, gk)
    return out
