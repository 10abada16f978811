"""Search-grid choice of the broadphase.

``heuristic_dims`` mirrors the device-side default of the library (make_plan
in csrc/cc_broadphase.cu): cells sized so about ``cell_target`` boxes fall in
each, but at least ``min_ratio`` mean box extents wide, capped at 1024 cells
per axis and ``g_max`` cells in total. The pair list does not depend on the
grid; only speed does.

``autotune`` measures a few (cell_target, min_ratio) settings on the actual
scene and keeps the fastest per size bucket; ``tune`` does the same on a
Context, together with the dense-cell threshold (which cells the tiled
dense-cell pair test takes), and leaves the fastest setting on the context.
"""
from __future__ import annotations

import math

import numpy as np

MAX_DIM = 1024


def heuristic_dims(aabb, cell_target=4.0, min_ratio=2.0, g_max=None):
    a = np.asarray(aabb, np.float32)
    n = a.shape[0] // 2
    if n == 0:
        return (1, 1, 1)
    mn, mx = a.min(0), a.max(0)
    origin = np.abs(mn)
    lo, hi = (mn + origin).astype(np.float32), (mx + origin).astype(np.float32)
    ext = (hi - lo).astype(np.float64)
    mean = (a[n:].astype(np.float64) - a[:n]).sum(0) / n
    mean_max = float(mean.max())
    floor_len = max(mean_max, 1e-30)
    vol = float(np.prod(np.maximum(ext, floor_len)))
    c = max(math.pow(vol * cell_target / n, 1.0 / 3.0), min_ratio * mean_max)
    dims = [int(min(max(e / c if c > 0 else 1.0, 1.0), MAX_DIM)) for e in ext]
    g_max = g_max or max(4096, n)
    while dims[0] * dims[1] * dims[2] > g_max:
        dims = [max(1, int(d * 0.8)) for d in dims]
    return tuple(dims)


_cache = {}


def size_bucket(n):
    return int(round(math.log2(max(n, 1)) * 2))


def autotune(run_with, candidates=((2.0, 2.0), (4.0, 2.0), (8.0, 2.0), (4.0, 1.0), (16.0, 1.0)), reps=3,
             key=None):
    """run_with(cell_target, min_ratio) -> seconds of one broadphase call.
    Returns the fastest (cell_target, min_ratio); cached under `key`."""
    if key is not None and key in _cache:
        return _cache[key]
    best, best_t = None, float("inf")
    for cand in candidates:
        t = min(run_with(*cand) for _ in range(reps))
        if t < best_t:
            best, best_t = cand, t
    if key is not None:
        _cache[key] = best
    return best


GRID_CANDIDATES = ((4.0, 2.0), (2.0, 2.0), (8.0, 2.0), (4.0, 1.0), (16.0, 1.0))
DENSE_CANDIDATES = (128, 256, 512)
# sparse pair test: (entries staged per warp, grid cap in blocks per SM)
SHAPE_CANDIDATES = ((96, 8), (64, 8), (128, 5), (96, 4), (64, 16))
DEFAULT = (4.0, 2.0, 128, 96, 8)


def _time_ms(run, reps):
    import torch
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def apply(ctx, choice):
    kt, mr, dc, win, bps = choice
    ctx.set_tuning(kt, mr)
    ctx.set_dense_cell(dc)
    ctx.set_pair_test_shape(win, bps)


def tune(ctx, run, grid_candidates=GRID_CANDIDATES, dense_candidates=DENSE_CANDIDATES,
         shape_candidates=SHAPE_CANDIDATES, reps=1):
    """Times run() (one call through `ctx`) with CUDA events: first every
    (cell_target, min_ratio, dense_cell) candidate at the default launch
    shape, then every pair-test launch shape at the fastest of those; leaves
    the fastest setting on `ctx` and returns (best, [(candidate, ms), ...])
    with candidates (cell_target, min_ratio, dense_cell, window, blocks_per_sm).
    Pairs and contacts do not depend on the choice."""
    table = []
    win0, bps0 = DEFAULT[3], DEFAULT[4]
    for kt, mr in grid_candidates:
        for dc in dense_candidates:
            cand = (kt, mr, dc, win0, bps0)
            apply(ctx, cand)
            run()  # sizes the scratch for this grid
            table.append((cand, _time_ms(run, reps)))
    best = min(table, key=lambda x: x[1])[0]
    for win, bps in shape_candidates:
        cand = best[:3] + (win, bps)
        if cand == best:
            continue
        apply(ctx, cand)
        run()
        table.append((cand, _time_ms(run, reps)))
    best = min(table, key=lambda x: x[1])[0]
    apply(ctx, best)
    return best, table


def tune_cached(ctx, run, n, kind="scene", **kw):
    """tune() once per (kind, size bucket of n): later calls of the same
    bucket only apply the cached choice. Returns (best, table or None)."""
    key = (kind, size_bucket(n))
    if key in _cache:
        apply(ctx, _cache[key])
        return _cache[key], None
    best, table = tune(ctx, run, **kw)
    _cache[key] = best
    return best, table
