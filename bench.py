#!/usr/bin/env python3
"""Benchmark: bodies/s of the collision pipeline (GenerateAABB ->
detectPossibleCollisions -> DoNarrowphase) at 1,048,576 mixed convex shapes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full pipeline pass over the scene (synthetic, seeded: 40%
spheres, 30% boxes, 15% ellipsoids, 15% cylinders; half extents U[0.001,
0.004]; random orientations; centres in [0,10]x[0,10]x[0,0.5]). `value` times
the pipeline on device-resident inputs (L2 flushed between steps), `e2e` the
same through the host-pointer C entry point with the host<->device copies
inside the timed region. N > 1 (torchrun) runs one independent replica per
GPU: weak scaling, no collective on the data path.

The reference arm (--impl reference) times the reference's own CPU/OpenMP
implementation (its sources compiled by oracle/Makefile into oracle/_ref) on
the same scene with every host thread.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "collision-detection_b200")
sys.path.insert(0, PKG_DIR)


def numpy_module(name):
    """collide_b200/<name>.py (scenes, tuner: NumPy only) loaded by file path,
    without running the package's __init__, which maps libcollide_b200.so.
    The reference arm and the CPU-baseline leg use these so that the process
    timing the reference's CPU build never loads this repository's GPU
    library."""
    import importlib.util
    key = f"_bench_{name}"
    if key not in sys.modules:
        spec = importlib.util.spec_from_file_location(key, os.path.join(PKG_DIR, "collide_b200", f"{name}.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[key] = mod  # dataclasses look their module up while the class is built
        spec.loader.exec_module(mod)
    return sys.modules[key]


def mapped_repo_libraries():
    """Shared libraries of this repository mapped into the current process."""
    libs = set()
    try:
        with open("/proc/self/maps") as f:
            for ln in f:
                p = ln.split()[-1] if ln.count("/") else ""
                if p.endswith(".so") and p.startswith(ROOT):
                    libs.add(os.path.relpath(p, ROOT))
    except OSError:
        pass
    return sorted(libs)


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"

N_BODIES = 1 << 20
WORKLOAD = ("mixed_slab: 1,048,576 convex shapes (40% sphere, 30% box, 15% ellipsoid, 15% cylinder), "
            "half extents U[0.001,0.004], uniform random orientations, centres U([0,10]x[0,10]x[0,0.5])")
METRIC, UNIT = "bodies/s", "bodies/s"
BINS = (16, 16, 16)  # the reference's default bins per axis (Broadphase.cu:37)

# Algorithmic bytes per launch of each stage (reads + writes a perfect
# implementation must move), as functions of N bodies, E search entries,
# G search cells, P pairs, C contacts.
STAGE_BYTES = {
    "aabb": lambda N, E, G, P, C: 112 * N,            # 88 B of shape/body data in, 24 B of AABB out
    "bounds": lambda N, E, G, P, C: 24 * N,
    "count": lambda N, E, G, P, C: 48 * N + 4 * G,     # shift in place (24 r + 24 w) + cell counts
    "scan_cells": lambda N, E, G, P, C: 8 * G,
    "scatter": lambda N, E, G, P, C: 24 * N + 4 * G + 32 * E,
    "pair_test": lambda N, E, G, P, C: 32 * E + 4 * G + 8 * P + 4 * N,
    "scan_owner": lambda N, E, G, P, C: 12 * N,
    "owner_scatter": lambda N, E, G, P, C: 16 * P + 8 * N,
    "segsort": lambda N, E, G, P, C: 8 * N + 16 * P,
    "mpr": lambda N, E, G, P, C: P * (8 + 2 * 88) + 56 * P,
    "np_compact": lambda N, E, G, P, C: 60 * P + 60 * C,
}


# Stages of the broadphase proper (detectPossibleCollisions after the AABBs),
# in pipeline order; stages absent from a run are skipped.
BP_STAGES = ("count", "scan_cells", "scatter", "pair_test", "scan_owner", "owner_scatter", "segsort")
STAGE_TIERS = {"segsort": ("segsort_mid", "segsort_big")}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", "--bodies", dest="n", type=int, default=N_BODIES, help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-scene batched measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream measurement")
    ap.add_argument("--no-clustered", action="store_true", help="skip the 16.7M clustered-sphere broadphase")
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--clustered-bodies", type=int, default=1 << 24,
                    help="body count of the clustered-sphere measurement (profiling uses smaller cases)")
    ap.add_argument("--only-clustered", action="store_true",
                    help="run only the clustered-sphere broadphase and print its object (one GPU)")
    ap.add_argument("--only-passes", type=int, default=0,
                    help="profiling: run this many pipeline passes of the headline workload and exit (no timing)")
    return ap.parse_args()


BATCH_WORKLOAD = ("batched_mixed: 512 independent scenes, bodies log-uniform [1,000, 200,000], the 1M workload's "
                  "shape mix, slab thickness 0.5/d with d ~ U[0.2,1.0] over a 10x10 footprint")


def tuner_report(best, table):
    keys = ("cell_target", "min_ratio", "dense_cell", "pair_window", "pair_blocks_per_sm")
    return {"chosen": dict(zip(keys, best)), "candidates_ms": [[list(c), round(t, 3)] for c, t in (table or [])]}


def bench_batched(cb, ctx, dev, steps=10):
    """512 uneven scenes: one cc_collide_batch pass (grid and launch shapes
    from the tuner, replayed as a CUDA graph) against cc_collide per scene."""
    import torch
    from collide_b200 import scenes as S
    from collide_b200 import tuner
    scenes = S.batched_mixed(512, seed=0)
    N = sum(s.n for s in scenes)
    db = cb.DeviceBatch(scenes, device=dev)
    bctx = cb.Context(ctx.device)
    bp = cb.BatchPipeline(db, grid=BINS, ctx=bctx)
    bp.run()
    best, table = tuner.tune_cached(bctx, bp.run, N, kind="batch")
    for _ in range(3):
        bp.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        bp.run()
    e1.record()
    torch.cuda.synchronize()
    tb = e0.elapsed_time(e1) / steps
    P, C = bp.n_pairs, bp.n_contacts
    check = check_batch_sample(bp, db, scenes)  # outside the timed region
    del bp, db
    pipes = [cb.DevicePipeline(cb.DeviceScene(s, device=dev), grid=BINS, ctx=ctx) for s in scenes]
    for p in pipes:
        p.run()
    torch.cuda.synchronize()
    e0.record()
    for p in pipes:
        p.run()
    e1.record()
    torch.cuda.synchronize()
    tl = e0.elapsed_time(e1)
    del pipes, bctx
    import gc
    gc.collect()
    torch.cuda.empty_cache()
    return {"workload": BATCH_WORKLOAD, "scenes": 512, "bodies": N, "pairs": P, "contacts": C,
            "ms_per_batch": tb, "value": N / (tb / 1000.0), "unit": "bodies/s",
            "per_scene_launch": {"ms": tl, "value": N / (tl / 1000.0), "unit": "bodies/s",
                                 "how": "cc_collide once per scene, in order, outputs preallocated"},
            "speedup_vs_per_scene": tl / tb, "steps": steps, "checked": check,
            "tuner": tuner_report(best, table),
            "graph_replay": "the pass repeats with the same configuration, so from the second call on it is one "
                            "CUDA graph launch (cc_collide_batch)"}


def contact_error_stats(gk, norm, cpta, cptb, depth, ref, scale):
    """max / p99 of the contact errors against the FP64 oracle on the pairs
    both report: unit-normal difference, depth difference in units of the
    largest shape size, point difference relative to the point's magnitude."""
    rk = ref["pairs"][: ref["n"]]
    common, gi, ri = np.intersect1d(gk, rk, return_indices=True)
    if not len(common):
        return None, 0, len(np.setdiff1d(gk, rk)) + len(np.setdiff1d(rk, gk))
    nrm = np.linalg.norm(norm[gi].astype(np.float64) - ref["norm"][ri], axis=1)
    dep = np.abs(depth[gi].astype(np.float64) - ref["depth"][ri]) / scale
    pa = np.linalg.norm(cpta[gi].astype(np.float64) - ref["cpta"][ri], axis=1)
    pb = np.linalg.norm(cptb[gi].astype(np.float64) - ref["cptb"][ri], axis=1)
    mag = np.maximum(np.maximum(np.linalg.norm(ref["cpta"][ri], axis=1), np.linalg.norm(ref["cptb"][ri], axis=1)),
                     scale)
    return {"normal": nrm, "depth": dep, "point": np.maximum(pa, pb) / mag}, len(common), \
        len(np.setdiff1d(gk, rk)) + len(np.setdiff1d(rk, gk))


def check_batch_sample(bp, db, scenes, k=16, seed=12345):
    """Checks a seeded sample of k scenes of a finished batch pass against the
    oracle (CPU, after the timing): each scene's pair list bit for bit
    against the oracle's broadphase of that scene alone, and the contacts
    against the FP64 MPR oracle (max / p99 errors over the sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    so = db.shape_offsets.astype(np.int64)
    P, C = bp.n_pairs, bp.n_contacts
    keys = bp.pairs[:P].cpu().numpy()
    ck = keys[:C]
    norm, cpta, cptb = (bp.norm[:C].cpu().numpy(), bp.cpta[:C].cpu().numpy(), bp.cptb[:C].cpu().numpy())
    depth = bp.depth[:C].cpu().numpy()
    coff = bp.contact_offsets.astype(np.int64)
    pick = sorted(np.random.default_rng(seed).choice(len(scenes), size=min(k, len(scenes)), replace=False).tolist())
    errs, exact, bodies, pairs_checked, contacts_checked, set_diff = [], True, 0, 0, 0, 0
    for s in pick:
        sc, a0, a1 = scenes[s], so[s], so[s + 1]
        own = keys >> 32
        mine = keys[(own >= a0) & (own < a1)]
        loc = np.sort(((mine >> 32) - a0) << 32 | ((mine & 0xFFFFFFFF) - a0))
        _, p_ref = O.broadphase(O.aabb(sc), BINS)
        exact &= bool(np.array_equal(loc, p_ref))
        bodies += sc.n
        pairs_checked += len(p_ref)
        c0, c1 = coff[s], coff[s + 1]
        gk = ((ck[c0:c1] >> 32) - a0) << 32 | ((ck[c0:c1] & 0xFFFFFFFF) - a0)
        ref = O.narrowphase(sc, p_ref, 0.0, "f64")
        e, ncom, diff = contact_error_stats(gk, norm[c0:c1], cpta[c0:c1], cptb[c0:c1], depth[c0:c1], ref,
                                            float(np.max(sc.B)))
        contacts_checked += ncom
        set_diff += diff
        if e:
            errs.append(e)
    out = {"scenes": pick, "bodies": int(bodies), "pairs_bit_exact_vs_oracle": exact, "pairs": int(pairs_checked),
           "contacts_compared": int(contacts_checked), "contact_set_differences": int(set_diff),
           "against": "oracle broadphase of each scene alone; FP64 MPR oracle (narrowphase exact mode)"}
    for key in ("normal", "depth", "point"):
        v = np.concatenate([e[key] for e in errs]) if errs else np.zeros(1)
        out[f"{key}_err_max"] = float(v.max())
        out[f"{key}_err_p99"] = float(np.percentile(v, 99))
    return out


CLUSTER_WORKLOAD = ("clustered_spheres: 16,777,216 spheres, radii log-uniform [0.0005,0.005], 90% from 64 "
                    "isotropic Gaussians (sigma 0.02, means U[0,1]^3), 10% U[0,1]^3; broadphase only")


def bench_clustered(cb, dev, steps=3, bodies=1 << 24):
    """The load-imbalanced broadphase: detectPossibleCollisions on 16.7M
    clustered spheres (~3.9e9 pairs, a list the reference's uint32 counters
    cannot hold)."""
    import torch
    from collide_b200 import scenes as S
    sc = S.clustered_spheres(bodies, seed=0)
    ds = cb.DeviceScene(sc, device=dev)
    a0 = cb.AABBGenerator().GenerateAABB(*ds.arrays())
    del ds
    from collide_b200 import tuner
    ctx = cb.Context()
    bp = cb.Broadphase(ctx)
    a = a0.clone()

    def once():
        a.copy_(a0)
        q = bp.detectPossibleCollisions(a)
        torch.cuda.synchronize()
        return int(q.numel())
    P = once()  # sizes the output and the scratch
    best, table = tuner.tune(ctx, once, grid_candidates=((4.0, 2.0), (2.0, 2.0), (8.0, 2.0), (4.0, 1.0)),
                             dense_candidates=(128, 512))
    ms = []
    for _ in range(steps):
        a.copy_(a0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        p = bp.detectPossibleCollisions(a)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
        del p
    dims, E = ctx.last_grid()
    t = statistics.median(ms)
    workload = CLUSTER_WORKLOAD if bodies == 1 << 24 else CLUSTER_WORKLOAD.replace("16,777,216", f"{bodies:,}")
    out = {"workload": workload, "bodies": sc.n, "pairs": P, "search_grid": list(dims), "entries": E,
           "ms_per_step": t, "steps": steps, "value": sc.n / (t / 1000.0), "unit": "bodies/s",
           "pairs_per_s": P / (t / 1000.0),
           "device_gb_in_use": (lambda f: (f[1] - f[0]) / 1e9)(torch.cuda.mem_get_info()),
           "reference": "infeasible: uint32 pair counters (Broadphase.cuh:45) cannot hold 3.9e9 pairs",
           "tuner": tuner_report(best, table)}
    del a, a0, bp, ctx
    torch.cuda.empty_cache()
    return out


SMALL_WORKLOAD = ("spheres_uniform: 16,384 spheres, centres U[0,1]^3, radii U[0.002,0.006], identity orientation "
                  "(the reference's CPU-runnable case)")


def bench_small(cb, dev, steps=200):
    """The 16,384-sphere scene: one cc_collide per step on device-resident
    inputs (graph replay after the second call); launch-latency bound."""
    import torch
    from collide_b200 import scenes as S
    sc = S.spheres_uniform(16384, seed=0)
    pipe = cb.DevicePipeline(cb.DeviceScene(sc, device=dev), grid=BINS, ctx=cb.Context())
    for _ in range(10):
        pipe.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        pipe.run()
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / steps
    return {"workload": SMALL_WORKLOAD, "bodies": sc.n, "pairs": pipe.n_pairs, "contacts": pipe.n_contacts,
            "ms_per_step": t, "value": sc.n / (t / 1000.0), "unit": "bodies/s", "steps": steps,
            "l2": "not flushed (the scene is 1.4 MB)"}


INCREMENTAL_MARGIN = 2.0  # mean box extents (cc_set_incremental)


def bench_incremental(cb, dev, scene, tuned, steps=60):
    """A time-step loop over the 1M scene: before every step all bodies move by
    N(0, 1e-4^2) and turn by at most 1e-3 rad (cc_perturb_bodies, outside the
    timed region); each cc_collide step is timed with CUDA events, with full
    rebuilds and with the incremental broadphase (candidate lists), and every
    step's pairs and contacts are compared between the two."""
    import torch
    from collide_b200 import serving as SV
    from collide_b200 import tuner
    out, ref = {}, []
    for mode in ("full", "incremental"):
        ds = cb.DeviceScene(scene, device=dev)
        ctx = cb.Context()
        tuner.apply(ctx, tuned)
        if mode == "incremental":
            ctx.set_incremental(True, INCREMENTAL_MARGIN)
        pipe = cb.DevicePipeline(ds, grid=BINS, ctx=ctx)
        for _ in range(3):
            pipe.run()
        times, rebuilds, same = [], 0, True
        for k in range(steps):
            SV.perturb_(ctx, ds, 7000 + k, sigma=1e-4, max_angle=1e-3)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            pipe.run()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            P, C = pipe.n_pairs, pipe.n_contacts
            o = (P, C, pipe.pairs[:P].cpu().numpy().tobytes(), pipe.norm[:C].cpu().numpy().tobytes(),
                 pipe.depth[:C].cpu().numpy().tobytes())
            if mode == "full":
                ref.append(o)
            else:
                same = same and o == ref[k]
                rebuilds += int(ctx.last_step_rebuilt() == 1)
        ms = statistics.median(times)
        out[mode] = {"ms_per_step_median": ms, "ms_per_step_mean": statistics.mean(times),
                     "value": scene.n / (ms / 1000.0), "unit": "bodies/s"}
        if mode == "incremental":
            out[mode].update({"rebuild_steps": rebuilds, "margin_mean_extents": INCREMENTAL_MARGIN,
                              "identical_to_full_every_step": same})
    out["workload"] = (f"{WORKLOAD}; {steps} steps, before each all bodies move by N(0,1e-4^2) and turn by <= "
                       "1e-3 rad; the step time excludes the move")
    out["speedup_median"] = out["full"]["ms_per_step_median"] / out["incremental"]["ms_per_step_median"]
    return out


SERVE_WORKLOAD = ("served: Poisson arrivals, 70% time-step updates of a resident scene (positions N(0,1e-4^2), turns "
                  "<= 1e-3 rad), 30% new scenes; 4,096 resident scenes of log-uniform [2,000, 500,000] mixed shapes "
                  "(128 generated scenes, each placed 32 times with its own seeded displacement field); a new scene "
                  "is a generated scene uploaded from pinned host memory and displaced by its query's own seeded "
                  "field; admission by byte accounting against a 150 GB HBM budget, scenes placed in an arena "
                  "reserved at start-up")


def bench_served(cb, dev, seconds):
    """Poisson streams (2,000 and 4,000 queries/s) on 4,096 resident scenes:
    continuous batching against the per-query path, plus the capacity of both
    with about 4,000 queries queued at once (a burst long enough that the
    batched passes run in steady state, not mostly filling and draining)."""
    from collide_b200 import serving as SV
    pool = [SV.PinnedScene(sc) for sc in SV.scene_pool(128, seed=0)]
    R = 4096
    out = {"workload": SERVE_WORKLOAD, "rate_qps": 2000.0, "duration_s": seconds}
    for mode in ("batched", "plain"):
        srv = SV.Server(pool, resident=R, budget_bytes=150e9, max_batch=256, grid=BINS, device=dev,
                        reserve_bytes=int(64e9), distinct=True, tune=True)
        # warm-up: passes of the sizes the timed streams produce, new-scene admissions included
        srv.serve(SV.poisson_stream(4000.0, 0.25, resident=R, pool=len(pool), seed=99), mode=mode)
        r = srv.serve(SV.poisson_stream(2000.0, seconds, resident=R, pool=len(pool), seed=1), mode=mode)
        hot = srv.serve(SV.poisson_stream(4000.0, seconds / 2, resident=R, pool=len(pool), seed=3), mode=mode)
        r["at_4000_qps"] = {k: hot[k] for k in ("queries", "queries_per_s", "p50_ms", "p99_ms", "mean_pass_queries")}
        cap = srv.serve(SV.poisson_stream(1e6, 4e-3, resident=R, pool=len(pool), seed=2), mode=mode)
        r["capacity_queries_per_s"] = cap["queries_per_s"]
        r["capacity_queries"] = cap["queries"]
        r["capacity_host_timing"] = cap.get("host_timing")
        r["initial_resident"] = srv.initial
        r["tuner"] = tuner_report(srv.tuned, None) if srv.tuned else None
        out[mode] = r
        del srv
    del pool
    import gc
    import torch
    gc.collect()  # the servers (arena, contexts) go now, not at some later collection
    torch.cuda.empty_cache()  # the servers' reserved working set goes back before the clustered run
    out["p99_ratio_plain_over_batched"] = out["plain"]["p99_ms"] / out["batched"]["p99_ms"]
    out["p99_ratio_plain_over_batched_at_4000_qps"] = (out["plain"]["at_4000_qps"]["p99_ms"] /
                                                       out["batched"]["at_4000_qps"]["p99_ms"])
    out["capacity_ratio_batched_over_plain"] = (out["batched"]["capacity_queries_per_s"] /
                                                 out["plain"]["capacity_queries_per_s"])
    return out


def scene_for(rank, n):
    return numpy_module("scenes").mixed_slab(n, seed=rank)


# The workload identity both arms print as `config` (rank r uses seed r).
def workload_config(n, world):
    return {"workload": WORKLOAD if n == N_BODIES else WORKLOAD.replace("1,048,576", f"{n:,}"), "bodies": n,
            "seeds": "rank r draws the scene with seed r", "bins_per_axis": list(BINS),
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


# ---------------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling (every 25 ms, with host timestamps) started before
    the warm-up; samples falling inside the timed windows (the device-resident
    pass through the end of the e2e pass, widened by one interval on each
    side) are summarised."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD = 0.025

    def __init__(self, index):
        import threading
        self.index, self.rows, self.stop_flag = index, [], False
        self.window = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", str(int(self.PERIOD * 1000))],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.p.stdout:
            self.rows.append((time.time(), line.strip().split(",")))

    def wait_first(self, timeout=5.0):
        t0 = time.time()
        while self.p is not None and not self.rows and time.time() - t0 < timeout:
            time.sleep(0.02)

    def mark(self, t0, t1):
        self.window = (t0, t1)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        lo, hi = self.window if self.window else (0, float("inf"))
        lo, hi = lo - self.PERIOD, hi + self.PERIOD
        sm, mx, reasons, n = [], 0.0, set(), 0
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, r in self.rows:
            if not (lo <= t <= hi):
                continue
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(k)
                n += 1
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": n}


# ---------------------------------------------------------------------------- distributed
def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def dist_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------- reference (CPU) timing
STAGE_NAMES = ("generate_aabb", "detect_possible_collisions", "do_narrowphase")


def reference_session(scene, threads, grid=None):
    """The reference's own CPU build (oracle/_ref) on `scene`. Its bins per
    axis default to the search grid the GPU path picks for the scene (the
    pair list does not depend on the grid, the reference's speed does)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if grid is None:
        grid = numpy_module("tuner").heuristic_dims(O.aabb(scene))
    return O.RefSession(scene, grid, threads=threads, all_parallel=True), tuple(int(g) for g in grid)


def time_reference(sess, warmup, steps=None, seconds=None, max_steps=50):
    """Per-stage seconds of `steps` runs (or of as many runs as fit in
    `seconds`, at least 3) after `warmup` untimed ones."""
    for _ in range(warmup):
        sess.run()
    rows, t0 = [], time.perf_counter()
    while True:
        t, P, C = sess.run()
        rows.append(t.copy())
        if steps is not None and len(rows) >= steps:
            break
        if steps is None and len(rows) >= 3 and (time.perf_counter() - t0 >= seconds or len(rows) >= max_steps):
            break
    return np.array(rows), P, C


def stage_summary_cpu(rows):
    med = np.median(rows, axis=0)
    return {name: round(1000.0 * float(v), 4) for name, v in zip(STAGE_NAMES, med)}


def cpu_baseline(scene, seconds):
    """The reference's own CPU path on this host, every thread, bounded time:
    the 1M workload at the GPU's grid, and the 16,384-sphere scene at the
    reference's default 16^3 bins (Broadphase.cu:37)."""
    sess, grid = reference_session(scene, os.cpu_count() or 1)
    rows, P, C = time_reference(sess, 1, seconds=seconds)
    med = float(np.median(rows.sum(1)))
    out = {"value": scene.n / med, "unit": UNIT, "cores": sess.threads, "kind": "reference",
           "cpu_model": cpu_model(), "nproc": os.cpu_count(),
           "stages_ms_median": stage_summary_cpu(rows),
           "sample": f"full {scene.n}-shape workload, {len(rows)} runs (median of the per-run stage sums), "
                     f"bins {list(grid)}, all setParallelConfiguration flags on; pairs {P}, contacts {C}"}
    sess.close()
    small = numpy_module("scenes").spheres_uniform(16384, seed=0)
    ss, g16 = reference_session(small, os.cpu_count() or 1, grid=BINS)
    rows, P, C = time_reference(ss, 3, seconds=min(2.0, seconds))
    med = float(np.median(rows.sum(1)))
    out["small_at_default_bins"] = {"workload": SMALL_WORKLOAD, "bins": list(g16), "value": small.n / med,
                                    "unit": UNIT, "ms_per_step": 1000.0 * med, "runs": len(rows),
                                    "stages_ms_median": stage_summary_cpu(rows), "pairs": P, "contacts": C}
    ss.close()
    return out


def run_reference(args):
    world, rank, _ = dist_setup(args.gpus)
    if rank != 0:
        return 0
    scene = scene_for(0, args.n)
    sess, grid = reference_session(scene, os.cpu_count() or 1)
    rows, P, C = time_reference(sess, args.warmup, steps=args.steps)
    ms = 1000.0 * float(rows.sum(1).mean())
    value = scene.n / (ms / 1000.0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(scene.n, world),
        "result": {"pairs": P, "contacts": C, "reference_bins": list(grid)},
        "stages_ms_mean": {k: round(1000.0 * float(v), 4) for k, v in zip(STAGE_NAMES, rows.mean(0))},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": sess.threads, "kind": "reference",
                         "cpu_model": cpu_model(), "nproc": os.cpu_count(),
                         "sample": f"each step = one GenerateAABB + detectPossibleCollisions + DoNarrowphase "
                                   f"of the reference's own CPU/OpenMP build on the full {scene.n}-shape scene, "
                                   f"bins {list(grid)}, every setParallelConfiguration flag on"},
        "native_libraries": mapped_repo_libraries(),
    }
    sess.close()
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------- our arm
def compact_cpus(cpus):
    if not cpus:
        return None
    cpus, out, i = sorted(cpus), [], 0
    while i < len(cpus):
        j = i
        while j + 1 < len(cpus) and cpus[j + 1] == cpus[j] + 1:
            j += 1
        out.append(f"{cpus[i]}-{cpus[j]}" if j > i else f"{cpus[i]}")
        i = j + 1
    return ",".join(out)


def h2d_rate(pinned, dev, stream):
    """GB/s of copying the pinned tensors `pinned` to the device (best of 5)."""
    import torch
    dst = [torch.empty(t.shape, dtype=t.dtype, device=dev) for t in pinned]
    nbytes = sum(t.numel() * t.element_size() for t in pinned)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for d, t in zip(dst, pinned):
            d.copy_(t, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del dst
    return nbytes / (best / 1000.0) / 1e9


def profile_figures():
    """Per-step figures of one ncu capture of this workload (DRAM bytes per
    stage, the MPR's FP64 FLOPs and pipe use), committed under profiles/."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_figures.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def sum_traffic(prof, stages):
    d = prof.get("dram_bytes_per_step") or {}
    if not stages or any(k not in d for k in stages):
        return None
    return sum(d[k] for k in stages)


def merge_tiers(stage):
    """Stages that run as several launches (the bucket sort's tiers) as one."""
    for parent, tiers in STAGE_TIERS.items():
        for tier in tiers:
            if tier in stage and parent in stage:
                stage[parent] = (stage[parent][0] + stage[tier][0], stage[parent][1])
                del stage[tier]
    return stage


def run_ours(args):
    import torch
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    import collide_b200 as cb
    if args.only_clustered:
        if rank == 0:
            print(json.dumps({"clustered": bench_clustered(cb, dev, bodies=args.clustered_bodies)}), flush=True)
        return 0
    scene = scene_for(rank, args.n)
    ctx = cb.Context(local)
    ds = cb.DeviceScene(scene, device=dev)
    pipe = cb.DevicePipeline(ds, grid=BINS, ctx=ctx)
    if args.only_passes:
        for _ in range(args.only_passes):
            pipe.run()
        torch.cuda.synchronize()
        print(json.dumps({"passes": args.only_passes, "pairs": pipe.n_pairs, "contacts": pipe.n_contacts,
                          "launches_per_pass": ctx.launches()}), flush=True)
        return 0
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream()

    # the library's tuner picks the search grid and the pair test's launch
    # shape for this scene (outside the timed region; the line reports it)
    from collide_b200 import tuner
    pipe.run()
    tuned, tune_table = tuner.tune_cached(ctx, pipe.run, scene.n, kind="scene")
    for i in range(max(args.warmup, 3)):
        pipe.run()
        flush.fill_(i & 255)
    torch.cuda.synchronize()
    P, C = pipe.n_pairs, pipe.n_contacts
    dims, E = ctx.last_grid()
    G = dims[0] * dims[1] * dims[2]

    # ---- value: device-resident, per-step CUDA events, L2 flushed between steps
    def timed_pass(profile, spans=False):
        ctx.set_profiling(profile, spans=spans)
        ctx.reset_stage_times()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        nl = 0
        dist_barrier(world)
        torch.cuda.synchronize()
        t0 = time.time()
        for i in range(args.steps):
            flush.fill_((i + 7) & 255)
            evs[i][0].record(stream)
            pipe.run()
            evs[i][1].record(stream)
            nl += ctx.launches()
        torch.cuda.synchronize()
        t1 = time.time()
        dist_barrier(world)
        stages = ctx.stage_times() if profile else None
        ctx.set_profiling(False)
        return sum(a.elapsed_time(b) for a, b in evs), nl, stages, (t0, t1)

    clocks = Clocks(local)
    clocks.wait_first()
    total_ms, launches, _, window = timed_pass(False)
    t_first = window[0]
    total_ms = dist_max(total_ms, world)
    ms = total_ms / args.steps
    value = world * scene.n / (ms / 1000.0)
    # the same steps again with CUDA events around every kernel stage (the
    # event records add host work, so this pass is not the value above)
    prof_ms, _, stage, _ = timed_pass(True)
    # and once more with one event pair around the whole broadphase and one
    # around the narrowphase (in order for this pass, so that the two spans
    # do not overlap): the broadphase's kernels then run back to back
    ov_default = ctx.narrowphase_overlap()
    ctx.set_narrowphase_overlap(False)
    for i in range(3):
        pipe.run()
    torch.cuda.synchronize()
    assert (pipe.n_pairs, pipe.n_contacts) == (P, C)
    span_ms, _, spans, _ = timed_pass(True, spans=True)
    ctx.set_narrowphase_overlap(ov_default)
    # the same steps with the narrowphase overlapped on (or off, whichever the
    # library's default is not): its MPR runs on the unsorted pairs while they are sorted
    alt_ctx = cb.Context(local)
    tuner.apply(alt_ctx, tuned)
    alt_on = not ctx.narrowphase_overlap()
    alt_ctx.set_narrowphase_overlap(alt_on)
    alt = cb.DevicePipeline(ds, grid=BINS, ctx=alt_ctx)
    for i in range(3):
        alt.run()
    torch.cuda.synchronize()
    assert (alt.n_pairs, alt.n_contacts) == (P, C)
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    alt_ms = 0.0
    for i in range(args.steps):
        flush.fill_((i + 11) & 255)
        a0.record(stream)
        alt.run()
        a1.record(stream)
        torch.cuda.synchronize()
        alt_ms += a0.elapsed_time(a1)
    alt_ms = dist_max(alt_ms / args.steps, world)
    alternative = {"narrowphase_overlap": alt_on, "ms_per_step": alt_ms,
                   "value": world * scene.n / (alt_ms / 1000.0),
                   "how": "cc_set_narrowphase_overlap flipped from the default, otherwise the headline's steps"}
    del alt, alt_ctx

    # ---- e2e: the host-pointer entry points, copies inside the timed region.
    # Blocking: cc_collide_host per step. Pipelined (the e2e value): steps
    # submitted two in flight (cc_collide_host_submit / _wait), so the copy of
    # step k+1's inputs overlaps step k's pipeline; every step still copies all
    # of its inputs in and its pairs and contacts out.
    hs = cb.HostSession(scene, grid=BINS, ctx=ctx)
    for i in range(2):
        hs.run()
    evs2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    dist_barrier(world)
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.fill_((i + 3) & 255)
        evs2[i][0].record(stream)
        hs.run()
        evs2[i][1].record(stream)
    torch.cuda.synchronize()
    blocking_ms = dist_max(sum(a.elapsed_time(b) for a, b in evs2) / args.steps, world)
    hp = cb.HostSession(scene, grid=BINS, ctx=ctx)
    for i in range(3):
        hp.submit()
        hp.wait()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist_barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    hp.submit()
    for i in range(1, args.steps):
        hp.submit()
        hp.wait()
    hp.wait()
    e1.record(stream)
    torch.cuda.synchronize()
    # the same pipelined steps with static shapes (cc_set_static_shapes): a
    # time-step loop whose shapes do not change copies the body poses alone
    ctx_s = cb.Context(local)
    tuner.apply(ctx_s, tuned)
    ctx_s.set_static_shapes(True)
    hq = cb.HostSession(scene, grid=BINS, ctx=ctx_s)
    for i in range(3):
        hq.submit()
        hq.wait()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist_barrier(world)
    torch.cuda.synchronize()
    f0.record(stream)
    hq.submit()
    for i in range(1, args.steps):
        hq.submit()
        hq.wait()
    hq.wait()
    f1.record(stream)
    torch.cuda.synchronize()
    clocks.mark(t_first, time.time())
    clk = clocks.stop()
    assert (hp.n_pairs, hp.n_contacts) == (hs.n_pairs, hs.n_contacts)
    e2e_ms = dist_max(e0.elapsed_time(e1) / args.steps, world)
    e2e = {"value": world * scene.n / (e2e_ms / 1000.0), "unit": UNIT, "ms_per_step": e2e_ms,
           "h2d_bytes_per_step": hp.input_bytes(), "d2h_bytes_per_step": hp.output_bytes(),
           "how": "cc_collide_host_submit/_wait, two steps in flight, pinned host buffers; CUDA events on the "
                  "caller's stream around all steps; every input array is copied each step except C, which the "
                  "library reads from the pinned buffer only for CONE and TRIANGLEMESH shapes (none in this "
                  "scene)",
           "blocking": {"ms_per_step": blocking_ms, "value": world * scene.n / (blocking_ms / 1000.0),
                        "how": "cc_collide_host, one step at a time"}}
    assert (hq.n_pairs, hq.n_contacts) == (hs.n_pairs, hs.n_contacts)
    static_ms = dist_max(f0.elapsed_time(f1) / args.steps, world)
    e2e["host_memory"] = {"gpu_numa_node": cb.gpu_numa_node(local),
                          "pinned_on_cpus": compact_cpus(cb.gpu_local_cpus(local)),
                          "h2d_GBps": h2d_rate(hp.inputs, dev, stream),
                          "how": "pinned input buffers allocated while the thread ran on the GPU's NUMA node "
                                 "(sysfs local_cpulist); h2d_GBps = one step's input copies, best of 5"}
    e2e["static_shapes"] = {"ms_per_step": static_ms, "value": world * scene.n / (static_ms / 1000.0),
                            "h2d_bytes_per_step": hq.input_bytes(poses_only=True),
                            "d2h_bytes_per_step": hq.output_bytes(),
                            "how": "as e2e with cc_set_static_shapes on: the shape arrays were copied in the "
                                   "warm-up, every timed step copies body poses and flags in and results out"}

    # ---- rooflines
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback (6650 GB/s)"
    prof = profile_figures()
    stage = merge_tiers(dict(stage))
    kern = {k: v for k, v in stage.items() if k in STAGE_BYTES}
    stage_summary = {k: {"ms_per_launch": v[0] / v[1], "share": v[0] / sum(x[0] for x in kern.values()),
                         "algorithmic_GBps": STAGE_BYTES[k](scene.n, E, G, P, C) / (v[0] / v[1] / 1000) / 1e9}
                     for k, v in kern.items()}
    timing = ("CUDA events around each stage on the launch stream, over a second pass of the same "
              f"{args.steps} steps ({prof_ms / args.steps:.4f} ms/step with the events)")

    # Headline: the broadphase (detectPossibleCollisions: shift and cell count
    # through the sorted pair list) as one unit against HBM bandwidth, with
    # the single-pass byte model 88N + 56E + 16C + 8P (C = candidates; the
    # home-cell test emits no pair twice, so C = P) over the summed stage times.
    bp_present = [k for k in BP_STAGES if k in kern]
    bp_stage_sum_ms = sum(kern[k][0] / kern[k][1] for k in bp_present)
    bp_ms = spans["broadphase_span"][0] / spans["broadphase_span"][1]
    np_span_ms = spans["narrowphase_span"][0] / spans["narrowphase_span"][1]
    bp_bytes = 88 * scene.n + 56 * E + 16 * P + 8 * P
    bp_traffic = sum_traffic(prof, bp_present)
    bp_achieved = bp_bytes / (bp_ms / 1000.0) / 1e9
    roofline = {"bound": "hbm", "kernel": "broadphase: " + " + ".join(bp_present), "achieved": bp_achieved,
                "peak": hbm, "unit": "GB/s", "frac": bp_achieved / hbm, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": bp_bytes, "model": "88*N + 56*E + 16*C + 8*P bytes per step",
                "traffic": bp_traffic, "traffic_source": prof.get("source") if bp_traffic else None,
                "ms_per_launch": bp_ms, "floor_bytes": 24 * scene.n + 8 * P,
                "floor_frac": (24 * scene.n + 8 * P) / (bp_ms / 1000.0) / 1e9 / hbm,
                "pairs_per_s": P / (bp_ms / 1000.0),
                "timing": ("one CUDA event pair around the broadphase's kernels (cell count through the sorted "
                           f"pair list) of each of {args.steps} in-order steps, L2 flushed between steps "
                           f"({span_ms / args.steps:.4f} ms/step; narrowphase span {np_span_ms:.4f} ms)"),
                "stage_sum_ms": bp_stage_sum_ms, "stage_timing": timing}

    # The exact MPR stage is bound by FP64 dependent-chain latency, not by
    # memory: its FP64 FLOPs per launch (ncu thread-instruction counts of the
    # same workload: 2 x DFMA + DADD + DMUL) over its event time, against the
    # FP64 FMA peak measured here by cc_fma_peak.
    fp64_peak = cb.fma_peak(fp64=True)
    fp32_peak = cb.fma_peak(fp64=False)
    mpr = None
    if "mpr" in kern:
        mpr_ms = kern["mpr"][0] / kern["mpr"][1]
        fl = (prof.get("fp64_flops_per_step") or {}).get("mpr")
        mpr = {"bound": "fp64 dependent-chain latency", "unit": "TFLOP/s", "ms_per_launch": mpr_ms,
               "peak": fp64_peak / 1e12, "peak_source": "measured by cc_fma_peak (FP64 FMA, this GPU, this run)",
               "fp32_peak": fp32_peak / 1e12, "flops_per_launch": fl,
               "achieved": fl / (mpr_ms / 1000.0) / 1e12 if fl else None,
               "frac": fl / (mpr_ms / 1000.0) / fp64_peak if fl else None,
               "fp64_pipe_active_pct": prof.get("mpr_fp64_pipe_active_pct"),
               "warps_active_pct": prof.get("mpr_warps_active_pct"),
               "traffic": sum_traffic(prof, ["mpr"]),
               "algorithmic_bytes_per_launch": STAGE_BYTES["mpr"](scene.n, E, G, P, C), "timing": timing}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(scene.n, world),
        "result": {"search_grid": list(dims), "entries": E, "pairs": P, "contacts": C,
                   "l2": "flushed between steps (256 MiB write)", "tuner": tuner_report(tuned, tune_table)},
        "e2e": e2e,
        "roofline": roofline,
        "roofline_mpr": mpr,
        "alternative": alternative,
        "stages": stage_summary,
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_batch:
        line["incremental"] = bench_incremental(cb, dev, scene, tuned)
        line["small"] = bench_small(cb, dev)
        line["batched"] = bench_batched(cb, ctx, dev)
    if rank == 0 and world == 1 and not args.no_serve:
        line["served"] = bench_served(cb, dev, args.serve_seconds)
    if rank == 0 and world == 1 and not args.no_clustered:
        line["clustered"] = bench_clustered(cb, dev, bodies=args.clustered_bodies)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(scene, args.cpu_seconds)
        except Exception as e:  # the reference build is missing: say so, do not fake it
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
