"""Serving: a request loop over device-resident scenes with continuous batching.

Scenes stay on the device between queries (one DeviceScene each). A query is
either a time-step update of a resident scene (positions moved by N(0, s^2),
orientations turned by a random-axis rotation of at most a given angle: one
cc_perturb_bodies launch on the device) or a new scene (copied from pinned
host memory, then admitted). Admission is by byte accounting against an HBM
budget: a new scene is admitted when its bytes fit, after evicting idle
scenes least recently used first; otherwise the query is rejected (and
counted). Resident scenes are placed in one device arena reserved when the
server starts, so serving a stream allocates no device memory.

Server.serve() runs an arrival stream against the wall clock. In batched
mode every loop iteration takes ALL queries that have arrived (up to
max_batch), applies their updates / uploads, and collides their scenes in ONE
cc_collide_scenes pass, so queries that arrive while a pass is on the GPU
join the next pass. In plain mode each query runs alone through cc_collide,
in arrival order (the per-query path). Latency is completion minus arrival;
the results of a scene are identical alone and in a batch (every scene gets
its own bounds, shift and grid).
"""
from __future__ import annotations

import ctypes
import gc
import math
import time
from collections import OrderedDict
from dataclasses import dataclass, field

import numpy as np
import torch

from . import Context, DevicePipeline, DeviceScene, ScenesPipeline, _lib, _stream, lib, numa_local
from . import scenes as S


def scene_bytes(scene) -> int:
    """Device bytes a resident scene holds: its inputs plus its AABBs."""
    return int(scene.nbytes() + 24 * scene.n)


def perturb_(ctx: Context, ds: DeviceScene, seed: int, sigma=1e-4, max_angle=1e-3):
    """Time-step update of a device-resident scene (cc_perturb_bodies)."""
    ctx.check(lib.cc_perturb_bodies(ctx.h, ds.nb, ds.pos.data_ptr(), ds.rot.data_ptr(), ctypes.c_uint64(seed),
                                    float(sigma), float(max_angle), _stream()), "cc_perturb_bodies")


def _pos_ptr(ds):
    return ds.pos_ptr if isinstance(ds, ArenaScene) else ds.pos.data_ptr()


def _rot_ptr(ds):
    return ds.rot_ptr if isinstance(ds, ArenaScene) else ds.rot.data_ptr()


def perturb_many(ctx: Context, updates, sigma=1e-4, max_angle=1e-3):
    """Time-step updates [(DeviceScene, seed), ...] in as few launches as
    possible (cc_perturb_scenes): one per round of distinct scenes, a scene
    updated twice going into the next round, so every scene gets its updates
    in list order, exactly as perturb_ one at a time gives them."""
    rounds = []
    for ds, seed in updates:
        for r in rounds:
            if id(ds) not in r:
                r[id(ds)] = (ds, seed)
                break
        else:
            rounds.append({id(ds): (ds, seed)})
    for r in rounds:
        items = list(r.values())
        k = len(items)
        nb = (ctypes.c_uint64 * k)(*[ds.nb for ds, _ in items])
        pos = (ctypes.c_void_p * k)(*[_pos_ptr(ds) for ds, _ in items])
        rot = (ctypes.c_void_p * k)(*[_rot_ptr(ds) for ds, _ in items])
        seeds = (ctypes.c_uint64 * k)(*[int(sd) & (2**64 - 1) for _, sd in items])
        ctx.check(lib.cc_perturb_scenes(ctx.h, k, nb, pos, rot, seeds, float(sigma), float(max_angle), _stream()),
                  "cc_perturb_scenes")


class PinnedScene:
    """A host scene in one pinned buffer laid out exactly as its device copy
    (the nine arrays at 256-byte aligned offsets), so an upload is a single
    copy into arena space. C comes last: it is read only for CONE and
    TRIANGLEMESH shapes, so a scene without them uploads everything before it
    (the arena keeps C's space; nothing reads it)."""

    FIELDS = (("T", np.int32), ("A", np.float32), ("B", np.float32), ("R", np.float32), ("ID", np.int32),
              ("pos", np.float32), ("rot", np.float32), ("active", np.uint8), ("C", np.float32))

    def __init__(self, scene):
        self.scene = scene
        self.n, self.nb = scene.n, scene.nb
        arrays = {k: np.ascontiguousarray(getattr(scene, k)) for k, _ in self.FIELDS}
        arrays["ID"] = np.ascontiguousarray(arrays["ID"], dtype=np.uint32).view(np.int32)
        self.layout, off = [], 0
        for k, dt in self.FIELDS:
            a = np.ascontiguousarray(arrays[k], dtype=dt)
            self.layout.append((k, off, a.shape, dt))
            off += _align(a.nbytes)
        self.total = off
        T = arrays["T"]
        needs_c = bool(np.any((T == 5) | (T == 6)))  # CONE, TRIANGLEMESH
        #: bytes an upload copies
        self.copy_bytes = self.total if needs_c else next(o for k, o, _, _ in self.layout if k == "C")
        with numa_local():  # pages on the GPU's NUMA node
            self.buf = torch.empty(max(self.total, 1), dtype=torch.uint8, pin_memory=True)
            host = self.buf.numpy()
            for k, off, shape, dt in self.layout:
                a = np.ascontiguousarray(arrays[k], dtype=dt)
                host[off:off + a.nbytes] = a.view(np.uint8).reshape(-1)

    def nbytes(self):
        return self.scene.nbytes()

    def device_bytes(self) -> int:
        """Bytes of the device copy, each array starting on a 256-byte boundary."""
        return self.total

    def upload(self, device, copy_stream=None, space=None) -> DeviceScene:
        """The device copy, filled by one copy on copy_stream if given. space:
        a uint8 device tensor of device_bytes() to hold the arrays (views into
        it); without it the scene gets one new allocation."""
        if space is None:
            space = torch.empty(max(self.total, 1), dtype=torch.uint8, device=device)
        k = self.copy_bytes
        if copy_stream is None:
            space[:k].copy_(self.buf[:k], non_blocking=True)
        else:
            with torch.cuda.stream(copy_stream):
                space[:k].copy_(self.buf[:k], non_blocking=True)
        return ArenaScene(space, self.layout, self.n, self.nb)


class ArenaScene(DeviceScene):
    """A DeviceScene whose nine arrays sit at fixed offsets of one device
    buffer. The C scene descriptor comes straight from the buffer's address;
    the torch views of the arrays are made only when something asks for one
    (an admission costs one copy, not nine view constructions)."""

    _FIELDS = tuple(k for k, _ in PinnedScene.FIELDS)

    def __init__(self, space, layout, n, nb):
        self.n, self.nb = n, nb
        self._space, self._layout = space, layout
        base = space.data_ptr()
        self._ptr = {k: base + off for k, off, _, _ in layout}

    def __getattr__(self, name):
        if name in ArenaScene._FIELDS:
            for k, off, shape, dt in self._layout:
                if k == name:
                    nbytes = int(np.prod(shape)) * np.dtype(dt).itemsize
                    t = self._space[off:off + nbytes].view(_TORCH_DTYPE[np.dtype(dt)])
                    t = t.view(shape) if len(shape) > 1 else t
                    setattr(self, name, t)
                    return t
        raise AttributeError(name)

    def c_scene(self):
        c = self.__dict__.get("_c")
        if c is not None:
            return c
        p = self._ptr
        c = _lib.Scene()
        c.n, c.nb = self.n, self.nb
        c.T, c.A, c.B, c.C, c.R, c.ID = p["T"], p["A"], p["B"], p["C"], p["R"], p["ID"]
        c.body_pos, c.body_rot, c.active = p["pos"], p["rot"], p["active"]
        self._c = c
        return c

    @property
    def pos_ptr(self):
        return self._ptr["pos"]

    @property
    def rot_ptr(self):
        return self._ptr["rot"]


_TORCH_DTYPE = {np.dtype(np.int32): torch.int32, np.dtype(np.float32): torch.float32,
                np.dtype(np.uint8): torch.uint8}


def _align(nbytes, a=256):
    return (int(nbytes) + a - 1) // a * a


class Arena:
    """One device buffer holding the resident scenes' arrays. Free ranges are
    indexed by size (best fit, O(log F)) and by both ends (a freed range merges
    with free neighbours in O(1)), so admissions stay cheap while evictions of
    scenes of very different sizes fragment the buffer. Admitting a scene is a
    copy into space the server already owns: no device allocation (cudaMalloc
    stalls every thread that uses the device) while queries are served."""

    def __init__(self, nbytes, device):
        from sortedcontainers import SortedList
        self.size = _align(nbytes)
        self.buf = torch.empty(self.size, dtype=torch.uint8, device=device)
        self._by_size = SortedList([(self.size, 0)])  # (bytes, offset)
        self._at_start = {0: self.size}               # offset -> bytes
        self._at_end = {self.size: 0}                 # offset + bytes -> offset

    @property
    def free(self):
        """Free ranges (offset, bytes) in address order."""
        return sorted(self._at_start.items())

    def _add(self, off, nbytes):
        self._by_size.add((nbytes, off))
        self._at_start[off] = nbytes
        self._at_end[off + nbytes] = off

    def _remove(self, off, nbytes):
        self._by_size.remove((nbytes, off))
        del self._at_start[off]
        del self._at_end[off + nbytes]

    def take(self, nbytes):
        nbytes = _align(nbytes)
        k = self._by_size.bisect_left((nbytes, -1))
        if k == len(self._by_size):
            return None
        sz, off = self._by_size[k]
        self._remove(off, sz)
        if sz > nbytes:
            self._add(off + nbytes, sz - nbytes)
        return off

    def give(self, off, nbytes):
        nbytes = _align(nbytes)
        nxt = self._at_start.get(off + nbytes)
        if nxt is not None:  # merge the next range
            self._remove(off + nbytes, nxt)
            nbytes += nxt
        prv = self._at_end.get(off)
        if prv is not None:  # and the previous
            psz = self._at_start[prv]
            self._remove(prv, psz)
            off, nbytes = prv, nbytes + psz
        self._add(off, nbytes)


@dataclass
class Query:
    arrival: float          # seconds after the stream starts
    kind: str               # "update" | "new"
    scene: int              # resident slot (update) or pool index (new)
    seed: int = 0
    done: float = math.nan  # completion time, seconds after the start
    n_pairs: int = 0
    n_contacts: int = 0
    record: bool = False    # keep this query's scene state and contacts (query.result) for checking
    result: dict | None = None


@dataclass
class Stream:
    queries: list = field(default_factory=list)


def poisson_stream(rate=2000.0, duration=1.0, resident=256, pool=64, update_frac=0.7, seed=0) -> Stream:
    """Poisson arrivals (mean `rate` per second) over `duration` seconds:
    `update_frac` updates of a random resident scene, the rest new scenes
    drawn from a pool of `pool` pre-generated scenes."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t, qs = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        if rng.random() < update_frac:
            qs.append(Query(t, "update", int(rng.integers(0, resident)), int(rng.integers(0, 2**31))))
        else:
            qs.append(Query(t, "new", int(rng.integers(0, pool)), int(rng.integers(0, 2**31))))
    return Stream(qs)


def scene_pool(count=64, nmin=2000, nmax=500_000, seed=0):
    """Scenes of log-uniform size in [nmin, nmax] with the 1M workload's shape
    mix, for new-scene queries and the initial resident set."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=count)).round().astype(np.int64)
    return [S.mixed_slab(int(n), seed=seed * 7919 + 1 + i, extent=(10.0, 10.0, 0.5)) for i, n in enumerate(sizes)]


# A new scene is a pool scene displaced by its query's own seeded field, so no
# two admitted scenes are equal (the resident set is placed the same way).
NEW_SIGMA, NEW_ANGLE = 1e-3, 1e-2


class Server:
    def __init__(self, pool, resident=256, budget_bytes=150e9, max_batch=256, grid=(16, 16, 16), precision="exact",
                 device="cuda", reserve_bytes=None, distinct=False, tune=False):
        # the resident scenes live in one arena reserved up front, so admitting
        # a scene costs a copy, not a device allocation (reserve_bytes=0: one
        # allocation per array instead)
        reserve = int(min(budget_bytes, 32e9) if reserve_bytes is None else reserve_bytes)
        self.arena = Arena(reserve, device) if reserve > 0 else None
        self.pool = [p if isinstance(p, PinnedScene) else PinnedScene(p) for p in pool]
        self.device = device
        # the batched loop's streams, kept for the server's lifetime
        self.copy_s, self.pass_s = torch.cuda.Stream(device), torch.cuda.Stream(device)
        self.budget, self.max_batch, self.grid = float(budget_bytes), int(max_batch), tuple(grid)
        self.ctx = Context()
        self.ctx.set_narrowphase_precision(precision)
        self.resident: OrderedDict[int, DeviceScene] = OrderedDict()  # LRU order, oldest first
        self.bytes = 0
        self.next_id = 0
        self.batch = ScenesPipeline(self.ctx, grid=self.grid)
        self.plain = None  # the per-query path's outputs, shared by every scene (sized for the largest)
        self.rejected = 0
        for i in range(resident):
            if self.admit(self.pool[i % len(self.pool)]) is None:
                break
        self.initial = len(self.resident)
        self.slots = list(self.resident)  # the scenes update queries address
        if distinct:  # every placement of a pool scene gets its own displacement
            perturb_many(self.ctx, [(self.resident[s], 1_000_003 * (k + 1)) for k, s in enumerate(self.slots)],
                         NEW_SIGMA, NEW_ANGLE)
        # size the library's scratch once for a full pass over resident scenes
        # (it only grows, by half at a time, after that)
        warm = [self.resident[s] for s in self.slots[: self.max_batch]]
        self.tuned = None
        if warm:
            self.batch.run(warm)
            if tune:  # search grid and launch shapes for passes of this size (cached per size bucket)
                from . import tuner
                self.tuned, _ = tuner.tune_cached(self.ctx, lambda: self.batch.run(warm),
                                                  sum(d.n for d in warm), kind="served")
        torch.cuda.synchronize()

    # -- residency ------------------------------------------------------
    def admit(self, ps: PinnedScene, pinned=(), copy_stream=None):
        """Makes a pool scene resident; evicts idle scenes (least recently
        used first, never one in `pinned`) until it fits. Returns its id, or
        None if it cannot fit. The upload runs on copy_stream if given."""
        need = int(ps.nbytes() + 24 * ps.n)
        place = ps.device_bytes()

        # evict least recently used idle scenes until the scene fits the
        # budget and a free range of the arena; the oldest idle scene is found
        # from the front of the LRU order, skipping only the pinned ones
        at = None
        while True:
            if self.bytes + need <= self.budget:
                at = self.arena.take(place) if self.arena is not None else -1
                if at is not None:
                    break
            sid = next((s for s in self.resident if s not in pinned), None)
            if sid is None:
                self.rejected += 1
                return None
            self._evict(sid)
        space = None if self.arena is None else self.arena.buf[at:at + place]
        ds = ps.upload(self.device, copy_stream, space)
        ds.arena_at, ds.arena_bytes = at, place
        ds.resident_bytes = need
        sid = self.next_id
        self.next_id += 1
        self.resident[sid] = ds
        self.bytes += need
        return sid

    def _evict(self, sid):
        ds = self.resident.pop(sid)
        self.bytes -= ds.resident_bytes
        if self.arena is not None:
            self.arena.give(ds.arena_at, ds.arena_bytes)

    def _prepare(self, q: Query, pinned=()):
        """Applies a query's input; returns its resident scene id (None: the
        scene is gone or did not fit the budget)."""
        if q.kind == "new":
            sid = self.admit(self.pool[q.scene], pinned)
            if sid is not None:
                perturb_(self.ctx, self.resident[sid], q.seed, NEW_SIGMA, NEW_ANGLE)
            return sid
        sid = self.slots[q.scene % len(self.slots)]
        if sid not in self.resident:  # evicted: the update has nothing to move
            return None
        self.resident.move_to_end(sid)
        perturb_(self.ctx, self.resident[sid], q.seed)
        return sid

    # -- passes ---------------------------------------------------------
    @staticmethod
    def _scene_copy(ds):
        return {k: getattr(ds, k).clone() for k, _ in PinnedScene.FIELDS}

    def _record_batch(self, k, scenes):
        """Scene k of the last batched pass: its arrays as collided and its
        contacts in the scene's own numbering."""
        b = self.batch
        co = b.contact_offsets.astype(np.int64)
        off = sum(d.n for d in scenes[:k])
        c0, c1 = int(co[k]), int(co[k + 1])
        keys = b.pairs[c0:c1]
        local = ((keys >> 32) - off) * (1 << 32) + ((keys & 0xFFFFFFFF) - off)
        return dict(scene=self._scene_copy(scenes[k]), n_pairs=int(b.scene_pairs[k]), n_contacts=c1 - c0,
                    contact_pairs=local.clone(), norm=b.norm[c0:c1].clone(), depth=b.depth[c0:c1].clone(),
                    cpta=b.cpta[c0:c1].clone(), cptb=b.cptb[c0:c1].clone())

    def _record_plain(self, sid):
        p = self.plain
        C = p.n_contacts
        return dict(scene=self._scene_copy(self.resident[sid]), n_pairs=p.n_pairs, n_contacts=C,
                    contact_pairs=p.pairs[:C].clone(), norm=p.norm[:C].clone(), depth=p.depth[:C].clone(),
                    cpta=p.cpta[:C].clone(), cptb=p.cptb[:C].clone())

    def collide_batch(self, sids):
        self.batch.run([self.resident[s] for s in sids])
        co = self.batch.contact_offsets.astype(np.int64)
        return [(int(self.batch.scene_pairs[i]), int(co[i + 1] - co[i])) for i in range(len(sids))]

    def collide_one(self, sid):
        """cc_collide on one resident scene into the shared output buffers."""
        if self.plain is None:
            big = max(self.pool, key=lambda ps: ps.n)
            self.plain = DevicePipeline(self.resident[sid], grid=self.grid, ctx=self.ctx,
                                        pairs_cap=max(1024, big.n // 4))
            self.plain.aabb = torch.zeros((2 * big.n, 3), dtype=torch.float32, device=self.device)
            self.plain.res.aabb = self.plain.aabb.data_ptr()
        p = self.plain
        p.ds = self.resident[sid]
        p.scene = p.ds.c_scene()
        return p.run()

    def serve(self, stream: Stream, mode="batched"):
        """Runs a query stream; Python's cyclic garbage collector is paused
        meanwhile (a full collection stalls the loop for tens of ms)."""
        was = gc.isenabled()
        gc.disable()
        try:
            return self._serve(stream, mode)
        finally:
            if was:
                gc.enable()

    def _serve(self, stream: Stream, mode):
        if mode == "batched":
            return self._serve_batched(stream)
        qs = stream.queries
        t0 = time.perf_counter()
        timing = {"prepare_s": 0.0, "collide_s": 0.0}
        self.last_timing = timing
        i = 0  # next query not yet taken
        while i < len(qs):
            now = time.perf_counter() - t0
            if qs[i].arrival > now:
                time.sleep(min(qs[i].arrival - now, 2e-4))
                continue
            q = qs[i]
            i += 1
            tp = time.perf_counter()
            sid = self._prepare(q)
            tc = time.perf_counter()
            if sid is not None:
                q.n_pairs, q.n_contacts = self.collide_one(sid)
                if q.record:
                    q.result = self._record_plain(sid)
            torch.cuda.synchronize()
            q.done = time.perf_counter() - t0
            timing["prepare_s"] += tc - tp
            timing["collide_s"] += time.perf_counter() - tc
        return self._report(qs, t0, [1] * len(qs), mode)

    def _report(self, qs, t0, passes, mode):
        wall = time.perf_counter() - t0
        lat = np.array([q.done - q.arrival for q in qs]) * 1e3
        out = dict(mode=mode, queries=len(qs), wall_s=wall, queries_per_s=len(qs) / wall,
                   p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                   mean_ms=float(lat.mean()), passes=len(passes), mean_pass_queries=float(np.mean(passes)),
                   rejected=self.rejected, resident=len(self.resident), resident_gb=self.bytes / 1e9)
        if getattr(self, "last_timing", None):
            out["host_timing"] = dict(self.last_timing)
        return out

    def _serve_batched(self, stream: Stream):
        """Continuous batching with the host side overlapped: a worker thread
        runs the passes (time-step updates, then one cc_collide_scenes over
        the pass's scenes, or cc_collide when the pass has one scene) on its
        own CUDA stream, while this thread admits
        the next arrivals and uploads their new scenes on a copy stream. A
        pass waits for its uploads (an event); scenes referenced by a pass in
        flight are never evicted."""
        import queue
        import threading
        qs = stream.queries
        jobs: queue.Queue = queue.Queue(maxsize=1)
        copy_s, pass_s = self.copy_s, self.pass_s
        busy: dict[int, int] = {}  # scene id -> passes in flight that use it
        lock = threading.Lock()
        passes = []
        failure = []
        t0 = time.perf_counter()
        # where the host time goes (seconds; bytes copied in for new scenes)
        timing = {"prepare_s": 0.0, "admit_s": 0.0, "pass_s": 0.0, "upload_bytes": 0}
        self.last_timing = timing

        def worker():
            try:
                with torch.cuda.stream(pass_s):
                    while True:
                        job = jobs.get()
                        if job is None:
                            return
                        ev, arrivals, updates, uniq, scenes, live, take = job
                        tw = time.perf_counter()
                        pass_s.wait_event(ev)
                        perturb_many(self.ctx, arrivals, NEW_SIGMA, NEW_ANGLE)
                        perturb_many(self.ctx, updates)
                        if len(uniq) == 1:
                            # a pass of one scene runs as a single-scene call (its CUDA graph
                            # replays; same results as in a batch)
                            sid = uniq[0]
                            one = self.collide_one(sid)
                            for q, _ in live:
                                q.n_pairs, q.n_contacts = one
                                if q.record:
                                    q.result = self._record_plain(sid)
                        elif uniq:
                            self.batch.run(scenes)
                            co = self.batch.contact_offsets.astype(np.int64)
                            res = {sid: (int(self.batch.scene_pairs[k]), int(co[k + 1] - co[k]))
                                   for k, sid in enumerate(uniq)}
                            for q, sid in live:
                                q.n_pairs, q.n_contacts = res[sid]
                                if q.record:
                                    q.result = self._record_batch(uniq.index(sid), scenes)
                        pass_s.synchronize()
                        t = time.perf_counter() - t0
                        timing["pass_s"] += time.perf_counter() - tw
                        for q in take:
                            q.done = t
                        with lock:
                            for sid in uniq:
                                busy[sid] -= 1
                                if busy[sid] == 0:
                                    del busy[sid]
            except Exception as e:  # surfaced by the main thread
                failure.append(e)

        th = threading.Thread(target=worker, daemon=True)
        th.start()
        i = 0
        try:
            while i < len(qs) and not failure:
                now = time.perf_counter() - t0
                if qs[i].arrival > now or jobs.full():
                    time.sleep(2e-4 if qs[i].arrival <= now else min(qs[i].arrival - now, 2e-4))
                    continue
                j = i
                while j < len(qs) and j - i < self.max_batch and qs[j].arrival <= now:
                    j += 1
                take = qs[i:j]
                i = j
                tp = time.perf_counter()
                with lock:
                    pinned = set(busy)
                updates, arrivals, live = [], [], []
                for q in take:
                    if q.kind == "new":
                        ta = time.perf_counter()
                        sid = self.admit(self.pool[q.scene], pinned, copy_s)
                        timing["admit_s"] += time.perf_counter() - ta
                        if sid is not None:
                            arrivals.append((self.resident[sid], q.seed))
                            timing["upload_bytes"] += self.pool[q.scene].copy_bytes
                    else:
                        sid = self.slots[q.scene % len(self.slots)]
                        if sid not in self.resident:
                            sid = None
                        else:
                            self.resident.move_to_end(sid)
                            updates.append((self.resident[sid], q.seed))
                    if sid is not None:
                        pinned.add(sid)
                        live.append((q, sid))
                ev = copy_s.record_event()
                # a scene updated twice in one pass is collided once, after both updates
                uniq = list(dict.fromkeys(sid for _, sid in live))
                scenes = [self.resident[sid] for sid in uniq]
                with lock:
                    for sid in uniq:
                        busy[sid] = busy.get(sid, 0) + 1
                timing["prepare_s"] += time.perf_counter() - tp
                jobs.put((ev, arrivals, updates, uniq, scenes, live, take))
                passes.append(len(take))
        finally:
            while th.is_alive():  # the worker may have stopped on an error
                try:
                    jobs.put(None, timeout=0.05)
                    break
                except queue.Full:
                    continue
            th.join()
        if failure:
            raise failure[0]
        torch.cuda.synchronize()
        return self._report(qs, t0, passes, "batched")
