"""collide_b200: the reference's collision classes over the B200 kernels.

Python mirror of the public C++ API of uwsbel/collision-detection
(src/aabb/AABBGenerator.cuh, src/broadphase/Broadphase.cuh,
src/narrowphase/Narrowphase.cuh) on torch CUDA tensors, calling
libcollide_b200.so through its C ABI. Method names, argument order and side
effects follow the reference:

* ``AABBGenerator.GenerateAABB(T, A, B, C, R, ID, body_pos, body_rot, aabb)``
* ``Broadphase.detectPossibleCollisions(aabb)`` shifts ``aabb`` in place and
  returns the sorted unique int64 pair keys ((min << 32) | max);
  ``setBinsPerAxis``/``getNumPossibleContacts`` and the other setters keep
  their meaning (``setParallelConfiguration`` chose OpenMP vs sequential
  Thrust on the host and has no effect on the GPU; ``setBodyPerBin`` only fed
  dead code in the reference, Broadphase.cu:458-468).
* ``Narrowphase.DoNarrowphase(...)`` returns the contacts and permutes the pair
  tensor in place (contacts' pairs first).

Where the reference returns nothing and reports no error, these raise
:class:`CollideError` with the C status.

PyTorch only provides device memory and the current stream here.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib
from ._lib import CollideError, lib, version  # noqa: F401
from . import scenes  # noqa: F401

__all__ = ["Context", "AABBGenerator", "Broadphase", "Narrowphase", "DeviceScene", "DevicePipeline", "HostSession",
           "collide", "collide_host", "CollideError", "version", "scenes"]

_default_ctx = {}


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _gpu_pci_dir(device):
    pr = torch.cuda.get_device_properties(device)
    bdf = f"{pr.pci_domain_id:04x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
    return os.path.join("/sys/bus/pci/devices", bdf)


def _parse_cpulist(text):
    cpus = set()
    for part in text.strip().split(","):
        if not part:
            continue
        lo, _, hi = part.partition("-")
        cpus.update(range(int(lo), int(hi or lo) + 1))
    return cpus


def gpu_numa_node(device=None):
    """NUMA node of the GPU's PCI device (sysfs), or None if unknown."""
    try:
        if device is None:
            device = torch.cuda.current_device()
        with open(os.path.join(_gpu_pci_dir(device), "numa_node")) as f:
            node = int(f.read().strip())
        return node if node >= 0 else None
    except Exception:
        return None


def gpu_local_cpus(device=None):
    """CPUs on the GPU's own NUMA node, or None if unknown: the PCI device's
    local_cpulist in sysfs (the same GPU as CUDA's device index, whatever
    CUDA_VISIBLE_DEVICES says), else NVML. Host buffers that feed the GPU
    belong on that node: a copy from the other socket's memory crosses the
    inter-socket link first."""
    if device is None:
        device = torch.cuda.current_device()
    try:
        with open(os.path.join(_gpu_pci_dir(device), "local_cpulist")) as f:
            cpus = _parse_cpulist(f.read()) & os.sched_getaffinity(0)
        if cpus:
            return cpus
    except Exception:
        pass
    try:
        import pynvml
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(device)
        try:
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            h = pynvml.nvmlDeviceGetHandleByIndex(device)
        words = pynvml.nvmlDeviceGetCpuAffinity(h, 64)
        cpus = {64 * i + b for i, w in enumerate(words) for b in range(64) if (w >> b) & 1}
        cpus &= os.sched_getaffinity(0)
        return cpus or None
    except Exception:
        return None


def fma_peak(fp64=True):
    """FMA throughput of the current GPU in FLOP/s (cc_fma_peak): the
    denominator of the exact MPR stage's roofline."""
    v = ctypes.c_double()
    st = lib.cc_fma_peak(int(bool(fp64)), ctypes.byref(v), _stream())
    if st != _lib.CC_OK:
        raise CollideError(st, "cc_fma_peak")
    return float(v.value)


class numa_local:
    """Context manager: the calling thread runs on the GPU's NUMA node while
    host buffers are allocated (pinned pages are placed where they are first
    touched), then gets its old CPU set back."""

    def __init__(self, device=None):
        self.device = device

    def __enter__(self):
        self.old = os.sched_getaffinity(0)
        cpus = gpu_local_cpus(self.device)
        if cpus:
            os.sched_setaffinity(0, cpus)
        return self

    def __exit__(self, *exc):
        os.sched_setaffinity(0, self.old)
        return False


def _ptr(t, dtype=None, name="tensor"):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    return ctypes.c_void_p(t.data_ptr())


class Context:
    """A cc_ctx: scratch memory, search-grid tuning and error text for one device."""

    def __init__(self, device=None):
        if device is None:
            device = torch.cuda.current_device()
        self.device = int(device)
        h = ctypes.c_void_p()
        st = lib.cc_ctx_create(ctypes.byref(h), self.device)
        if st != _lib.CC_OK:
            raise CollideError(st, "cc_ctx_create")
        self.h = h

    def check(self, st, what=""):
        if st != _lib.CC_OK:
            raise CollideError(st, f"{what}: {lib.cc_last_error(self.h).decode()}")

    def set_search_grid(self, dims=(0, 0, 0)):
        self.check(lib.cc_set_search_grid(self.h, *[int(d) for d in dims]), "cc_set_search_grid")

    def set_tuning(self, cell_target=4.0, min_ratio=2.0):
        self.check(lib.cc_set_tuning(self.h, float(cell_target), float(min_ratio)), "cc_set_tuning")

    def set_incremental(self, on=True, margin=2.0):
        """Time steps of one scene test a kept candidate pair list, found on
        the boxes inflated by `margin` mean extents, while no box has moved
        more than half that since (cc_set_incremental); results are identical
        either way."""
        self.check(lib.cc_set_incremental(self.h, int(bool(on)), float(margin)), "cc_set_incremental")

    def set_static_shapes(self, on=True):
        """Host steps copy the shape arrays (T, A, B, C, R, ID) only when they
        are other arrays than last time; body poses are copied every step.
        Call again after changing shape arrays in place."""
        self.check(lib.cc_set_static_shapes(self.h, int(bool(on))), "cc_set_static_shapes")

    def last_step_rebuilt(self):
        return int(lib.cc_last_step_rebuilt(self.h))

    def set_dense_cell(self, entries=128):
        """Cells holding more entries go to the tiled dense-cell pair test
        (0: never)."""
        self.check(lib.cc_set_dense_cell(self.h, int(entries)), "cc_set_dense_cell")

    def narrowphase_overlap(self):
        return bool(getattr(self, "_np_overlap", True))

    def set_narrowphase_overlap(self, on=True):
        """Run cc_collide's MPR on the unsorted pairs while they are sorted
        (identical results)."""
        self.check(lib.cc_set_narrowphase_overlap(self.h, int(bool(on))), "cc_set_narrowphase_overlap")
        self._np_overlap = bool(on)

    def set_pair_test_shape(self, window=96, blocks_per_sm=8):
        """Launch shape of the sparse pair test: entries staged per warp (64,
        96, 128) and the grid cap in blocks per SM."""
        self.check(lib.cc_set_pair_test_shape(self.h, int(window), int(blocks_per_sm)), "cc_set_pair_test_shape")

    def set_narrowphase_precision(self, mode="exact"):
        """"exact" (default): the reference's MPR arithmetic in FP64, equal to
        the FP64 oracle up to float rounding of the outputs; "fp64": FP64 in a
        pair-local frame with FMA; "mixed": FP32 support maps."""
        self.check(lib.cc_set_narrowphase_precision(self.h, {"exact": 0, "fp64": 1, "mixed": 2}[mode]),
                   "cc_set_narrowphase_precision")

    def last_grid(self):
        dims = (ctypes.c_int * 3)()
        e = ctypes.c_uint64()
        lib.cc_get_last_grid(self.h, dims, ctypes.byref(e))
        return tuple(dims), int(e.value)

    def launches(self):
        return int(lib.cc_last_launch_count(self.h))

    def set_graph_replay(self, on=True):
        """Replay cc_collide as one CUDA graph once a configuration repeats
        (default on; results are identical)."""
        self.check(lib.cc_set_graph_replay(self.h, int(bool(on))), "cc_set_graph_replay")

    def set_profiling(self, on=True, spans=False):
        """Stage timing: every kernel stage (on), or with spans=True only the
        broadphase and narrowphase spans of an in-order cc_collide step."""
        self.check(lib.cc_set_profiling(self.h, (2 if spans else 1) if on else 0), "cc_set_profiling")

    def reset_stage_times(self):
        lib.cc_reset_stage_times(self.h)

    def stage_times(self):
        """{stage: (total device ms, launches)} accumulated while profiling."""
        k = lib.cc_stage_count()
        ms = (ctypes.c_double * k)()
        nl = (ctypes.c_uint64 * k)()
        lib.cc_stage_times(self.h, ms, nl, k)
        return {lib.cc_stage_name(i).decode(): (float(ms[i]), int(nl[i])) for i in range(k) if nl[i]}

    def close(self):
        if getattr(self, "h", None):
            lib.cc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_context(device=None) -> Context:
    if device is None:
        device = torch.cuda.current_device()
    if device not in _default_ctx:
        _default_ctx[device] = Context(device)
    return _default_ctx[device]


class DeviceScene:
    """A scene (collide_b200.scenes.Scene) resident in device memory."""

    def __init__(self, scene, device="cuda"):
        self.n, self.nb = scene.n, scene.nb
        to = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(device)  # noqa: E731
        self.T = to(scene.T, np.int32)
        self.A = to(scene.A, np.float32)
        self.B = to(scene.B, np.float32)
        self.C = to(scene.C, np.float32)
        self.R = to(scene.R, np.float32)
        self.ID = to(np.ascontiguousarray(scene.ID, dtype=np.uint32).view(np.int32), np.int32)  # uint32 bits
        self.pos = to(scene.pos, np.float32)
        self.rot = to(scene.rot, np.float32)
        self.active = to(scene.active, np.uint8)

    def arrays(self):
        return (self.T, self.A, self.B, self.C, self.R, self.ID, self.pos, self.rot)

    def c_scene(self):
        c = getattr(self, "_c", None)
        if c is not None:  # the tensors are only ever updated in place
            return c
        s = _lib.Scene()
        s.n, s.nb = self.n, self.nb
        s.T, s.A, s.B, s.C = self.T.data_ptr(), self.A.data_ptr(), self.B.data_ptr(), self.C.data_ptr()
        s.R, s.ID = self.R.data_ptr(), self.ID.data_ptr()
        s.body_pos, s.body_rot, s.active = self.pos.data_ptr(), self.rot.data_ptr(), self.active.data_ptr()
        self._c = s
        return s


class AABBGenerator:
    """AABBGenerator (src/aabb/AABBGenerator.cuh:14-49)."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()

    def GenerateAABB(self, T, A, B, C, R, ID, body_pos, body_rot, aabb_data=None):
        n = int(T.shape[0])
        if aabb_data is None or aabb_data.numel() != 6 * n:
            aabb_data = torch.zeros((2 * n, 3), dtype=torch.float32, device=T.device)
        st = lib.cc_generate_aabb(self.ctx.h, n, _ptr(T, torch.int32, "T"), _ptr(A, torch.float32, "A"),
                                  _ptr(B, torch.float32, "B"), _ptr(C, torch.float32, "C"),
                                  _ptr(R, torch.float32, "R"), _ptr(ID, None, "ID"), int(body_pos.shape[0]),
                                  _ptr(body_pos, torch.float32, "body_pos"), _ptr(body_rot, torch.float32, "body_rot"),
                                  _ptr(aabb_data, torch.float32, "aabb_data"), _stream())
        self.ctx.check(st, "GenerateAABB")
        return aabb_data


class Broadphase:
    """Broadphase (src/broadphase/Broadphase.cuh:14-82)."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.grid_size = (16, 16, 16)           # Broadphase.cu:37
        self.min_body_per_bin, self.max_body_per_bin = 25, 50   # :38-39
        self.parallel = (1, 0, 1, 0, 0, 0, 0, 0, 1, 0)          # :40
        self.number_of_contacts_possible = 0

    def setBinsPerAxis(self, binsPerAxis):
        self.grid_size = tuple(int(v) for v in binsPerAxis)
        return 0

    def getBinsPerAxis(self):
        return self.grid_size

    def setBodyPerBin(self, max_, min_):
        self.max_body_per_bin, self.min_body_per_bin = int(max_), int(min_)
        return 0

    def getMaxBodyPerBin(self):
        return self.max_body_per_bin

    def getMinBodyPerBin(self):
        return self.min_body_per_bin

    def getNumPossibleContacts(self):
        return self.number_of_contacts_possible

    def setParallelConfiguration(self, *flags):
        if len(flags) != 10:
            raise ValueError("setParallelConfiguration takes 10 flags")
        self.parallel = tuple(int(bool(f)) for f in flags)

    def getParallelConfiguration(self):
        return self.parallel

    def detectPossibleCollisions(self, aabb_data):
        """Shifts aabb_data ((2N,3) float32, CUDA) in place and returns the
        sorted unique int64 pair keys."""
        n = int(aabb_data.shape[0]) // 2
        # capacity: the previous call's pair count with some slack, so a
        # steady scene needs one library call (else cc_broadphase_fetch)
        cap = max(1024, n // 4, self.number_of_contacts_possible + self.number_of_contacts_possible // 16)
        out = torch.empty(cap, dtype=torch.int64, device=aabb_data.device)
        np_ = ctypes.c_uint64()
        st = lib.cc_broadphase(self.ctx.h, n, _ptr(aabb_data, torch.float32, "aabb_data"), *self.grid_size,
                               _ptr(out), cap, ctypes.byref(np_), _stream())
        if st == _lib.CC_ERR_CAPACITY:
            out = torch.empty(int(np_.value), dtype=torch.int64, device=aabb_data.device)
            st = lib.cc_broadphase_fetch(self.ctx.h, _ptr(out), int(np_.value), _stream())
        self.ctx.check(st, "detectPossibleCollisions")
        self.number_of_contacts_possible = int(np_.value)
        return out[: self.number_of_contacts_possible]

    def bins(self, aabb_data):
        """The reference's internal sorted bin list at the current bins per
        axis (Broadphase.cu:394-480); shifts aabb_data in place."""
        n = int(aabb_data.shape[0]) // 2
        ne, na = ctypes.c_uint64(), ctypes.c_uint64()
        probe = aabb_data.clone()
        st = lib.cc_broadphase_bins(self.ctx.h, n, _ptr(probe), *self.grid_size, None, None, 0, ctypes.byref(ne),
                                    None, None, 0, ctypes.byref(na), _stream())
        self.ctx.check(st, "bins (size)")
        dev = aabb_data.device
        bn = torch.empty(int(ne.value), dtype=torch.int32, device=dev)
        bd = torch.empty_like(bn)
        ab = torch.empty(int(na.value), dtype=torch.int32, device=dev)
        be = torch.empty_like(ab)
        st = lib.cc_broadphase_bins(self.ctx.h, n, _ptr(aabb_data), *self.grid_size, _ptr(bn), _ptr(bd),
                                    int(ne.value), ctypes.byref(ne), _ptr(ab), _ptr(be), int(na.value),
                                    ctypes.byref(na), _stream())
        self.ctx.check(st, "bins")
        return dict(bin_number=bn, body_number=bd, active_bins=ab, bin_end=be)


class Narrowphase:
    """Narrowphase (src/narrowphase/Narrowphase.cuh:13-63)."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.collision_envelope = 0.0   # Narrowphase.cu:505-509

    def SetCollisionEnvelope(self, envelope):
        self.collision_envelope = float(envelope)

    def GetCollisionEnvelope(self):
        return self.collision_envelope

    def DoNarrowphase(self, T, A, B, C, R, ID, obj_active, body_pos, body_rot, potentialCollisions):
        """Returns (norm, cpta, cptb, depth, bids, number_of_contacts); the
        first number_of_contacts rows are valid. potentialCollisions is
        permuted in place (contacts' pairs first)."""
        P_ = int(potentialCollisions.shape[0])
        dev = T.device
        norm = torch.empty((max(P_, 1), 3), dtype=torch.float32, device=dev)
        cpta = torch.empty_like(norm)
        cptb = torch.empty_like(norm)
        depth = torch.empty(max(P_, 1), dtype=torch.float32, device=dev)
        bids = torch.empty((max(P_, 1), 2), dtype=torch.int32, device=dev)
        nc = ctypes.c_uint64()
        st = lib.cc_narrowphase(self.ctx.h, int(T.shape[0]), _ptr(T, torch.int32, "T"), _ptr(A), _ptr(B), _ptr(C),
                                _ptr(R), _ptr(ID), int(body_pos.shape[0]), _ptr(obj_active, torch.uint8, "obj_active"),
                                _ptr(body_pos), _ptr(body_rot), float(self.collision_envelope),
                                _ptr(potentialCollisions, torch.int64, "potentialCollisions"), P_, _ptr(norm),
                                _ptr(cpta), _ptr(cptb), _ptr(depth), _ptr(bids), ctypes.byref(nc), _stream())
        self.ctx.check(st, "DoNarrowphase")
        k = int(nc.value)
        return norm[:k], cpta[:k], cptb[:k], depth[:k], bids[:k], k


def collide(ds: DeviceScene, grid=(16, 16, 16), envelope=0.0, ctx: Context | None = None, pairs_cap=None,
            aabb=None):
    """GenerateAABB -> detectPossibleCollisions -> DoNarrowphase on a device
    scene (cc_collide). Returns a dict of device tensors."""
    ctx = ctx or default_context()
    dev = ds.T.device
    if aabb is None:
        aabb = torch.zeros((2 * ds.n, 3), dtype=torch.float32, device=dev)
    # a call whose pair output was too small has already shifted `aabb` in
    # place: the retry starts again from the caller's boxes (those of RECT and
    # TRIANGLEMESH shapes are not regenerated)
    aabb_in = aabb.clone()
    cap = int(pairs_cap or max(1024, ds.n // 4))
    first = True
    while True:
        if not first:
            aabb.copy_(aabb_in)
        first = False
        pairs = torch.empty(cap, dtype=torch.int64, device=dev)
        norm = torch.empty((cap, 3), dtype=torch.float32, device=dev)
        cpta, cptb = torch.empty_like(norm), torch.empty_like(norm)
        depth = torch.empty(cap, dtype=torch.float32, device=dev)
        bids = torch.empty((cap, 2), dtype=torch.int32, device=dev)
        res = _lib.Result()
        res.aabb, res.pairs, res.pairs_cap = aabb.data_ptr(), pairs.data_ptr(), cap
        res.norm, res.cpta, res.cptb = norm.data_ptr(), cpta.data_ptr(), cptb.data_ptr()
        res.depth, res.bids = depth.data_ptr(), bids.data_ptr()
        sc = ds.c_scene()
        st = lib.cc_collide(ctx.h, ctypes.byref(sc), *[int(g) for g in grid], float(envelope), ctypes.byref(res),
                            _stream())
        if st == _lib.CC_ERR_CAPACITY and res.n_pairs > cap:
            cap = int(res.n_pairs)
            continue
        ctx.check(st, "cc_collide")
        P_, k = int(res.n_pairs), int(res.n_contacts)
        return dict(aabb=aabb, pairs=pairs[:P_], contact_pairs=pairs[:k], norm=norm[:k], cpta=cpta[:k],
                    cptb=cptb[:k], depth=depth[:k], bids=bids[:k], n_pairs=P_, n_contacts=k)


class HostSession:
    """End-to-end use from host memory (cc_collide_host): the scene lives in
    pinned host buffers (pageable ones with pinned=False); every run() copies
    it to the device, runs the pipeline and copies pairs and contacts back into
    pinned host buffers."""

    def __init__(self, scene, grid=(16, 16, 16), envelope=0.0, ctx: Context | None = None, pairs_cap=None,
                 want_aabb=False, pinned=True):
        self.ctx = ctx or default_context()
        self.grid, self.envelope = tuple(int(g) for g in grid), float(envelope)
        self.pinned = bool(pinned)
        # the count of shapes whose third array (C) the device reads: CONE and TRIANGLEMESH
        self.c_shapes = int(np.count_nonzero((np.asarray(scene.T) == 5) | (np.asarray(scene.T) == 6)))

        def pin(a, dt):
            t = torch.from_numpy(np.ascontiguousarray(a, dtype=dt))
            return t.pin_memory() if self.pinned else t.clone()
        self.n, self.nb = scene.n, scene.nb
        self.want_aabb = want_aabb
        self.n_pairs = self.n_contacts = 0
        with numa_local(self.ctx.device):  # pinned buffers on the GPU's node
            self.inputs = [pin(scene.T, np.int32), pin(scene.A, np.float32), pin(scene.B, np.float32),
                           pin(scene.C, np.float32), pin(scene.R, np.float32),
                           pin(np.ascontiguousarray(scene.ID, dtype=np.uint32).view(np.int32), np.int32),
                           pin(scene.pos, np.float32), pin(scene.rot, np.float32), pin(scene.active, np.uint8)]
            self._alloc(int(pairs_cap or max(1024, self.n // 4)))

    def _alloc(self, cap):
        self.cap = cap
        e = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True)  # noqa: E731
        if getattr(self, "aabb", None) is None:  # kept on regrowth: it holds the caller's input boxes
            self.aabb = e((2 * self.n, 3), torch.float32) if self.want_aabb else None
        self.pairs = e(cap, torch.int64)
        self.norm, self.cpta, self.cptb = (e((cap, 3), torch.float32), e((cap, 3), torch.float32),
                                           e((cap, 3), torch.float32))
        self.depth = e(cap, torch.float32)
        self.bids = e((cap, 2), torch.int32)

    def input_bytes(self, poses_only=False):
        """Host-to-device bytes of one step: every input array, or with static
        shapes (Context.set_static_shapes) the body poses and flags alone. From
        pinned buffers the library reads C only for the CONE and TRIANGLEMESH
        shapes (12 bytes each), so only those bytes of C count."""
        if poses_only:
            return int(sum(t.numel() * t.element_size() for t in self.inputs[6:]))
        total = int(sum(t.numel() * t.element_size() for t in self.inputs))
        if self.pinned:
            total -= self.inputs[3].numel() * self.inputs[3].element_size() - 12 * self.c_shapes
        return total

    def output_bytes(self):
        k = self.n_contacts
        return 8 * self.n_pairs + k * (12 * 3 + 4 + 8) + (24 * self.n if self.aabb is not None else 0)

    def run(self):
        while True:
            T, A, B, C, R, ID, pos, rot, act = self.inputs
            sc = _lib.Scene()
            sc.n, sc.nb = self.n, self.nb
            sc.T, sc.A, sc.B, sc.C, sc.R, sc.ID = (T.data_ptr(), A.data_ptr(), B.data_ptr(), C.data_ptr(),
                                                    R.data_ptr(), ID.data_ptr())
            sc.body_pos, sc.body_rot, sc.active = pos.data_ptr(), rot.data_ptr(), act.data_ptr()
            res = _lib.Result()
            res.aabb = self.aabb.data_ptr() if self.aabb is not None else None
            res.pairs, res.pairs_cap = self.pairs.data_ptr(), self.cap
            res.norm, res.cpta, res.cptb = self.norm.data_ptr(), self.cpta.data_ptr(), self.cptb.data_ptr()
            res.depth, res.bids = self.depth.data_ptr(), self.bids.data_ptr()
            st = lib.cc_collide_host(self.ctx.h, ctypes.byref(sc), *self.grid, self.envelope, ctypes.byref(res),
                                     _stream())
            if st == _lib.CC_ERR_CAPACITY and res.n_pairs > self.cap:
                self._alloc(int(res.n_pairs * 5 // 4))
                continue
            self.ctx.check(st, "cc_collide_host")
            self.n_pairs, self.n_contacts = int(res.n_pairs), int(res.n_contacts)
            return self.n_pairs, self.n_contacts

    # -- pipelined steps: submit() returns at once, wait() finishes the oldest
    def _structs(self):
        T, A, B, C, R, ID, pos, rot, act = self.inputs
        sc = _lib.Scene()
        sc.n, sc.nb = self.n, self.nb
        sc.T, sc.A, sc.B, sc.C, sc.R, sc.ID = (T.data_ptr(), A.data_ptr(), B.data_ptr(), C.data_ptr(),
                                                R.data_ptr(), ID.data_ptr())
        sc.body_pos, sc.body_rot, sc.active = pos.data_ptr(), rot.data_ptr(), act.data_ptr()
        res = _lib.Result()
        res.aabb = self.aabb.data_ptr() if self.aabb is not None else None
        res.pairs, res.pairs_cap = self.pairs.data_ptr(), self.cap
        res.norm, res.cpta, res.cptb = self.norm.data_ptr(), self.cpta.data_ptr(), self.cptb.data_ptr()
        res.depth, res.bids = self.depth.data_ptr(), self.bids.data_ptr()
        # the structs and the buffers they point at stay alive while a step uses them
        keep = (self.aabb, self.pairs, self.norm, self.cpta, self.cptb, self.depth, self.bids)
        self._cur = (sc, res, keep)

    def submit(self):
        """cc_collide_host_submit: enqueue one step (at most two in flight).
        The host inputs must stay unchanged until the step's wait()."""
        if getattr(self, "_cur", None) is None:
            self._structs()
        if not hasattr(self, "_pending"):
            self._pending = []
        sc, res, keep = self._cur
        self.ctx.check(lib.cc_collide_host_submit(self.ctx.h, ctypes.byref(sc), *self.grid, self.envelope,
                                                  ctypes.byref(res), _stream()), "cc_collide_host_submit")
        self._pending.append(self._cur)

    def wait(self):
        """cc_collide_host_wait: finish the oldest submitted step; its pairs
        and contacts are in this session's host buffers until the next wait."""
        sc, res, keep = self._pending.pop(0)
        st = lib.cc_collide_host_wait(self.ctx.h, ctypes.byref(res), _stream())
        if st == _lib.CC_ERR_CAPACITY and res.n_pairs > res.pairs_cap:
            # larger buffers for the steps to come; this one runs again blocking
            if res.n_pairs > self.cap:
                self._alloc(int(res.n_pairs) * 5 // 4)
                self._cur = None
            return self.run()
        self.ctx.check(st, "cc_collide_host_wait")
        self.n_pairs, self.n_contacts = int(res.n_pairs), int(res.n_contacts)
        return self.n_pairs, self.n_contacts


def collide_host(scene, grid=(16, 16, 16), envelope=0.0, ctx: Context | None = None):
    """One end-to-end call from host arrays; returns numpy results."""
    hs = HostSession(scene, grid, envelope, ctx, want_aabb=True)
    P_, k = hs.run()
    return dict(aabb=hs.aabb.numpy().copy(), pairs=hs.pairs[:P_].numpy().copy(), n_pairs=P_, n_contacts=k,
                norm=hs.norm[:k].numpy().copy(), cpta=hs.cpta[:k].numpy().copy(), cptb=hs.cptb[:k].numpy().copy(),
                depth=hs.depth[:k].numpy().copy(), bids=hs.bids[:k].numpy().copy(),
                contact_pairs=hs.pairs[:k].numpy().copy())


class DevicePipeline:
    """cc_collide on a device-resident scene with preallocated outputs: run()
    is one GenerateAABB -> detectPossibleCollisions -> DoNarrowphase step."""

    def __init__(self, ds: DeviceScene, grid=(16, 16, 16), envelope=0.0, ctx: Context | None = None, pairs_cap=None):
        self.ds, self.ctx = ds, ctx or default_context()
        self.grid, self.envelope = tuple(int(g) for g in grid), float(envelope)
        self.aabb = torch.zeros((2 * ds.n, 3), dtype=torch.float32, device=ds.T.device)
        self.scene = ds.c_scene()
        self._alloc(int(pairs_cap or max(1024, ds.n // 4)))
        self.n_pairs = self.n_contacts = 0

    def _alloc(self, cap, dev=None):
        dev = dev or self.ds.T.device
        self.cap = cap
        self.pairs = torch.empty(cap, dtype=torch.int64, device=dev)
        self.norm = torch.empty((cap, 3), dtype=torch.float32, device=dev)
        self.cpta, self.cptb = torch.empty_like(self.norm), torch.empty_like(self.norm)
        self.depth = torch.empty(cap, dtype=torch.float32, device=dev)
        self.bids = torch.empty((cap, 2), dtype=torch.int32, device=dev)
        r = _lib.Result()
        r.aabb, r.pairs, r.pairs_cap = self.aabb.data_ptr(), self.pairs.data_ptr(), cap
        r.norm, r.cpta, r.cptb = self.norm.data_ptr(), self.cpta.data_ptr(), self.cptb.data_ptr()
        r.depth, r.bids = self.depth.data_ptr(), self.bids.data_ptr()
        self.res = r

    def run(self):
        while True:
            st = lib.cc_collide(self.ctx.h, ctypes.byref(self.scene), *self.grid, self.envelope,
                                ctypes.byref(self.res), _stream())
            if st == _lib.CC_ERR_CAPACITY and self.res.n_pairs > self.cap:
                self._alloc(int(self.res.n_pairs * 5 // 4))
                continue
            self.ctx.check(st, "cc_collide")
            self.n_pairs, self.n_contacts = int(self.res.n_pairs), int(self.res.n_contacts)
            return self.n_pairs, self.n_contacts


class DeviceBatch:
    """Independent scenes resident on the device as one concatenated scene
    (cc_batch): shapes [shape_offsets[s], shape_offsets[s+1]) and bodies
    [body_offsets[s], body_offsets[s+1]) belong to scene s."""

    def __init__(self, scenes, device="cuda"):
        from . import scenes as _sc
        cat, self.shape_offsets, self.body_offsets = _sc.concat(list(scenes))
        self.ds = DeviceScene(cat, device=device)
        self.num_scenes = len(self.shape_offsets) - 1
        self.n, self.nb = self.ds.n, self.ds.nb

    def c_batch(self):
        b = _lib.Batch()
        b.num_scenes = self.num_scenes
        b.shape_offsets = self.shape_offsets.ctypes.data
        b.body_offsets = self.body_offsets.ctypes.data
        b.scene = self.ds.c_scene()
        return b


class BatchPipeline:
    """cc_collide_batch with preallocated outputs: run() collides every scene
    of a DeviceBatch in one pass. After run(): scene_pairs[s] pairs and
    contacts [contact_offsets[s], contact_offsets[s+1]) for scene s; pair keys
    and bids use the concatenated numbering."""

    def __init__(self, db: DeviceBatch, grid=(16, 16, 16), envelope=0.0, ctx: Context | None = None, pairs_cap=None):
        self.db, self.ds, self.ctx = db, db.ds, ctx or default_context()
        self.grid, self.envelope = tuple(int(g) for g in grid), float(envelope)
        dev = db.ds.T.device
        self.aabb = torch.zeros((2 * db.n, 3), dtype=torch.float32, device=dev)
        self.batch = db.c_batch()
        self.scene_pairs = np.zeros(db.num_scenes, np.uint64)
        self.contact_offsets = np.zeros(db.num_scenes + 1, np.uint64)
        self._alloc(int(pairs_cap or max(1024, db.n // 4)))
        self.n_pairs = self.n_contacts = 0

    _alloc = DevicePipeline._alloc

    def run(self):
        while True:
            st = lib.cc_collide_batch(self.ctx.h, ctypes.byref(self.batch), *self.grid, self.envelope,
                                      ctypes.byref(self.res), self.scene_pairs.ctypes.data,
                                      self.contact_offsets.ctypes.data, _stream())
            if st == _lib.CC_ERR_CAPACITY and self.res.n_pairs > self.cap:
                self._alloc(int(self.res.n_pairs * 5 // 4))
                continue
            self.ctx.check(st, "cc_collide_batch")
            self.n_pairs, self.n_contacts = int(self.res.n_pairs), int(self.res.n_contacts)
            return self.n_pairs, self.n_contacts


def collide_batch(db: DeviceBatch, grid=(16, 16, 16), envelope=0.0, ctx: Context | None = None, pairs_cap=None):
    """cc_collide_batch once; returns device tensors (concatenated numbering)
    plus per-scene pair counts and contact offsets (numpy)."""
    bp = BatchPipeline(db, grid, envelope, ctx, pairs_cap)
    P, k = bp.run()
    return dict(aabb=bp.aabb, pairs=bp.pairs[:P], contact_pairs=bp.pairs[:k], norm=bp.norm[:k], cpta=bp.cpta[:k],
                cptb=bp.cptb[:k], depth=bp.depth[:k], bids=bp.bids[:k], n_pairs=P, n_contacts=k,
                scene_pairs=bp.scene_pairs.copy(), contact_offsets=bp.contact_offsets.copy())


class ScenesPipeline:
    """cc_collide_scenes: one batched pass over scenes that stay in their own
    device allocations (a list of DeviceScene). Outputs as BatchPipeline, in
    the concatenated numbering of the list's order."""

    def __init__(self, ctx: Context | None = None, grid=(16, 16, 16), envelope=0.0, pairs_cap=1 << 16):
        self.ctx = ctx or default_context()
        self.grid, self.envelope = tuple(int(g) for g in grid), float(envelope)
        self.cap = 0
        self.aabb = None
        self._want_cap = int(pairs_cap)
        self.n_pairs = self.n_contacts = 0

    _alloc = DevicePipeline._alloc

    def run(self, scenes):
        k = len(scenes)
        arr = (_lib.Scene * max(k, 1))()
        for i, d in enumerate(scenes):
            arr[i] = d.c_scene()
        n = sum(d.n for d in scenes)
        dev = scenes[0].T.device if k else torch.device("cuda")
        if self.aabb is None or self.aabb.shape[0] < 2 * n:
            self.aabb = torch.empty((max(2 * n, 2), 3), dtype=torch.float32, device=dev)
        if self.cap < self._want_cap:
            self._alloc(self._want_cap, dev)
        self.res.aabb = self.aabb.data_ptr()
        self.scene_pairs = np.zeros(max(k, 1), np.uint64)
        self.contact_offsets = np.zeros(k + 1, np.uint64)
        while True:
            st = lib.cc_collide_scenes(self.ctx.h, k, arr, *self.grid, self.envelope, ctypes.byref(self.res),
                                       self.scene_pairs.ctypes.data, self.contact_offsets.ctypes.data, _stream())
            if st == _lib.CC_ERR_CAPACITY and self.res.n_pairs > self.cap:
                self._alloc(int(self.res.n_pairs * 5 // 4), dev)
                self.res.aabb = self.aabb.data_ptr()
                continue
            self.ctx.check(st, "cc_collide_scenes")
            self.n_pairs, self.n_contacts = int(self.res.n_pairs), int(self.res.n_contacts)
            return self.n_pairs, self.n_contacts
