"""ctypes binding of libcollide_b200.so (the C ABI in include/collide_b200.h).

The library is built in-tree by ``make -C collision-detection_b200`` (or
``__graft_entry__.build()``). There is no fallback: importing this module
without the built library raises ImportError.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcollide_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `make -C collision-detection_b200`")

P = ctypes.c_void_p
U64 = ctypes.c_uint64
I32 = ctypes.c_int
F32 = ctypes.c_float
PU64 = ctypes.POINTER(ctypes.c_uint64)

lib = ctypes.CDLL(LIB_PATH)

CC_OK = 0
STATUS = {
    0: "CC_OK",
    1: "CC_ERR_INVALID_ARGUMENT",
    2: "CC_ERR_INVALID_INPUT",
    3: "CC_ERR_CAPACITY",
    4: "CC_ERR_CUDA",
    5: "CC_ERR_OUT_OF_MEMORY",
    6: "CC_ERR_INTERNAL",
    7: "CC_ERR_NO_RESULT",
}
CC_ERR_CAPACITY = 3

#: Every function the C header declares, with (restype, argtypes).
SIGNATURES = {
    "cc_ctx_create": (I32, [ctypes.POINTER(P), I32]),
    "cc_ctx_destroy": (None, [P]),
    "cc_status_string": (ctypes.c_char_p, [I32]),
    "cc_last_error": (ctypes.c_char_p, [P]),
    "cc_version": (ctypes.c_char_p, []),
    "cc_set_search_grid": (I32, [P, I32, I32, I32]),
    "cc_set_tuning": (I32, [P, F32, F32]),
    "cc_set_dense_cell": (I32, [P, ctypes.c_uint32]),
    "cc_set_pair_test_shape": (I32, [P, I32, I32]),
    "cc_set_narrowphase_overlap": (I32, [P, I32]),
    "cc_set_incremental": (I32, [P, I32, F32]),
    "cc_set_static_shapes": (I32, [P, I32]),
    "cc_last_step_rebuilt": (I32, [P]),
    "cc_set_narrowphase_precision": (I32, [P, I32]),
    "cc_get_last_grid": (I32, [P, ctypes.POINTER(ctypes.c_int), PU64]),
    "cc_generate_aabb": (I32, [P, U64, P, P, P, P, P, P, U64, P, P, P, P]),
    "cc_broadphase": (I32, [P, U64, P, I32, I32, I32, P, U64, PU64, P]),
    "cc_broadphase_fetch": (I32, [P, P, U64, P]),
    "cc_broadphase_bins": (I32, [P, U64, P, I32, I32, I32, P, P, U64, PU64, P, P, U64, PU64, P]),
    "cc_narrowphase": (I32, [P, U64, P, P, P, P, P, P, U64, P, P, P, F32, P, U64, P, P, P, P, P, PU64, P]),
    "cc_collide": (I32, [P, P, I32, I32, I32, F32, P, P]),
    "cc_collide_host": (I32, [P, P, I32, I32, I32, F32, P, P]),
    "cc_collide_host_submit": (I32, [P, P, I32, I32, I32, F32, P, P]),
    "cc_collide_host_wait": (I32, [P, P, P]),
    "cc_collide_batch": (I32, [P, P, I32, I32, I32, F32, P, P, P, P]),
    "cc_collide_scenes": (I32, [P, U64, P, I32, I32, I32, F32, P, P, P, P]),
    "cc_perturb_bodies": (I32, [P, U64, P, P, U64, F32, F32, P]),
    "cc_last_launch_count": (U64, [P]),
    "cc_set_profiling": (I32, [P, I32]),
    "cc_set_graph_replay": (I32, [P, I32]),
    "cc_stage_count": (I32, []),
    "cc_stage_name": (ctypes.c_char_p, [I32]),
    "cc_stage_times": (I32, [P, ctypes.POINTER(ctypes.c_double), PU64, I32]),
    "cc_reset_stage_times": (I32, [P]),
    "cc_broadphase_noalloc": (I32, [U64, P, I32, I32, I32, P, U64, PU64, P]),
    "cc_fma_peak": (I32, [I32, ctypes.POINTER(ctypes.c_double), P]),
    "cc_perturb_scenes": (I32, [P, U64, P, P, P, P, F32, F32, P]),
}

for _name, (_res, _args) in SIGNATURES.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


class Scene(ctypes.Structure):
    """struct cc_scene."""
    _fields_ = [("n", U64), ("T", P), ("A", P), ("B", P), ("C", P), ("R", P), ("ID", P), ("nb", U64),
                ("body_pos", P), ("body_rot", P), ("active", P)]


class Batch(ctypes.Structure):
    """struct cc_batch."""
    _fields_ = [("num_scenes", U64), ("shape_offsets", P), ("body_offsets", P), ("scene", Scene)]


class Result(ctypes.Structure):
    """struct cc_result."""
    _fields_ = [("aabb", P), ("pairs", P), ("pairs_cap", U64), ("norm", P), ("cpta", P), ("cptb", P),
                ("depth", P), ("bids", P), ("n_pairs", U64), ("n_contacts", U64)]


class CollideError(RuntimeError):
    def __init__(self, status, detail=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {detail}")


def version() -> str:
    return lib.cc_version().decode()
