"""ctypes binding of the C ABI in include/avbd_cuda.h (libavbd_cuda.so, built in-tree).

The product path has no fallback: if the CUDA library is missing or no GPU is present,
loading raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libavbd_cuda.so")

AVBD_OK = 0
AVBD_ERR_ARGUMENT, AVBD_ERR_CUDA, AVBD_ERR_CAPACITY, AVBD_ERR_STATE, AVBD_ERR_LATCHED = -1, -2, -3, -4, -5
ERRORS = {-1: "argument", -2: "cuda", -3: "capacity", -4: "state", -5: "latched"}

c_float_p = ctypes.POINTER(ctypes.c_float)
c_int_p = ctypes.POINTER(ctypes.c_int32)
c_i64_p = ctypes.POINTER(ctypes.c_int64)


class AvbdParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_float), ("gravity", ctypes.c_float), ("iterations", ctypes.c_int32),
                ("alpha", ctypes.c_float), ("betaLin", ctypes.c_float), ("betaAng", ctypes.c_float),
                ("gamma", ctypes.c_float), ("broadphase", ctypes.c_int32)]


class AvbdBodies(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32)] + [(k, ctypes.c_void_p) for k in (
        "position3", "orientation4", "velocity3", "angular3", "prev_velocity3", "size3", "mass", "moment3",
        "friction", "radius", "shape", "shape_radius", "half_length")]


class AvbdBodyState(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in (
        "position3", "orientation4", "velocity3", "angular3", "prev_velocity3", "initial_position3",
        "initial_orientation4", "inertial_position3", "inertial_orientation4")]


class AvbdJoints(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32)] + [(k, ctypes.c_void_p) for k in ("body_ab2", "seq", "state28", "broken")]


class AvbdSprings(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32)] + [(k, ctypes.c_void_p) for k in ("body_ab2", "seq", "state8")]


class AvbdIgnores(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32)] + [(k, ctypes.c_void_p) for k in ("body_ab2", "seq")]


class AvbdManifolds(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32)] + [(k, ctypes.c_void_p) for k in (
        "body_ab2", "seq", "num_contacts", "basis9", "friction", "keys8", "contact15x8", "stick8")]


class AvbdManifoldsOut(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in (
        "body_ab2", "seq", "num_contacts", "basis9", "friction", "keys8", "contact15x8", "stick8")]


class AvbdJointsOut(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in ("body_ab2", "seq", "state28", "broken")]


class AvbdExternalContacts(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32)] + [(k, ctypes.c_void_p) for k in (
        "body_ab2", "num_contacts", "basis9", "keys8", "contact15x8", "stick8", "creates")]


class AvbdStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in (
        "body_count", "pair_checks", "sphere_hits", "constrained_hits", "manifolds_created", "manifold_count",
        "contact_count", "joint_count", "spring_count", "solved_bodies", "colours", "colour_rounds",
        "primal_rows", "grid_rescaled", "device_steps", "redone_steps")] + [("step_ms", ctypes.c_float)]


PHASES = ("broadphase", "force_init", "adjacency", "body_init", "colouring", "primal", "dual", "velocity")


class AvbdProfile(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int64), ("phase_ms", ctypes.c_double * len(PHASES)),
                ("phase_spans", ctypes.c_int64 * len(PHASES)), ("launches", ctypes.c_int64)]


class AvbdAdjointGrad(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in (
        "position", "orientation", "velocity", "angular_velocity", "prev_velocity", "mass", "pair_friction",
        "body_friction")]


# name -> (restype, argtypes); every symbol declared in include/avbd_cuda.h
SIGNATURES = {
    "avbd_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32, ctypes.c_void_p]),
    "avbd_destroy": (None, [ctypes.c_void_p]),
    "avbd_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "avbd_clear_error": (None, [ctypes.c_void_p]),
    "avbd_backend_name": (ctypes.c_char_p, []),
    "avbd_set_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AvbdParams)]),
    "avbd_load_world": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AvbdBodies), ctypes.POINTER(AvbdJoints),
                                       ctypes.POINTER(AvbdSprings), ctypes.POINTER(AvbdIgnores),
                                       ctypes.POINTER(AvbdManifolds), ctypes.c_int64]),
    "avbd_load_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, c_int_p, ctypes.POINTER(AvbdBodies),
                                       ctypes.POINTER(AvbdJoints), ctypes.POINTER(AvbdSprings),
                                       ctypes.POINTER(AvbdIgnores), ctypes.POINTER(AvbdManifolds), ctypes.c_int64]),
    "avbd_write_bodies": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AvbdBodies)]),
    "avbd_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "avbd_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "avbd_set_step_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "avbd_step_external": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, c_int_p,
                                          ctypes.POINTER(AvbdExternalContacts)]),
    "avbd_set_manifold_headroom": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    "avbd_set_wait_limits": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    "avbd_broadphase_only": (ctypes.c_int, [ctypes.c_void_p]),
    "avbd_read_bodies": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AvbdBodyState)]),
    "avbd_num_manifolds": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
    "avbd_read_manifolds": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AvbdManifoldsOut)]),
    "avbd_num_joints": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
    "avbd_read_joints": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AvbdJointsOut)]),
    "avbd_next_seq": (ctypes.c_int, [ctypes.c_void_p, c_i64_p]),
    "avbd_snapshot_binary": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, c_int_p,
                                            ctypes.c_void_p, ctypes.c_int64, c_i64_p]),
    "avbd_snapshot_json": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, c_int_p,
                                          ctypes.c_char_p, ctypes.c_int64, c_i64_p]),
    "avbd_set_iteration_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "avbd_iteration_mode": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
    "avbd_add_joints": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AvbdJoints)]),
    "avbd_remove_joints": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, c_i64_p]),
    "avbd_write_joints": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AvbdJoints)]),
    "avbd_read_colours": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p]),
    "avbd_read_solve_order": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p]),
    "avbd_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AvbdStats)]),
    "avbd_device_pose": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "avbd_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "avbd_set_colouring": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "avbd_colour_graph_noalloc": (ctypes.c_int, [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_int32, ctypes.c_void_p, c_int_p, ctypes.c_void_p]),
    "avbd_num_primal_variants": (ctypes.c_int, [c_int_p, c_int_p, c_int_p]),
    "avbd_set_primal_variant": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "avbd_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, c_int_p, c_float_p]),
    "avbd_read_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AvbdProfile)]),
    "avbd_reset_profile": (ctypes.c_int, [ctypes.c_void_p]),
    "avbd_adjoint_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    "avbd_adjoint_num_pairs": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
    "avbd_adjoint_read_pairs": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_float_p]),
    "avbd_adjoint_backward": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 4
                              + [ctypes.POINTER(AvbdAdjointGrad)]),
    "avbd_adjoint_replay_state": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 4),
    "avbd_adjoint_tape_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, c_int_p, ctypes.c_void_p,
                                              ctypes.c_void_p, c_int_p]),
}

_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libavbd_cuda.so and bind every exported symbol. Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library {path} is not built; run __graft_entry__.build() or "
                           f"python -m avbd_demo3d_b200.build")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class AvbdError(RuntimeError):
    pass
