"""ctypes front end for the CPU checkers (TEST INFRASTRUCTURE, not the product).

Two interchangeable backends with one interface:
  * ``kind="oracle"``: liboracle.so, the plain-C restatement of the reference step
  * ``kind="ref"``:    _ref/libavbd_ref.so, the reference solver compiled from its own
                      sources with a thin driver (built only where the reference exists;
                      the prebuilt library travels with the repository)

Only the tests, the smoke check and the benchmark's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes
import struct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libavbd_ref.so")
REF64_LIB = os.path.join(HERE, "_ref", "libavbd_ref64.so")

_libs: dict[str, ctypes.CDLL] = {}


class _Params(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_float), ("gravity", ctypes.c_float), ("iterations", ctypes.c_int),
                ("alpha", ctypes.c_float), ("betaLin", ctypes.c_float), ("betaAng", ctypes.c_float),
                ("gamma", ctypes.c_float), ("broadphase", ctypes.c_int), ("orderMode", ctypes.c_int)]


ORACLE_SOURCES = [os.path.join(HERE, f) for f in ("avbd_oracle.c", "avbd_oracle.h", "adjoint_ref.cpp")] + [
    os.path.join(HERE, "..", "avbd_demo3d_b200", "csrc", "avbd_diff.h")]


class _TapeStep(ctypes.Structure):
    _fields_ = [("nMan", ctypes.c_int), ("nSolve", ctypes.c_int), ("nColours", ctypes.c_int),
                ("iterations", ctypes.c_int), ("bodyIn", ctypes.POINTER(ctypes.c_float)),
                ("bodyFlags", ctypes.POINTER(ctypes.c_uint8)), ("ab", ctypes.POINTER(ctypes.c_int)),
                ("basis", ctypes.POINTER(ctypes.c_float)), ("friction", ctypes.POINTER(ctypes.c_float)),
                ("ncontacts", ctypes.POINTER(ctypes.c_int)), ("keys", ctypes.POINTER(ctypes.c_int)),
                ("geo", ctypes.POINTER(ctypes.c_float)), ("init", ctypes.POINTER(ctypes.c_float)),
                ("src", ctypes.POINTER(ctypes.c_int)), ("initFlags", ctypes.POINTER(ctypes.c_uint8)),
                ("solveOrder", ctypes.POINTER(ctypes.c_int)), ("colourStart", ctypes.POINTER(ctypes.c_int)),
                ("flags", ctypes.POINTER(ctypes.c_uint16))]


def build_oracle() -> str:
    """Compile liboracle.so if missing or stale (gcc/g++ only; works on any box)."""
    newest = max(os.path.getmtime(f) for f in ORACLE_SOURCES if os.path.exists(f))
    if not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < newest:
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return ORACLE_LIB


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref64_available() -> bool:
    return os.path.exists(REF64_LIB)


def _lib(kind: str) -> ctypes.CDLL:
    if kind in _libs:
        return _libs[kind]
    if kind == "oracle":
        lib = ctypes.CDLL(build_oracle())
        p = "oracle_"
    elif kind == "ref":
        if not ref_available():
            raise FileNotFoundError(f"{REF_LIB} not built (needs the reference sources: make -C oracle ref)")
        lib = ctypes.CDLL(REF_LIB)
        p = "ref_"
    else:
        raise ValueError(kind)
    vp, ip, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p
    getattr(lib, p + "create").restype = vp
    getattr(lib, p + "create").argtypes = [ctypes.POINTER(_Params), ip] + [fp] * 6 + [ip] + [fp] * 6
    getattr(lib, p + "create_shapes").restype = vp
    getattr(lib, p + "create_shapes").argtypes = [ctypes.POINTER(_Params), ip, fp, fp] + [fp] * 6 + [ip] + [fp] * 6
    for name in ("destroy",):
        getattr(lib, p + name).argtypes = [vp]
        getattr(lib, p + name).restype = None
    for name in ("prepare", "iterate", "finish", "num_bodies", "num_manifolds", "num_joints", "broadphase_only"):
        getattr(lib, p + name).argtypes = [vp]
        getattr(lib, p + name).restype = ip
    if p == "ref_":
        lib.ref_world_bodies.argtypes = [vp] + [ctypes.c_void_p] * 9
        lib.ref_world_bodies.restype = ip
    getattr(lib, p + "add_joint").argtypes = [vp, ip, ip, fp, fp, ctypes.c_float, ctypes.c_float, ctypes.c_float]
    getattr(lib, p + "add_joint").restype = ctypes.c_int64
    getattr(lib, p + "set_joint_anchor").argtypes = [vp, ctypes.c_int64, fp]
    getattr(lib, p + "set_joint_anchor").restype = ip
    getattr(lib, p + "remove_joint").argtypes = [vp, ctypes.c_int64]
    getattr(lib, p + "remove_joint").restype = ip
    getattr(lib, p + "step").argtypes = [vp, ip]
    getattr(lib, p + "step").restype = ip
    getattr(lib, p + "set_params").argtypes = [vp, ctypes.POINTER(_Params)]
    getattr(lib, p + "set_params").restype = None
    getattr(lib, p + "get_bodies").argtypes = [vp] + [fp] * 5
    getattr(lib, p + "get_bodies").restype = None
    getattr(lib, p + "get_body_props").argtypes = [vp] + [fp] * 5
    getattr(lib, p + "get_body_props").restype = None
    getattr(lib, p + "get_manifolds").argtypes = [vp] + [fp] * 8
    getattr(lib, p + "get_manifolds").restype = None
    getattr(lib, p + "get_joints").argtypes = [vp] + [fp] * 3
    getattr(lib, p + "get_joints").restype = None
    getattr(lib, p + "get_counters").argtypes = [vp, fp]
    getattr(lib, p + "get_counters").restype = None
    getattr(lib, p + "collide_boxes").argtypes = [fp] * 10
    getattr(lib, p + "collide_boxes").restype = ip
    if kind == "oracle":
        lib.oracle_get_colours.argtypes = [vp, fp, fp]
        lib.oracle_get_colours.restype = None
        lib.oracle_get_solve_order.argtypes = [vp, fp]
        lib.oracle_get_solve_order.restype = ip
        lib.oracle_get_body_aux.argtypes = [vp] + [fp] * 4
        lib.oracle_get_body_aux.restype = None
        lib.oracle_set_bodies.argtypes = [vp] + [fp] * 5
        lib.oracle_set_bodies.restype = None
        lib.oracle_colour_priority.argtypes = [ctypes.c_uint32]
        lib.oracle_colour_priority.restype = ctypes.c_uint32
        lib.oracle_tape_begin.argtypes = [vp]
        lib.oracle_tape_begin.restype = ip
        lib.oracle_tape_end.argtypes = [vp]
        lib.oracle_tape_end.restype = None
        lib.oracle_tape_steps.argtypes = [vp]
        lib.oracle_tape_steps.restype = ip
        lib.oracle_tape_step.argtypes = [vp, ip]
        lib.oracle_tape_step.restype = ctypes.POINTER(_TapeStep)
        for name in ("adjref_num_params", "adjref_num_pairs"):
            getattr(lib, name).argtypes = [vp]
            getattr(lib, name).restype = ip
        lib.adjref_pairs.argtypes = [vp, fp, fp]
        lib.adjref_pairs.restype = None
        lib.adjref_theta0.argtypes = [vp, fp]
        lib.adjref_theta0.restype = None
        lib.adjref_loss.argtypes = [vp, fp, fp, fp]
        lib.adjref_loss.restype = ctypes.c_double
        lib.adjref_gradient.argtypes = [vp, fp, fp, fp]
        lib.adjref_gradient.restype = ctypes.c_double
        lib.adjref_fd.argtypes = [vp, fp, fp, ip, fp, ctypes.c_double, ip, fp]
        lib.adjref_fd.restype = None
        lib.adjref_selftest.argtypes = []
        lib.adjref_selftest.restype = ctypes.c_double
    else:
        lib.ref_iterate_ordered.argtypes = [vp, fp, ip]
        lib.ref_iterate_ordered.restype = ip
        lib.ref_prepare_external.argtypes = [vp, ip, fp, ip] + [fp] * 6
        lib.ref_prepare_external.restype = ip
    _libs[kind] = lib
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def make_params(params, order_mode: int = 0) -> _Params:
    return _Params(params.dt, params.gravity, params.iterations, params.alpha, params.betaLin, params.betaAng,
                   params.gamma, params.broadphase, order_mode)


class World:
    """A scene stepped by the oracle or the reference; all queries are in list order."""

    def __init__(self, scene, kind: str = "oracle", order_mode: int = 0):
        self.kind = kind
        self.lib = _lib(kind)
        self.p = "oracle_" if kind == "oracle" else "ref_"
        self._keep = [np.ascontiguousarray(x) for x in (
            scene.size, scene.density, scene.friction, scene.pos, scene.vel, scene.quat,
            scene.ftype, scene.fa, scene.fb, scene.frA, scene.frB, scene.fparam)]
        k = self._keep
        self.params = make_params(scene.params, order_mode)
        if getattr(scene, "shape", None) is None:
            self.h = self._f("create")(ctypes.byref(self.params), scene.n_bodies, *[_ptr(x) for x in k[:6]],
                                       scene.n_forces, *[_ptr(x) for x in k[6:]])
        else:  # round bodies built by the shape constructors
            self._keep += [np.ascontiguousarray(scene.shape, np.int32), np.ascontiguousarray(scene.dims, np.float32)]
            self.h = self._f("create_shapes")(ctypes.byref(self.params), scene.n_bodies, _ptr(self._keep[-2]),
                                              _ptr(self._keep[-1]), *[_ptr(x) for x in k[:6]], scene.n_forces,
                                              *[_ptr(x) for x in k[6:12]])
        self.n = scene.n_bodies

    def _f(self, name):
        return getattr(self.lib, self.p + name)

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        self._f("step")(self.h, n)

    def broadphase_only(self):
        self._f("broadphase_only")(self.h)

    # reference only: the dense SimWorld bodies (the snapshot source)
    def world_bodies(self) -> dict:
        n = self.lib.ref_world_bodies(self.h, *([None] * 9))
        out = {"active": np.zeros(n, np.int32), "shape": np.zeros(n, np.int32), "mass": np.zeros(n, np.float32),
               "pos": np.zeros((n, 3), np.float32), "quat": np.zeros((n, 4), np.float32),
               "size": np.zeros((n, 3), np.float32), "radius": np.zeros(n, np.float32),
               "half_length": np.zeros(n, np.float32), "list_index": np.zeros(n, np.int32)}
        self.lib.ref_world_bodies(self.h, *[_ptr(out[k]) for k in ("active", "shape", "mass", "pos", "quat", "size",
                                                                   "radius", "half_length", "list_index")])
        return out

    # joint edits between steps (list-order bodies; a = -1 anchors to the world point rA)
    def add_joint(self, a, b, rA, rB, stiff_lin=float("inf"), stiff_ang=0.0, fracture=float("inf")) -> int:
        rA = np.ascontiguousarray(rA, np.float32)
        rB = np.ascontiguousarray(rB, np.float32)
        h = self._f("add_joint")(self.h, int(a), int(b), _ptr(rA), _ptr(rB), stiff_lin, stiff_ang, fracture)
        if h < 0:
            raise ValueError("add_joint refused")
        return int(h)

    def set_joint_anchor(self, handle, rA):
        rA = np.ascontiguousarray(rA, np.float32)
        if self._f("set_joint_anchor")(self.h, int(handle), _ptr(rA)) != 0:
            raise ValueError("unknown joint")

    def remove_joint(self, handle):
        if self._f("remove_joint")(self.h, int(handle)) != 0:
            raise ValueError("unknown joint")

    def prepare(self):
        self._f("prepare")(self.h)

    def iterate(self):
        self._f("iterate")(self.h)

    def prepare_external(self, pairs, contacts: dict | None = None):
        """Reference only: prepareStep with the caller's pairs (and contacts) in place of the
        broadphase (and narrowphase), as stepCpuReferenceWithExternalBroadphase sets up."""
        pairs = np.ascontiguousarray(np.asarray(pairs, np.int32).reshape(-1, 2))
        c = contacts or {"ab": np.zeros((0, 2), np.int32), "n": np.zeros(0, np.int32),
                         "basis": np.zeros((0, 9), np.float32), "keys": np.zeros((0, 8), np.int32),
                         "contact": np.zeros((0, 8, 15), np.float32), "stick": np.zeros((0, 8), np.int32)}
        arr = [np.ascontiguousarray(c[k], dt) for k, dt in (("ab", np.int32), ("n", np.int32), ("basis", np.float32),
                                                            ("keys", np.int32), ("contact", np.float32),
                                                            ("stick", np.int32))]
        self.lib.ref_prepare_external(self.h, len(pairs), _ptr(pairs), len(arr[1]), *[_ptr(a) for a in arr])

    def iterate_ordered(self, order: np.ndarray):
        order = np.ascontiguousarray(order, dtype=np.int32)
        self.lib.ref_iterate_ordered(self.h, _ptr(order), int(order.size))

    def finish(self):
        self._f("finish")(self.h)

    def bodies(self) -> dict:
        n = self.n
        out = {k: np.zeros((n, d), np.float32) for k, d in
               (("pos", 3), ("quat", 4), ("vel", 3), ("angvel", 3), ("prevvel", 3))}
        self._f("get_bodies")(self.h, *[_ptr(out[k]) for k in ("pos", "quat", "vel", "angvel", "prevvel")])
        return out

    def body_props(self) -> dict:
        n = self.n
        out = {"mass": np.zeros(n, np.float32), "moment": np.zeros((n, 3), np.float32),
               "radius": np.zeros(n, np.float32), "size": np.zeros((n, 3), np.float32),
               "friction": np.zeros(n, np.float32)}
        self._f("get_body_props")(self.h, *[_ptr(out[k]) for k in ("mass", "moment", "radius", "size", "friction")])
        return out

    def manifolds(self) -> dict:
        m = self._f("num_manifolds")(self.h)
        out = {"ab": np.zeros((m, 2), np.int32), "seq": np.zeros(m, np.int64), "n": np.zeros(m, np.int32),
               "basis": np.zeros((m, 9), np.float32), "friction": np.zeros(m, np.float32),
               "keys": np.zeros((m, 8), np.int32), "contact": np.zeros((m, 8, 15), np.float32),
               "stick": np.zeros((m, 8), np.int32)}
        self._f("get_manifolds")(self.h, *[_ptr(out[k]) for k in
                                           ("ab", "seq", "n", "basis", "friction", "keys", "contact", "stick")])
        return out

    def joints(self) -> dict:
        m = self._f("num_joints")(self.h)
        out = {"ab": np.zeros((m, 2), np.int32), "state": np.zeros((m, 18), np.float32),
               "broken": np.zeros(m, np.int32)}
        self._f("get_joints")(self.h, _ptr(out["ab"]), _ptr(out["state"]), _ptr(out["broken"]))
        return out

    def counters(self) -> np.ndarray:
        c = np.zeros(9, np.int64)
        self._f("get_counters")(self.h, _ptr(c))
        return c

    # oracle-only
    def colours(self):
        c = np.zeros(self.n, np.int32)
        nc = np.zeros(1, np.int32)
        self.lib.oracle_get_colours(self.h, _ptr(c), _ptr(nc))
        return c, int(nc[0])

    def solve_order(self) -> np.ndarray:
        o = np.zeros(max(self.n, 1), np.int32)
        k = self.lib.oracle_get_solve_order(self.h, _ptr(o))
        return o[:k].copy()

    def body_aux(self) -> dict:
        n = self.n
        out = {"init_lin": np.zeros((n, 3), np.float32), "init_ang": np.zeros((n, 4), np.float32),
               "inert_lin": np.zeros((n, 3), np.float32), "inert_ang": np.zeros((n, 4), np.float32)}
        self.lib.oracle_get_body_aux(self.h, *[_ptr(out[k]) for k in ("init_lin", "init_ang", "inert_lin", "inert_ang")])
        return out


    # frozen-branch tape, FP64 replay and reference adjoint (oracle only)
    def tape_begin(self):
        if self.lib.oracle_tape_begin(self.h) != 0:
            raise ValueError("the differentiable step covers contact-only worlds")

    def tape_steps(self) -> int:
        return int(self.lib.oracle_tape_steps(self.h))

    def tape_step(self, s: int) -> dict:
        """One recorded step: flags (iterations x nMan x 8 x 3: primal as A, as B, dual),
        body flags, links to the previous step's slots, initialisation clamp flags."""
        t = self.lib.oracle_tape_step(self.h, s).contents
        M, n, it = t.nMan, self.n, t.iterations
        arr = lambda ptr, count: np.ctypeslib.as_array(ptr, shape=(count,)).copy() if count else np.zeros(0)
        return {"nMan": M, "flags": arr(t.flags, it * M * 8 * 3).reshape(it, M, 8, 3),
                "body_flags": arr(t.bodyFlags, n), "src": arr(t.src, M * 8).reshape(M, 8),
                "init_flags": arr(t.initFlags, M * 8).reshape(M, 8), "ncontacts": arr(t.ncontacts, M)}

    def adj_pairs(self):
        """Friction pairs (lo, hi) in parameter order and their nominal coefficients."""
        P = self.lib.adjref_num_pairs(self.h)
        lohi = np.zeros((max(P, 0), 2), np.int32)
        mu = np.zeros(max(P, 0), np.float32)
        self.lib.adjref_pairs(self.h, _ptr(lohi), _ptr(mu))
        return lohi, mu

    def adj_theta0(self) -> np.ndarray:
        th = np.zeros(self.lib.adjref_num_params(self.h), np.float64)
        self.lib.adjref_theta0(self.h, _ptr(th))
        return th

    def adj_loss(self, theta, target):
        theta = np.ascontiguousarray(theta, np.float64)
        target = np.ascontiguousarray(target, np.float64)
        pos = np.zeros((self.n, 3), np.float64)
        loss = self.lib.adjref_loss(self.h, _ptr(theta), _ptr(target), _ptr(pos))
        return float(loss), pos

    def adj_gradient(self, theta, target):
        theta = np.ascontiguousarray(theta, np.float64)
        target = np.ascontiguousarray(target, np.float64)
        g = np.zeros_like(theta)
        loss = self.lib.adjref_gradient(self.h, _ptr(theta), _ptr(target), _ptr(g))
        return float(loss), g

    def adj_fd(self, theta, target, dirs, h=1e-4, threads=None):
        theta = np.ascontiguousarray(theta, np.float64)
        target = np.ascontiguousarray(target, np.float64)
        dirs = np.ascontiguousarray(dirs, np.float64)
        out = np.zeros(2 * dirs.shape[0], np.float64)
        threads = threads or max(1, min(os.cpu_count() or 1, 2 * dirs.shape[0]))
        self.lib.adjref_fd(self.h, _ptr(theta), _ptr(target), int(dirs.shape[0]), _ptr(dirs), float(h),
                           int(threads), _ptr(out))
        return out[:dirs.shape[0]].copy()


class Fp64Reference:
    """The reference solver built in double precision (oracle/make_fp64.py), stepped by its
    stock CPU backend in its own list order from the scene's single-precision inputs
    (widened exactly). Box worlds with joints, springs and ignore pairs."""

    def __init__(self, scene):
        if getattr(scene, "shape", None) is not None:
            raise ValueError("the FP64 reference driver builds box worlds only")
        if not ref64_available():
            raise FileNotFoundError(f"{REF64_LIB} not built (make -C oracle ref64)")
        lib = _libs.get("ref64")
        if lib is None:
            lib = ctypes.CDLL(REF64_LIB)
            vp, ip, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p
            lib.ref64_create.restype = vp
            lib.ref64_create.argtypes = [ctypes.POINTER(_Params), ip] + [fp] * 6 + [ip] + [fp] * 6
            lib.ref64_destroy.argtypes = [vp]
            lib.ref64_destroy.restype = None
            lib.ref64_step.argtypes = [vp, ip]
            lib.ref64_step.restype = ip
            lib.ref64_num_bodies.argtypes = [vp]
            lib.ref64_num_bodies.restype = ip
            lib.ref64_get_bodies.argtypes = [vp] + [fp] * 4
            lib.ref64_get_bodies.restype = None
            lib.ref64_is_double.argtypes = []
            lib.ref64_is_double.restype = ip
            if lib.ref64_is_double() != 1:
                raise RuntimeError("libavbd_ref64.so was not built in double precision")
            _libs["ref64"] = lib
        self.lib = lib
        self._keep = [np.ascontiguousarray(x) for x in (
            scene.size, scene.density, scene.friction, scene.pos, scene.vel, scene.quat,
            scene.ftype, scene.fa, scene.fb, scene.frA, scene.frB, scene.fparam)]
        self.params = make_params(scene.params, 0)
        self.h = lib.ref64_create(ctypes.byref(self.params), scene.n_bodies, *[_ptr(x) for x in self._keep[:6]],
                                  scene.n_forces, *[_ptr(x) for x in self._keep[6:]])
        self.n = scene.n_bodies

    def step(self, n: int = 1):
        self.lib.ref64_step(self.h, n)

    def bodies(self) -> dict:
        n = self.n
        out = {k: np.zeros((n, d), np.float64) for k, d in (("pos", 3), ("quat", 4), ("vel", 3), ("angvel", 3))}
        self.lib.ref64_get_bodies(self.h, *[_ptr(out[k]) for k in ("pos", "quat", "vel", "angvel")])
        return out

    def close(self):
        if self.h:
            self.lib.ref64_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pose_error(a: dict, b: dict) -> tuple[float, float]:
    """Largest position difference (m) and largest rotation angle between orientations
    (rad) over all bodies of two body-state dicts, evaluated in double precision."""
    dp = float(np.abs(np.asarray(a["pos"], np.float64) - np.asarray(b["pos"], np.float64)).max()) \
        if len(a["pos"]) else 0.0
    qa = np.asarray(a["quat"], np.float64)
    qb = np.asarray(b["quat"], np.float64)
    qa = qa / np.linalg.norm(qa, axis=1, keepdims=True)
    qb = qb / np.linalg.norm(qb, axis=1, keepdims=True)
    c = np.clip(np.abs(np.sum(qa * qb, axis=1)), 0.0, 1.0)
    # 2 asin(|qa x qb| ...) is better conditioned than 2 acos(c) for tiny angles
    s = np.sqrt(np.maximum(0.0, 1.0 - c * c))
    ang = 2.0 * np.arctan2(s, c)
    return dp, float(ang.max()) if len(ang) else 0.0


def adjoint_selftest() -> float:
    """Largest relative error of the step's VJP primitives against central differences."""
    return float(_lib("oracle").adjref_selftest())


def collide_boxes(kind: str, pA, qA, sA, pB, qB, sB):
    lib = _lib(kind)
    f = getattr(lib, ("oracle_" if kind == "oracle" else "ref_") + "collide_boxes")
    args = [np.ascontiguousarray(np.asarray(x, np.float32)) for x in (pA, qA, sA, pB, qB, sB)]
    keys = np.zeros(8, np.int32)
    rA = np.zeros((8, 3), np.float32)
    rB = np.zeros((8, 3), np.float32)
    basis = np.zeros(9, np.float32)
    n = f(*[_ptr(a) for a in args], _ptr(keys), _ptr(rA), _ptr(rB), _ptr(basis))
    return n, keys, rA, rB, basis


def colour_priority(b: int) -> int:
    return int(_lib("oracle").oracle_colour_priority(b))


# ---------------------------------------------------------------------------
# Viewer-bridge snapshots (test restatement of viewer_bridge.cpp:748-842 and of the
# viewer's decoder, viewer/src/main.js:986-1050)
# ---------------------------------------------------------------------------

SNAPSHOT_MAGIC = 0x53425641
SHAPE_NAMES = {0: "box", 1: "sphere", 2: "capsule", 3: "cylinder"}


def material_id(mass, shape):
    """materialIdForBody (viewer_bridge.cpp:475-493)."""
    if mass <= 0.0:
        return 0
    return {0: 1, 1: 3, 3: 4, 2: 5}.get(int(shape), 1)


def snapshot_fields(ids, shape, mass, pos, quat, size, radius, half_length) -> list:
    """Per-body snapshot fields in ascending id order (one dict each)."""
    order = np.argsort(np.asarray(ids), kind="stable")
    return [{"id": int(ids[i]), "shape": int(shape[i]), "material": material_id(float(mass[i]), shape[i]),
             "dynamic": bool(mass[i] > 0), "pos": np.asarray(pos[i], np.float32),
             "quat": np.asarray(quat[i], np.float32), "size": np.asarray(size[i], np.float32),
             "radius": np.float32(radius[i]), "half_length": np.float32(half_length[i])} for i in order]


def encode_snapshot(frame: int, scene: str, bodies: list) -> bytes:
    """makeSnapshotBinary (viewer_bridge.cpp:800-842)."""
    name = scene.encode()
    out = [struct.pack("<IIQII", SNAPSHOT_MAGIC, 1, frame, len(name), len(bodies)), name]
    for b in bodies:
        out.append(struct.pack("<IIII", b["id"], b["shape"], b["material"], 1 if b["dynamic"] else 0))
        out.append(np.concatenate([b["pos"], b["quat"], b["size"], [b["radius"], b["half_length"]]]).astype(
            "<f4").tobytes())
    return b"".join(out)


def decode_snapshot(buf: bytes) -> dict:
    """decodeBinarySnapshot (viewer/src/main.js:986-1050)."""
    magic, version, frame, scene_bytes, count = struct.unpack_from("<IIQII", buf, 0)
    if magic != SNAPSHOT_MAGIC or version != 1:
        raise ValueError("not an AVBD binary snapshot")
    off = 24
    scene = buf[off:off + scene_bytes].decode()
    off += scene_bytes
    bodies = []
    for _ in range(count):
        i, shape, material, dynamic = struct.unpack_from("<IIII", buf, off)
        f = np.frombuffer(buf, "<f4", 12, off + 16)
        bodies.append({"id": i, "shape": shape, "material": material, "dynamic": dynamic != 0, "pos": f[0:3],
                       "quat": f[3:7], "size": f[7:10], "radius": f[10], "half_length": f[11]})
        off += 64
    if off != len(buf):
        raise ValueError("trailing bytes")
    return {"frame": frame, "scene": scene, "bodies": bodies}


def _json_escape(text: str) -> str:
    """jsonEscape (viewer_bridge.cpp:495-530)."""
    out = []
    for ch in text:
        if ch in '"\\':
            out.append("\\" + ch)
        elif ch == "\n":
            out.append("\\n")
        elif ch == "\r":
            out.append("\\r")
        elif ch == "\t":
            out.append("\\t")
        elif ord(ch) < 0x20:
            out.append("\\u%04x" % ord(ch))
        else:
            out.append(ch)
    return "".join(out)


def snapshot_json(frame: int, scene: str, bodies: list) -> str:
    """makeSnapshotJson (viewer_bridge.cpp:748-777): fixed notation, 5 decimals."""
    f = lambda x: "%.5f" % float(x)
    items = []
    for b in bodies:
        items.append('{"id":%d,"shape":"%s","position":[%s],"rotation":[%s],"size":[%s],"radius":%s,'
                     '"halfLength":%s,"dynamic":%s,"material":%d}' % (
                         b["id"], SHAPE_NAMES.get(b["shape"], "box"), ",".join(map(f, b["pos"])),
                         ",".join(map(f, b["quat"])), ",".join(map(f, b["size"])), f(b["radius"]),
                         f(b["half_length"]), "true" if b["dynamic"] else "false", b["material"]))
    return ('{"type":"snapshot","version":1,"frame":%d,"scene":"%s","bodies":[' % (frame, _json_escape(scene))
            + ",".join(items) + "]}")
