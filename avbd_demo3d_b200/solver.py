"""Host side of the CUDA AVBD step, mirroring the reference's interfaces.

``World`` owns one device context (include/avbd_cuda.h) holding a scene; it is what the
benchmark and the parity tests drive. ``Solver``, ``Rigid``, ``Joint``, ``Spring``,
``IgnoreCollision`` and ``CudaAvbdBackend`` mirror the reference's C++ classes
(source/solver.h:197-417) with the same constructor arguments and parameter names, so a
scene is built the way source/scenes.h builds it and ``solver.step()`` runs the GPU step.

Derived quantities (mass, moment, bounding radius, joint torque arm, spring rest
length) are computed in float32 with the reference's operation order
(rigid.cpp:34-40, joint.cpp:33, spring.cpp:18-24), so the device starts from the same
bits the reference would hold.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from . import scenes as _scenes

F32 = np.float32


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=dtype))
    return a if shape is None else a.reshape(shape)


# ---------------------------------------------------------------------------
# float32 arithmetic in the reference's order
# ---------------------------------------------------------------------------


def _cross32(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def rotate32(q: np.ndarray, v: np.ndarray) -> np.ndarray:
    """rotate(q, v) = v + t*w + cross(u, t), t = 2 cross(u, v)   (maths.h:441-446)"""
    q = np.asarray(q, F32)
    v = np.asarray(v, F32)
    u = q[..., :3]
    t = _cross32(u, v) * F32(2.0)
    return (v + t * q[..., 3:4]) + _cross32(u, t)


def _dot32(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def box_properties(size: np.ndarray, density: np.ndarray):
    """Mass, moment and bounding radius of boxes (rigid.cpp:34-40)."""
    s = np.asarray(size, F32).reshape(-1, 3)
    d = np.asarray(density, F32).reshape(-1)
    mass = ((s[:, 0] * s[:, 1]) * s[:, 2]) * d
    twelve = F32(12.0)
    moment = np.stack([(s[:, 1] * s[:, 1] + s[:, 2] * s[:, 2]) / twelve * mass,
                       (s[:, 0] * s[:, 0] + s[:, 2] * s[:, 2]) / twelve * mass,
                       (s[:, 0] * s[:, 0] + s[:, 1] * s[:, 1]) / twelve * mass], axis=1)
    h = s * F32(0.5)
    radius = np.sqrt(_dot32(h, h))
    return mass.astype(F32), moment.astype(F32), radius.astype(F32)


def round_properties(shape: np.ndarray, dims: np.ndarray, density: np.ndarray, mass, moment, radius):
    """Mass, moment and bounding radius of spheres, capsules and cylinders, written over the
    box values in place (Rigid::makeSphere / makeCapsule / makeCylinder, rigid.cpp:44-90, in
    float32 with the same operation order)."""
    pi = F32(3.14159265358979323846)
    r = np.asarray(dims, F32)[:, 0]
    h = np.asarray(dims, F32)[:, 1]
    d = np.asarray(density, F32)
    two5 = F32(2.0) / F32(5.0)
    sphere_mass = (((F32(4.0) / F32(3.0) * pi) * r) * r) * r * d
    for t in (1, 2, 3):
        sel = np.asarray(shape) == t
        if not sel.any():
            continue
        rs, hs, ds, sm = r[sel], h[sel], d[sel], sphere_mass[sel]
        if t == 1:  # sphere
            m = sm
            i = ((two5 * m) * rs) * rs
            mom = np.stack([i, i, i], axis=1)
            rad = rs
        elif t == 2:  # capsule
            L = hs * F32(2.0)
            cm = (((pi * rs) * rs) * L) * ds
            m = cm + sm
            axial = ((F32(0.5) * cm) * rs) * rs + ((two5 * sm) * rs) * rs
            trans = ((F32(3.0) * rs) * rs + L * L) / F32(12.0) * cm + ((two5 * sm) * rs) * rs + (sm * hs) * hs
            mom = np.stack([trans, trans, axial], axis=1)
            rad = hs + rs
        else:  # cylinder
            H = hs * F32(2.0)
            m = (((pi * rs) * rs) * H) * ds
            axial = ((F32(0.5) * m) * rs) * rs
            trans = ((F32(3.0) * rs) * rs + H * H) / F32(12.0) * m
            mom = np.stack([trans, trans, axial], axis=1)
            rad = np.sqrt(rs * rs + hs * hs)
        mass[sel] = m
        moment[sel] = mom
        radius[sel] = rad


# ---------------------------------------------------------------------------
# Device world
# ---------------------------------------------------------------------------


class World:
    """Scenes resident on one GPU. A single scene is one world; a list of scenes is a batch of
    independent worlds stepped together (each evolves exactly as it would alone). Body
    arrays are in list order per world (index 0 of a world = its newest body, the head of
    the reference's Solver::bodies), worlds concatenated; `world_start` gives the ranges."""

    def __init__(self, scene, device: int = 0, stream: int | None = None):
        self.lib = _lib.load()
        self.h = ctypes.c_void_p()
        rc = self.lib.avbd_create(ctypes.byref(self.h), device, stream)
        if rc != _lib.AVBD_OK:
            raise _lib.AvbdError(f"avbd_create failed ({rc}); is a CUDA device present?")
        self.scenes = list(scene) if isinstance(scene, (list, tuple)) else [scene]
        self.scene = self.scenes[0]
        self.n = sum(sc.n_bodies for sc in self.scenes)
        self.world_start = np.concatenate([[0], np.cumsum([sc.n_bodies for sc in self.scenes])]).astype(np.int32)
        self.set_params(self.scene.params)
        self._load(self.scenes)

    # -- helpers
    def _check(self, rc: int, what: str):
        if rc != _lib.AVBD_OK:
            msg = self.lib.avbd_last_error(self.h).decode(errors="replace")
            raise _lib.AvbdError(f"{what} failed ({_lib.ERRORS.get(rc, rc)}): {msg}")

    def close(self):
        if self.h:
            self.lib.avbd_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p):
        self.params = _lib.AvbdParams(p.dt, p.gravity, p.iterations, p.alpha, p.betaLin, p.betaAng, p.gamma,
                                      p.broadphase)
        self._check(self.lib.avbd_set_params(self.h, ctypes.byref(self.params)), "avbd_set_params")

    @staticmethod
    def list_order(a):
        """Creation order -> list order (the reference prepends every new body)."""
        return np.ascontiguousarray(a[::-1])

    @staticmethod
    def _scene_arrays(sc: _scenes.Scene, offset: int, seq0: int):
        """One world's bodies (list order) and forces (global body indices, sequence numbers
        from seq0 in creation order)."""
        n = sc.n_bodies
        if sc.n_forces and (sc.fb.min() < 0 or sc.fb.max() >= n or sc.fa.max() >= n or sc.fa.min() < -1):
            raise _lib.AvbdError("avbd_load_world failed (argument): force body index out of range")
        mass, moment, radius = box_properties(sc.size, sc.density)
        shape = np.zeros(n, np.int32)
        shape_radius, half_length = radius.copy(), np.zeros(n, F32)  # a box's shape radius is its bounding radius
        if getattr(sc, "shape", None) is not None:
            round_properties(sc.shape, sc.dims, sc.density, mass, moment, radius)
            shape = np.asarray(sc.shape, np.int32)
            rnd = shape != 0
            shape_radius[rnd] = np.asarray(sc.dims, F32)[rnd, 0]
            half_length[rnd] = np.asarray(sc.dims, F32)[rnd, 1]
        L = World.list_order
        body = dict(position3=L(sc.pos), orientation4=L(sc.quat), velocity3=L(sc.vel),
                    angular3=np.zeros((n, 3), F32), prev_velocity3=L(sc.vel), size3=L(sc.size), mass=L(mass),
                    moment3=L(moment), friction=L(sc.friction), radius=L(radius), shape=L(shape),
                    shape_radius=L(shape_radius), half_length=L(half_length))
        local = lambda c: np.where(c >= 0, n - 1 - c, -1).astype(np.int32)
        glob = lambda c: np.where(c >= 0, c + offset, -1).astype(np.int32)
        seq = np.arange(seq0, seq0 + sc.n_forces, dtype=np.int64)
        fa, fb = local(sc.fa), local(sc.fb)
        jm = sc.ftype == _scenes.FORCE_JOINT
        sm = sc.ftype == _scenes.FORCE_SPRING
        im = sc.ftype == _scenes.FORCE_IGNORE
        lp, lq, lsize = body["position3"], body["orientation4"], body["size3"]
        # joints (joint.cpp:25-33): torqueArm = lengthSq(sizeA + sizeB)
        J = int(jm.sum())
        j_state = np.zeros((J, 28), F32)
        if J:
            sa = np.where((fa[jm] >= 0)[:, None], lsize[np.maximum(fa[jm], 0)], F32(0.0)).astype(F32)
            ssum = sa + lsize[fb[jm]]
            j_state[:, 0:3] = sc.frA[jm]
            j_state[:, 3:6] = sc.frB[jm]
            j_state[:, 24:27] = sc.fparam[jm]
            j_state[:, 27] = _dot32(ssum, ssum)
        # springs (spring.cpp:14-25): rest < 0 -> initial distance of the anchor points
        S = int(sm.sum())
        s_state = np.zeros((S, 8), F32)
        if S:
            a, b = fa[sm], fb[sm]
            rA, rB = sc.frA[sm], sc.frB[sm]
            d = (rotate32(lq[a], rA) + lp[a]) - (rotate32(lq[b], rB) + lp[b])
            dist = np.sqrt(_dot32(d, d))
            rest = sc.fparam[sm][:, 1].copy()
            s_state[:, 0:3] = rA
            s_state[:, 3:6] = rB
            s_state[:, 6] = np.where(rest < 0, dist, rest).astype(F32)
            s_state[:, 7] = sc.fparam[sm][:, 0]
        ab = lambda m: np.stack([glob(fa[m]), glob(fb[m])], axis=1).reshape(-1, 2).astype(np.int32)
        forces = dict(j_ab=ab(jm), j_seq=seq[jm], j_state=j_state, j_broken=np.zeros(J, np.int32), s_ab=ab(sm),
                      s_seq=seq[sm], s_state=s_state, i_ab=ab(im), i_seq=seq[im])
        return body, forces

    def _load(self, scenes_list):
        bodies, forces = [], []
        offset, seq0 = 0, 0
        for sc in scenes_list:
            b, f = self._scene_arrays(sc, offset, seq0)
            bodies.append(b)
            forces.append(f)
            offset += sc.n_bodies
            seq0 += sc.n_forces
        self._body_arrays = {k: np.ascontiguousarray(np.concatenate([b[k] for b in bodies])) for k in bodies[0]}
        self._force_arrays = {k: np.ascontiguousarray(np.concatenate([f[k] for f in forces])) for k in forces[0]}
        for k in ("j_ab", "s_ab", "i_ab"):
            self._force_arrays[k] = self._force_arrays[k].reshape(-1, 2).astype(np.int32)
        self.props = {"mass": self._body_arrays["mass"], "moment": self._body_arrays["moment3"],
                      "radius": self._body_arrays["radius"], "size": self._body_arrays["size3"],
                      "friction": self._body_arrays["friction"]}
        ba, fa_ = self._body_arrays, self._force_arrays
        has_shapes = bool((ba["shape"] != 0).any())
        bodies_s = _lib.AvbdBodies(self.n, *[_ptr(ba[k]) for k in (
            "position3", "orientation4", "velocity3", "angular3", "prev_velocity3", "size3", "mass", "moment3",
            "friction", "radius")], *([_ptr(ba[k]) for k in ("shape", "shape_radius", "half_length")]
                                      if has_shapes else [None, None, None]))
        joints = _lib.AvbdJoints(len(fa_["j_seq"]), _ptr(fa_["j_ab"]), _ptr(fa_["j_seq"]), _ptr(fa_["j_state"]),
                                 _ptr(fa_["j_broken"]))
        springs = _lib.AvbdSprings(len(fa_["s_seq"]), _ptr(fa_["s_ab"]), _ptr(fa_["s_seq"]), _ptr(fa_["s_state"]))
        ignores = _lib.AvbdIgnores(len(fa_["i_seq"]), _ptr(fa_["i_ab"]), _ptr(fa_["i_seq"]))
        manifolds = _lib.AvbdManifolds(0)
        ws = np.ascontiguousarray(self.world_start)
        self._check(self.lib.avbd_load_batch(self.h, len(scenes_list), ws.ctypes.data_as(_lib.c_int_p),
                                             ctypes.byref(bodies_s), ctypes.byref(joints), ctypes.byref(springs),
                                             ctypes.byref(ignores), ctypes.byref(manifolds), seq0),
                    "avbd_load_batch")

    # -- stepping
    def step(self, n: int = 1, sync: bool = True):
        self._check(self.lib.avbd_step(self.h, n), "avbd_step")
        if sync:
            self.synchronize()

    def step_external(self, pairs, contacts: dict | None = None):
        """One step with the broadphase replaced by `pairs` ((k, 2) list indices) and, for the
        pairs of `contacts` (dict of ab (e, 2), n (e,), basis (e, 9), keys (e, 8),
        contact (e, 8, 15), stick (e, 8), optional creates (e,)), the narrowphase replaced by
        the given contacts (Solver::stepCpuReferenceWithExternalBroadphase)."""
        pairs = _c(np.asarray(pairs, np.int32).reshape(-1, 2), np.int32)
        ext = None
        if contacts is not None:
            arr = {k: _c(contacts[k], dt) for k, dt in (("ab", np.int32), ("n", np.int32), ("basis", F32),
                                                        ("keys", np.int32), ("contact", F32), ("stick", np.int32))}
            cr = contacts.get("creates")
            arr["creates"] = None if cr is None else _c(cr, np.int32)
            self._ext_keep = arr
            ext = _lib.AvbdExternalContacts(len(arr["n"]), *[_ptr(arr[k]) for k in (
                "ab", "n", "basis", "keys", "contact", "stick", "creates")])
        rc = self.lib.avbd_step_external(self.h, len(pairs), pairs.ctypes.data_as(_lib.c_int_p),
                                         ctypes.byref(ext) if ext is not None else None)
        self._check(rc, "avbd_step_external")

    def broadphase_only(self):
        """The reference's collision-only step: drop every manifold, run the broadphase alone."""
        self._check(self.lib.avbd_broadphase_only(self.h), "avbd_broadphase_only")

    def synchronize(self):
        self._check(self.lib.avbd_synchronize(self.h), "avbd_synchronize")

    # -- readback
    _BODY_WIDTH = {"pos": 3, "quat": 4, "vel": 3, "angvel": 3, "prevvel": 3, "init_lin": 3, "init_ang": 4,
                   "inert_lin": 3, "inert_ang": 4}

    def bodies(self, aux: bool = False, out: dict | None = None) -> dict:
        """Body state in list order. `out`: caller-owned arrays to fill in place (float32,
        C-contiguous, (n, width)); a simulation loop that reads every step reuses them."""
        n = self.n
        if out is not None:
            for k, v in out.items():
                if k not in self._BODY_WIDTH or not isinstance(v, np.ndarray) or v.dtype != F32 or \
                        v.shape != (n, self._BODY_WIDTH[k]) or not v.flags.c_contiguous:
                    raise ValueError(f"bodies(out=...): {k} must be a C-contiguous float32 array of shape "
                                     f"({n}, {self._BODY_WIDTH.get(k)})")
            # the checked arrays' addresses directly (out holds them for the call)
            st = _lib.AvbdBodyState(*[out[k].ctypes.data if k in out else None for k in (
                "pos", "quat", "vel", "angvel", "prevvel", "init_lin", "init_ang", "inert_lin", "inert_ang")])
            self._check(self.lib.avbd_read_bodies(self.h, ctypes.byref(st)), "avbd_read_bodies")
            return out
        else:
            out = {"pos": np.zeros((n, 3), F32), "quat": np.zeros((n, 4), F32), "vel": np.zeros((n, 3), F32),
                   "angvel": np.zeros((n, 3), F32), "prevvel": np.zeros((n, 3), F32)}
            if aux:
                out.update(init_lin=np.zeros((n, 3), F32), init_ang=np.zeros((n, 4), F32),
                           inert_lin=np.zeros((n, 3), F32), inert_ang=np.zeros((n, 4), F32))
        st = _lib.AvbdBodyState(*[_ptr(out.get(k)) for k in (
            "pos", "quat", "vel", "angvel", "prevvel", "init_lin", "init_ang", "inert_lin", "inert_ang")])
        self._check(self.lib.avbd_read_bodies(self.h, ctypes.byref(st)), "avbd_read_bodies")
        return out

    def write_bodies(self, pos=None, quat=None, vel=None, angvel=None, prevvel=None):
        """Overwrite body state (list order) between steps; fields not given keep their values."""
        given = (pos, quat, vel, angvel, prevvel)
        n = self.n
        if all(isinstance(x, np.ndarray) and x.dtype == F32 and x.flags.c_contiguous and x.shape == (n, w)
               for x, w in zip(given, (3, 4, 3, 3, 3))):
            # every field already float32 and packed: their addresses directly (held by the caller)
            b = _lib.AvbdBodies(n, *[x.ctypes.data for x in given], None, None, None, None, None)
            self._check(self.lib.avbd_write_bodies(self.h, ctypes.byref(b)), "avbd_write_bodies")
            return
        cur = self.bodies() if any(x is None for x in given) else {}
        arr = dict(position3=_c(cur["pos"] if pos is None else pos, F32),
                   orientation4=_c(cur["quat"] if quat is None else quat, F32),
                   velocity3=_c(cur["vel"] if vel is None else vel, F32),
                   angular3=_c(cur["angvel"] if angvel is None else angvel, F32),
                   prev_velocity3=_c(cur["prevvel"] if prevvel is None else prevvel, F32))
        b = _lib.AvbdBodies(self.n, _ptr(arr["position3"]), _ptr(arr["orientation4"]), _ptr(arr["velocity3"]),
                            _ptr(arr["angular3"]), _ptr(arr["prev_velocity3"]), None, None, None, None, None)
        self._check(self.lib.avbd_write_bodies(self.h, ctypes.byref(b)), "avbd_write_bodies")

    def manifolds(self) -> dict:
        m = ctypes.c_int32()
        self._check(self.lib.avbd_num_manifolds(self.h, ctypes.byref(m)), "avbd_num_manifolds")
        m = m.value
        out = {"ab": np.zeros((m, 2), np.int32), "seq": np.zeros(m, np.int64), "n": np.zeros(m, np.int32),
               "basis": np.zeros((m, 9), F32), "friction": np.zeros(m, F32), "keys": np.zeros((m, 8), np.int32),
               "contact": np.zeros((m, 8, 15), F32), "stick": np.zeros((m, 8), np.int32)}
        o = _lib.AvbdManifoldsOut(*[_ptr(out[k]) for k in ("ab", "seq", "n", "basis", "friction", "keys", "contact",
                                                            "stick")])
        self._check(self.lib.avbd_read_manifolds(self.h, ctypes.byref(o)), "avbd_read_manifolds")
        return out

    def joints(self) -> dict:
        m = ctypes.c_int32()
        self._check(self.lib.avbd_num_joints(self.h, ctypes.byref(m)), "avbd_num_joints")
        m = m.value
        out = {"ab": np.zeros((m, 2), np.int32), "seq": np.zeros(m, np.int64), "state28": np.zeros((m, 28), F32),
               "broken": np.zeros(m, np.int32)}
        o = _lib.AvbdJointsOut(_ptr(out["ab"]), _ptr(out["seq"]), _ptr(out["state28"]), _ptr(out["broken"]))
        self._check(self.lib.avbd_read_joints(self.h, ctypes.byref(o)), "avbd_read_joints")
        # same 18-float view as the checkers: C0Lin C0Ang penLin penAng lamLin lamAng
        out["state"] = np.ascontiguousarray(out["state28"][:, 6:24])
        return out

    # -- joint edits between steps (SimulationHost's drag, simulation_host.cpp:242-274)
    def next_seq(self) -> int:
        q = ctypes.c_int64()
        self._check(self.lib.avbd_next_seq(self.h, ctypes.byref(q)), "avbd_next_seq")
        return q.value

    def add_joint(self, a, b, rA, rB, stiff_lin=float("inf"), stiff_ang=0.0, fracture=float("inf")) -> int:
        """new Joint(solver, a, b, rA, rB, stiffLin, stiffAng, fracture) (joint.cpp:25-33) on
        list-order bodies (a = -1: anchored to the world point rA). Returns its sequence number."""
        seq = self.next_seq()
        size = self.props["size"]
        sa = size[a] if a >= 0 else np.zeros(3, F32)
        ssum = (sa + size[b]).astype(F32)
        state = np.zeros((1, 28), F32)
        state[0, 0:3] = rA
        state[0, 3:6] = rB
        state[0, 24:27] = (stiff_lin, stiff_ang, fracture)
        state[0, 27] = _dot32(ssum[None], ssum[None])[0]
        self._edit_joints("avbd_add_joints", np.array([[a, b]], np.int32), np.array([seq], np.int64), state)
        return seq

    def _edit_joints(self, fn, ab, seq, state, broken=None):
        ab, seq, state = _c(ab, np.int32), _c(seq, np.int64), _c(state, F32)
        broken = _c(np.zeros(len(seq), np.int32) if broken is None else broken, np.int32)
        j = _lib.AvbdJoints(len(seq), _ptr(ab), _ptr(seq), _ptr(state), _ptr(broken))
        self._check(getattr(self.lib, fn)(self.h, ctypes.byref(j)), fn)

    def write_joints(self, ab, seq, state28, broken=None):
        """Overwrite the state of existing joints, matched by sequence number."""
        self._edit_joints("avbd_write_joints", ab, seq, state28, broken)

    def set_joint_anchor(self, seq, rA):
        """Joint::rA = rA (updateDrag)."""
        j = self.joints()
        k = np.flatnonzero(j["seq"] == seq)
        if k.size != 1:
            raise _lib.AvbdError(f"no joint with sequence number {seq}")
        st = j["state28"][k].copy()
        st[0, 0:3] = rA
        self.write_joints(j["ab"][k], j["seq"][k], st, j["broken"][k])

    def remove_joint(self, seq):
        """delete joint (releaseDrag)."""
        q = np.array([seq], np.int64)
        self._check(self.lib.avbd_remove_joints(self.h, 1, q.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))),
                    "avbd_remove_joints")

    def colours(self):
        c = np.zeros(max(self.n, 1), np.int32)
        nc = ctypes.c_int32()
        self._check(self.lib.avbd_read_colours(self.h, c.ctypes.data_as(_lib.c_int_p), ctypes.byref(nc)),
                    "avbd_read_colours")
        return c[:self.n], nc.value

    def solve_order(self) -> np.ndarray:
        o = np.zeros(max(self.n, 1), np.int32)
        k = ctypes.c_int32()
        self._check(self.lib.avbd_read_solve_order(self.h, o.ctypes.data_as(_lib.c_int_p), ctypes.byref(k)),
                    "avbd_read_solve_order")
        return o[:k.value].copy()

    @staticmethod
    def primal_variants() -> list:
        lib = _lib.load()
        n = ctypes.c_int32()
        lib.avbd_num_primal_variants(ctypes.byref(n), None, None)
        g = np.zeros(n.value, np.int32)
        m = np.zeros(n.value, np.int32)
        lib.avbd_num_primal_variants(ctypes.byref(n), g.ctypes.data_as(_lib.c_int_p), m.ctypes.data_as(_lib.c_int_p))
        return [{"group": int(a), "min_blocks": int(b)} for a, b in zip(g, m)]

    def set_primal_variant(self, v: int):
        self._check(self.lib.avbd_set_primal_variant(self.h, v), "avbd_set_primal_variant")

    def autotune(self, repeats: int = 3):
        """Time every primal variant on the current colouring and keep the fastest."""
        n = len(self.primal_variants())
        us = np.zeros(n, F32)
        best = ctypes.c_int32()
        self._check(self.lib.avbd_autotune(self.h, repeats, ctypes.byref(best), us.ctypes.data_as(_lib.c_float_p)),
                    "avbd_autotune")
        return best.value, us

    # -- viewer-bridge snapshots (viewer_bridge.cpp:748-842)
    def _snapshot(self, fn, frame, scene, body_id, make):
        ids = None if body_id is None else _c(body_id, np.int32)
        idp = None if ids is None else ids.ctypes.data_as(_lib.c_int_p)
        name = scene.encode()
        size = ctypes.c_int64()
        self._check(getattr(self.lib, fn)(self.h, frame, name, idp, None, 0, ctypes.byref(size)), fn)
        buf = make(size.value)
        self._check(getattr(self.lib, fn)(self.h, frame, name, idp, buf, size.value, ctypes.byref(size)), fn)
        return buf

    def snapshot_binary(self, frame: int = 0, scene: str = "", body_id=None) -> bytes:
        """The AVBS binary snapshot of every body, in ascending id order (ids: the creation rank
        unless body_id gives each list-order body's id)."""
        return bytes(self._snapshot("avbd_snapshot_binary", frame, scene, body_id,
                                    lambda n: (ctypes.c_uint8 * n)()))

    def snapshot_json(self, frame: int = 0, scene: str = "", body_id=None) -> str:
        """makeSnapshotJson's text for every body."""
        buf = self._snapshot("avbd_snapshot_json", frame, scene, body_id, ctypes.create_string_buffer)
        return buf.value.decode()

    def set_iteration_mode(self, mode: int):
        """0 = one launch per colour and iteration plus the dual sweep, 1 = every iteration in
        one cooperative launch (default). Both give the same bits."""
        self._check(self.lib.avbd_set_iteration_mode(self.h, mode), "avbd_set_iteration_mode")

    def iteration_mode(self) -> int:
        m = ctypes.c_int32()
        self._check(self.lib.avbd_iteration_mode(self.h, ctypes.byref(m)), "avbd_iteration_mode")
        return m.value

    def set_colouring(self, mode: int):
        """0 = greedy colouring in list order (default), 1 = hashed priorities."""
        self._check(self.lib.avbd_set_colouring(self.h, mode), "avbd_set_colouring")

    STEP_DEVICE, STEP_HOST = 0, 1

    def set_step_mode(self, mode: int):
        """STEP_DEVICE (default): a step keeps its counts on the device and never waits for
        it; STEP_HOST: the host reads the counts each step needs. Both give the same bits."""
        self._check(self.lib.avbd_set_step_mode(self.h, mode), "avbd_set_step_mode")

    def set_manifold_headroom(self, spare: int):
        """Manifold room beyond the live count for device-resident steps (0 = default)."""
        self._check(self.lib.avbd_set_manifold_headroom(self.h, int(spare)), "avbd_set_manifold_headroom")

    def set_wait_limits(self, colouring_polls: int = 0, iteration_polls: int = 0):
        """Poll limits of the bounded waits (0 = defaults)."""
        self._check(self.lib.avbd_set_wait_limits(self.h, colouring_polls, iteration_polls),
                    "avbd_set_wait_limits")

    def clear_error(self):
        self.lib.avbd_clear_error(self.h)

    def last_error(self) -> str:
        return self.lib.avbd_last_error(self.h).decode(errors="replace")

    def reload(self):
        """Load the world's scenes again (a fresh start in the same context)."""
        self._load(self.scenes)

    # -- differentiable step
    def adjoint_forward(self, steps: int, checkpoint_every: int = 10, sync: bool = True):
        """Step like step(steps), keeping a state snapshot every checkpoint_every steps for
        adjoint_backward."""
        self._check(self.lib.avbd_adjoint_forward(self.h, steps, checkpoint_every), "avbd_adjoint_forward")
        if sync:
            self.synchronize()

    def adjoint_pairs(self):
        """Friction pairs (lo, hi) of the last adjoint_forward and their nominal coefficients."""
        k = ctypes.c_int32()
        self._check(self.lib.avbd_adjoint_num_pairs(self.h, ctypes.byref(k)), "avbd_adjoint_num_pairs")
        lohi = np.zeros((k.value, 2), np.int32)
        mu = np.zeros(k.value, F32)
        self._check(self.lib.avbd_adjoint_read_pairs(self.h, lohi.ctypes.data_as(_lib.c_int_p),
                                                     mu.ctypes.data_as(_lib.c_float_p)), "avbd_adjoint_read_pairs")
        return lohi, mu

    def adjoint_replay_state(self) -> dict:
        """Double-precision final state of the frozen-branch replay of the last forward."""
        n = self.n
        out = {"pos": np.zeros((n, 3)), "quat": np.zeros((n, 4)), "vel": np.zeros((n, 3)), "angvel": np.zeros((n, 3))}
        self._check(self.lib.avbd_adjoint_replay_state(self.h, *[_ptr(out[k]) for k in ("pos", "quat", "vel",
                                                                                         "angvel")]),
                    "avbd_adjoint_replay_state")
        return out

    def adjoint_tape(self, step: int) -> dict:
        """Parity dump of the forward's tape for one step (avbd_adjoint_tape_step)."""
        m = ctypes.c_int32()
        self._check(self.lib.avbd_adjoint_tape_step(self.h, step, ctypes.byref(m), None, None, None),
                    "avbd_adjoint_tape_step")
        it = self.params.iterations
        flags = np.zeros((it, m.value, 8), np.uint16)
        bflags = np.zeros(self.n, np.uint8)
        link = np.zeros((m.value, 8), np.int32)
        self._check(self.lib.avbd_adjoint_tape_step(self.h, step, ctypes.byref(m), _ptr(flags), _ptr(bflags),
                                                    link.ctypes.data_as(_lib.c_int_p)), "avbd_adjoint_tape_step")
        return {"nMan": m.value, "flags": flags, "body_flags": bflags, "src": link}

    def adjoint_backward(self, d_pos=None, d_quat=None, d_vel=None, d_angvel=None) -> dict:
        """Gradient with respect to the state before adjoint_forward and to the parameters,
        given the gradient of a loss with respect to the final state (list order)."""
        n = self.n
        k = ctypes.c_int32()
        self._check(self.lib.avbd_adjoint_num_pairs(self.h, ctypes.byref(k)), "avbd_adjoint_num_pairs")
        out = {"pos": np.zeros((n, 3)), "quat": np.zeros((n, 4)), "vel": np.zeros((n, 3)),
               "angvel": np.zeros((n, 3)), "prevvel": np.zeros((n, 3)), "mass": np.zeros(n),
               "pair_friction": np.zeros(k.value), "friction": np.zeros(n)}
        g = _lib.AvbdAdjointGrad(*[_ptr(out[key]) for key in (
            "pos", "quat", "vel", "angvel", "prevvel", "mass", "pair_friction", "friction")])
        ins = [None if a is None else _c(a, np.float64) for a in (d_pos, d_quat, d_vel, d_angvel)]
        self._check(self.lib.avbd_adjoint_backward(self.h, *[_ptr(a) for a in ins], ctypes.byref(g)),
                    "avbd_adjoint_backward")
        return out

    def set_profiling(self, on: bool = True):
        self._check(self.lib.avbd_set_profiling(self.h, 1 if on else 0), "avbd_set_profiling")

    def reset_profile(self):
        self._check(self.lib.avbd_reset_profile(self.h), "avbd_reset_profile")

    def profile(self) -> dict:
        p = _lib.AvbdProfile()
        self._check(self.lib.avbd_read_profile(self.h, ctypes.byref(p)), "avbd_read_profile")
        out = {"steps": p.steps, "launches": p.launches}
        for k, name in enumerate(_lib.PHASES):
            out[name + "_ms"] = p.phase_ms[k]
            out[name + "_spans"] = p.phase_spans[k]
        return out

    def stats(self) -> dict:
        s = _lib.AvbdStats()
        self._check(self.lib.avbd_get_stats(self.h, ctypes.byref(s)), "avbd_get_stats")
        return {k: getattr(s, k) for k, _ in s._fields_}


# ---------------------------------------------------------------------------
# Mirror of the reference's object interface (solver.h)
# ---------------------------------------------------------------------------


class Rigid:
    """``Rigid(solver, size, density, friction, position, velocity)`` (solver.h:221). After a
    step its state reads from the device world."""

    def __init__(self, solver: "Solver", size, density, friction, position, velocity=(0, 0, 0)):
        self.solver = solver
        self.creation = solver._builder.body(size, density, friction, position, velocity)
        solver._topology_changed()

    @property
    def index(self) -> int:
        """Position in the solver's body list (0 = newest)."""
        return self.solver._n_bodies() - 1 - self.creation

    def _state(self, key):
        st = self.solver._state()
        if st is None:
            b = self.solver._builder.b
            return {"pos": b["pos"], "quat": b["quat"], "vel": b["vel"]}[key][self.creation]
        return st[key][self.index]

    @property
    def positionLin(self):
        return self._state("pos")

    @property
    def positionAng(self):
        return self._state("quat")

    @positionAng.setter
    def positionAng(self, q):
        if self.solver._world is not None:
            raise RuntimeError("orientation edits after the first step go through World.write_bodies")
        self.solver._builder.b["quat"][self.creation] = np.asarray(q, F32).reshape(4)

    @property
    def velocityLin(self):
        return self._state("vel")


class Joint:
    """``Joint(solver, bodyA, bodyB, rA, rB, stiffnessLin=INFINITY, stiffnessAng=0, fracture=INFINITY)``
    (solver.h:252-267); bodyA None anchors bodyB to the world point rA."""

    def __init__(self, solver, bodyA, bodyB, rA, rB, stiffnessLin=math.inf, stiffnessAng=0.0, fracture=math.inf):
        solver._builder.joint(None if bodyA is None else bodyA.creation, bodyB.creation, rA, rB, stiffnessLin,
                              stiffnessAng, fracture)
        solver._topology_changed()


class Spring:
    """``Spring(solver, bodyA, bodyB, rA, rB, stiffness, rest=-1)`` (solver.h:270-281)."""

    def __init__(self, solver, bodyA, bodyB, rA, rB, stiffness, rest=-1.0):
        solver._builder.spring(bodyA.creation, bodyB.creation, rA, rB, stiffness, rest)
        solver._topology_changed()


class IgnoreCollision:
    """``IgnoreCollision(solver, bodyA, bodyB)`` (solver.h:284-291)."""

    def __init__(self, solver, bodyA, bodyB):
        solver._builder.ignore_collision(bodyA.creation, bodyB.creation)
        solver._topology_changed()


class CudaAvbdBackend:
    """The ``PhysicsBackend`` (solver.h:410-417) that runs ``Solver::step`` on the GPU."""

    def __init__(self, device: int = 0):
        self.device = device

    def name(self) -> str:
        return _lib.load().avbd_backend_name().decode()

    def step(self, solver: "Solver"):
        if solver._world is None:
            solver._world = World(solver._scene(), self.device)
        else:
            solver._world.set_params(solver._params())
        solver._world.step(1)
        solver._cached = None


class Solver:
    """``Solver`` (solver.h:346-408): parameters, scene construction, ``step()``."""

    def __init__(self, device: int = 0):
        self.physicsBackend = CudaAvbdBackend(device)
        self.broadphaseMode = _scenes.BROADPHASE_GRID
        self.clear()
        self.defaultParams()

    def defaultParams(self):
        """solver.cpp:909-932"""
        self.dt = float(F32(1.0) / F32(60.0))
        self.gravity = -10.0
        self.iterations = 10
        self.betaLin = 10000.0
        self.betaAng = 100.0
        self.alpha = 0.99
        self.gamma = 0.999

    def clear(self):
        self._builder = _scenes.SceneBuilder("solver", _scenes.Params())
        self._world = None
        self._cached = None

    def _params(self):
        return _scenes.Params(self.dt, self.gravity, self.iterations, self.alpha, self.betaLin, self.betaAng,
                              self.gamma, self.broadphaseMode)

    def _scene(self):
        self._builder.params = self._params()
        return self._builder.build()

    def _topology_changed(self):
        if self._world is not None:
            raise RuntimeError("adding bodies or forces after the first step needs a reload: call clear()")

    def _n_bodies(self):
        return len(self._builder.b["size"])

    def _state(self):
        if self._world is None:
            return None
        if self._cached is None:
            self._cached = self._world.bodies()
        return self._cached

    def step(self):
        """Solver::step -> physicsBackend->step(*this) (solver.cpp:934-937)."""
        self.physicsBackend.step(self)

    @property
    def world(self) -> World | None:
        return self._world
