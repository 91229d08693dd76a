"""C ABI behaviour on the GPU: argument checking, error latching, state round trips,
and the reference-style object interface."""
import ctypes

import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import IgnoreCollision, Joint, Rigid, Solver, Spring, World, _lib, scenes

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_invalid_arguments_are_reported(gpu):
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.avbd_create(ctypes.byref(h), 0, None) == 0
    assert lib.avbd_step(h, 1) == -4  # no world loaded
    assert b"no world" in lib.avbd_last_error(h)
    lib.avbd_clear_error(h)
    bad = _lib.AvbdParams(0.0, -10.0, 10, 0.99, 1e4, 100.0, 0.999, 1)
    assert lib.avbd_set_params(h, ctypes.byref(bad)) == -1
    lib.avbd_clear_error(h)
    unknown = _lib.AvbdParams(1 / 60, -10.0, 10, 0.99, 1e4, 100.0, 0.999, 7)  # no such broadphase mode
    assert lib.avbd_set_params(h, ctypes.byref(unknown)) == -1
    lib.avbd_clear_error(h)
    sap = _lib.AvbdParams(1 / 60, -10.0, 10, 0.99, 1e4, 100.0, 0.999, 2)  # sweep and prune
    assert lib.avbd_set_params(h, ctypes.byref(sap)) == 0
    lib.avbd_destroy(h)


def test_bad_joint_indices_rejected_and_error_latches(gpu):
    sc = scenes.rope(5)
    sc.fb[0] = 999  # body out of range
    with pytest.raises(_lib.AvbdError):
        World(sc)
    # the same through the C ABI directly: rejected, error latched until cleared
    w = World(scenes.rope(5))
    ab = np.array([[0, 99]], np.int32)
    seq = np.zeros(1, np.int64)
    st = np.zeros((1, 28), np.float32)
    P = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    props = w._body_arrays
    bodies = _lib.AvbdBodies(w.n, *[P(props[k]) for k in ("position3", "orientation4", "velocity3", "angular3",
                                                           "prev_velocity3", "size3", "mass", "moment3", "friction",
                                                           "radius")])
    joints = _lib.AvbdJoints(1, P(ab), P(seq), P(st), None)
    rc = w.lib.avbd_load_world(w.h, ctypes.byref(bodies), ctypes.byref(joints), None, None, None, 1)
    assert rc == -1 and b"joint" in w.lib.avbd_last_error(w.h)
    assert w.lib.avbd_step(w.h, 1) == -5  # latched
    w.lib.avbd_clear_error(w.h)


def test_world_reload_from_readback_continues_identically(gpu):
    """Checkpoint/restore: read the full state back, load it into a new context, and the
    continued run matches an uninterrupted one bit for bit."""
    sc = scenes.mixed_drop(1500, 10, 12, 0.1, extent=(24, 24, 16), seed=8)
    a = World(sc)
    a.step(40)
    b_state, m, j = a.bodies(), a.manifolds(), a.joints()
    nseq = ctypes.c_int64()
    a.lib.avbd_next_seq(a.h, ctypes.byref(nseq))
    b = World(sc)
    props = b._body_arrays
    arrs = dict(position3=b_state["pos"], orientation4=b_state["quat"], velocity3=b_state["vel"],
                angular3=b_state["angvel"], prev_velocity3=b_state["prevvel"])
    arrs = {k: np.ascontiguousarray(v) for k, v in arrs.items()}
    P = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    bodies = _lib.AvbdBodies(sc.n_bodies, P(arrs["position3"]), P(arrs["orientation4"]), P(arrs["velocity3"]),
                             P(arrs["angular3"]), P(arrs["prev_velocity3"]), P(props["size3"]), P(props["mass"]),
                             P(props["moment3"]), P(props["friction"]), P(props["radius"]))
    fa = b._force_arrays
    jst = np.ascontiguousarray(j["state28"])
    joints = _lib.AvbdJoints(len(j["ab"]), P(np.ascontiguousarray(j["ab"])), P(np.ascontiguousarray(j["seq"])),
                             P(jst), P(np.ascontiguousarray(j["broken"])))
    springs = _lib.AvbdSprings(len(fa["s_ab"]), P(fa["s_ab"]), P(fa["s_seq"]), P(fa["s_state"]))
    ignores = _lib.AvbdIgnores(0)
    man = {k: np.ascontiguousarray(v) for k, v in m.items()}
    manifolds = _lib.AvbdManifolds(len(man["n"]), *[P(man[k]) for k in ("ab", "seq", "n", "basis", "friction", "keys",
                                                                         "contact", "stick")])
    b._check(b.lib.avbd_load_world(b.h, ctypes.byref(bodies), ctypes.byref(joints), ctypes.byref(springs),
                                   ctypes.byref(ignores), ctypes.byref(manifolds), nseq.value), "reload")
    a.step(30)
    b.step(30)
    ba, bb = a.bodies(), b.bodies()
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(bits(ba[k]), bits(bb[k])), k


def test_write_bodies_between_steps(gpu):
    sc = scenes.stack_grid(4, 4, 4, seed=2)
    g = World(sc)
    o = checkers.World(sc, "oracle", order_mode=1)
    g.step(5)
    o.step(5)
    st = o.bodies()
    kick = st["vel"].copy()
    kick[:, 0] += np.float32(0.5)
    g.write_bodies(vel=kick)
    o.lib.oracle_set_bodies(o.h, None, None, kick.ctypes.data_as(ctypes.c_void_p), None, None)
    g.step(10)
    o.step(10)
    assert np.array_equal(bits(g.bodies()["pos"]), bits(o.bodies()["pos"]))


def test_bodies_into_caller_arrays(gpu):
    """bodies(out=...) fills the caller's arrays in place with what bodies() returns, and
    refuses arrays of the wrong shape, type or layout."""
    sc = scenes.stack_grid(3, 3, 4, seed=6)
    g = World(sc)
    g.step(4)
    ref = g.bodies(aux=True)
    out = {k: np.full_like(v, np.nan) for k, v in ref.items()}
    same = g.bodies(out=out)
    assert same is out
    for k in ref:
        assert np.array_equal(bits(out[k]), bits(ref[k])), k
    part = {"quat": np.zeros((g.n, 4), np.float32)}
    g.bodies(out=part)
    assert np.array_equal(bits(part["quat"]), bits(ref["quat"]))
    for bad in ({"pos": np.zeros((g.n, 4), np.float32)}, {"pos": np.zeros((g.n, 3), np.float64)},
                {"pos": np.zeros((3, g.n), np.float32).T}, {"spin": np.zeros((g.n, 3), np.float32)}):
        with pytest.raises(ValueError):
            g.bodies(out=bad)
    g.close()


def test_reference_style_interface(gpu):
    """Scenes built with the mirrored constructors step on the GPU like the oracle."""
    solver = Solver()
    solver.gravity = -9.81
    Rigid(solver, (100, 100, 1), 0.0, 0.5, (0, 0, -0.5))
    prev = None
    for i in range(6):
        cur = Rigid(solver, (1, 0.5, 0.5), 1.0, 0.5, (float(i), 0.0, 3.0))
        if prev is not None:
            Joint(solver, prev, cur, (0.5, 0, 0), (-0.5, 0, 0))
        prev = cur
    a = Rigid(solver, (1, 1, 1), 1.0, 0.5, (4.0, 3.0, 2.0))
    bb = Rigid(solver, (1, 1, 1), 1.0, 0.5, (4.0, 5.0, 2.0))
    Spring(solver, a, bb, (0, 0, 0), (0, 0, 0), 500.0)
    IgnoreCollision(solver, a, bb)
    assert solver.physicsBackend.name().startswith("CUDA AVBD")
    scene = solver._scene()
    o = checkers.World(scene, "oracle", order_mode=1)
    for _ in range(30):
        solver.step()
        o.step(1)
    assert np.array_equal(bits(solver.world.bodies()["pos"]), bits(o.bodies()["pos"]))
    z = a.positionLin[2]
    assert z < 2.0  # fell under gravity
