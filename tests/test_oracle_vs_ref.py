"""Live lockstep of the oracle against the reference compiled from its own sources.
Skipped where the prebuilt reference library is absent."""
import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import scenes

pytestmark = pytest.mark.skipif(not checkers.ref_available(), reason="reference library not built")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def lockstep(sc, steps, colour):
    o = checkers.World(sc, "oracle", order_mode=1 if colour else 0)
    r = checkers.World(sc, "ref")
    for s in range(steps):
        if colour:
            o.prepare()
            r.prepare()
            r.iterate_ordered(o.solve_order())
            o.iterate()
            o.finish()
            r.finish()
        else:
            o.step(1)
            r.step(1)
        bo, br = o.bodies(), r.bodies()
        for k in bo:
            assert np.array_equal(bits(bo[k]), bits(br[k])), (sc.name, s + 1, k)
    mo, mr = o.manifolds(), r.manifolds()
    assert np.array_equal(mo["ab"], mr["ab"]) and np.array_equal(mo["keys"], mr["keys"])
    assert np.array_equal(bits(mo["contact"]), bits(mr["contact"]))
    assert np.array_equal(o.counters()[:7], r.counters()[:7])


@pytest.mark.parametrize("colour", [False, True])
def test_stacks(colour):
    lockstep(scenes.stack_grid(8, 8, 8, seed=21), 40, colour)


@pytest.mark.parametrize("colour", [False, True])
def test_mixed_constraints(colour):
    lockstep(scenes.mixed_drop(2000, 12, 10, 0.1, extent=(26, 26, 18), seed=23), 50, colour)


@pytest.mark.parametrize("colour", [False, True])
@pytest.mark.parametrize("scene", ["round_mix", "sphere_pour"])
def test_round_shapes(scene, colour):
    """Spheres, capsules and cylinders (rigid.cpp:44-90, collision.cpp round paths) with
    rolling friction: the same bodies, manifolds and counters as the reference."""
    sc = scenes.round_mix(300, seed=11, cols=6) if scene == "round_mix" else scenes.sphere_pour(300)
    lockstep(sc, 60, colour)


def test_sphere_pour_2000_colour_order():
    """2,000 spheres poured among static cylinders: many simultaneous sphere-sphere and
    sphere-cylinder contacts with rolling friction, in the GPU's colour order."""
    lockstep(scenes.sphere_pour(2000), 120, True)  # the pour lands after about 40 steps


def test_round_mix_long_horizon():
    """Spheres, capsules and cylinders settling on static cylinders and a raised slab for
    200 steps in list order: the trajectory stays bit-identical well past the impacts."""
    lockstep(scenes.round_mix(400, seed=17, cols=8), 200, False)


def test_round_body_properties_match_reference():
    """Mass and shape fields of round bodies as the reference's SimWorld holds them."""
    sc = scenes.round_mix(200, seed=19, cols=5)
    o = checkers.World(sc, "oracle", order_mode=0)
    r = checkers.World(sc, "ref")
    wb, pr = r.world_bodies(), o.body_props()
    n = sc.n_bodies
    assert np.array_equal(wb["shape"], np.asarray(sc.shape, np.int32))
    assert np.array_equal(bits(wb["mass"]), bits(pr["mass"][::-1]))
    rnd = np.asarray(sc.shape) != 0
    assert np.array_equal(bits(wb["radius"][rnd]), bits(np.asarray(sc.dims, np.float32)[rnd, 0]))
    assert np.array_equal(bits(wb["half_length"][rnd]), bits(np.asarray(sc.dims, np.float32)[rnd, 1]))
    assert len(wb["active"]) == n


@pytest.mark.parametrize("mode", [scenes.BROADPHASE_ALL_PAIRS, scenes.BROADPHASE_SAP])
def test_other_broadphase_modes(mode):
    sc = scenes.stack_grid(5, 5, 6, seed=25)
    sc.params.broadphase = mode
    lockstep(sc, 40, False)


@pytest.mark.parametrize("mode", [scenes.BROADPHASE_GRID, scenes.BROADPHASE_SAP, scenes.BROADPHASE_ALL_PAIRS])
@pytest.mark.parametrize("world", ["boxes", "round"])
def test_broadphase_only_matches_reference(mode, world):
    """Solver::benchmarkBroadphaseOnly after some steps: same new pairs, same counters, and
    the next steps (which initialise the new manifolds) stay bit-identical. Round bodies
    enter the broadphase with bounds from their shape radius."""
    sc = (scenes.mixed_drop(1500, 8, 10, 0.1, extent=(22, 22, 14), seed=29) if world == "boxes"
          else scenes.round_mix(500, seed=23, cols=8))
    sc.params.broadphase = mode
    o = checkers.World(sc, "oracle", order_mode=0)
    r = checkers.World(sc, "ref")
    o.step(30)
    r.step(30)
    o.broadphase_only()
    r.broadphase_only()
    mo, mr = o.manifolds(), r.manifolds()
    assert len(mo["ab"]) > 0 and np.array_equal(mo["ab"], mr["ab"])
    assert np.all(mo["n"] == 0) and np.all(mr["n"] == 0)
    assert np.array_equal(o.counters()[:5], r.counters()[:5])
    for _ in range(5):
        o.step(1)
        r.step(1)
    bo, br = o.bodies(), r.bodies()
    for k in bo:
        assert np.array_equal(bits(bo[k]), bits(br[k])), k


def _drag_script(w, props, steps=60):
    """SimulationHost's drag between steps: beginDrag (a world-anchored Joint, stiffness 5000,
    0), updateDrag moving the anchor every step, a body-body joint added on the way,
    releaseDrag, then a few free steps. Yields after every step."""
    b = int(np.flatnonzero(props["mass"] > 0)[-1])
    pos = w.bodies()["pos"][b].astype(np.float64)
    local = np.array([0.1, -0.05, 0.2], np.float32)
    h = w.add_joint(-1, b, pos.astype(np.float32), local, 5000.0, 0.0)
    link = None
    for s in range(steps):
        target = (pos + np.array([0.05 * s, 0.02 * s, 0.04 * s])).astype(np.float32)
        w.set_joint_anchor(h, target)
        if s == 20:
            link = w.add_joint(b, b - 1, [0.0, 0.5, 0.0], [0.0, -0.5, 0.0], float("inf"), 100.0, 1e4)
        if s == 40:
            w.remove_joint(link)
        w.step(1)
        yield s
    w.remove_joint(h)
    for s in range(10):
        w.step(1)
        yield steps + s


@pytest.mark.parametrize("world", ["boxes", "round"])
def test_drag_edits_match_reference(world):
    """Joint edits between steps (drag begin / move / release, a body-body joint added and
    deleted) keep the oracle bit-identical to the reference, on boxes and on round bodies."""
    sc = (scenes.mixed_drop(1200, 8, 10, 0.1, extent=(20, 20, 14), seed=31) if world == "boxes"
          else scenes.round_mix(400, seed=29, cols=8))
    o = checkers.World(sc, "oracle", order_mode=0)
    r = checkers.World(sc, "ref")
    o.step(20)
    r.step(20)
    props = o.body_props()
    for so, sr in zip(_drag_script(o, props), _drag_script(r, props)):
        assert so == sr
        bo, br = o.bodies(), r.bodies()
        for k in bo:
            assert np.array_equal(bits(bo[k]), bits(br[k])), (so, k)
        jo, jr = o.joints(), r.joints()
        assert np.array_equal(jo["ab"], jr["ab"]) and np.array_equal(bits(jo["state"]), bits(jr["state"])), so


def test_snapshot_fields_match_reference_world():
    """The viewer-bridge snapshot of the oracle's state (dense id = creation rank, shape box,
    full size, bounding radius, half length 0) is byte-identical to the one assembled from the
    reference's own SimWorld, and the viewer's decoder reads it back."""
    sc = scenes.mixed_drop(900, 6, 8, 0.1, extent=(18, 18, 12), seed=37)
    o = checkers.World(sc, "oracle", order_mode=0)
    r = checkers.World(sc, "ref")
    o.step(25)
    r.step(25)
    wb = r.world_bodies()
    n = sc.n_bodies
    assert len(wb["active"]) == n and wb["active"].all()
    assert np.array_equal(wb["list_index"], n - 1 - np.arange(n))  # dense id = creation rank
    ref = checkers.snapshot_fields(np.arange(n), wb["shape"], wb["mass"], wb["pos"], wb["quat"], wb["size"],
                                   wb["radius"], wb["half_length"])
    ob, pr = o.bodies(), o.body_props()
    mine = checkers.snapshot_fields(n - 1 - np.arange(n), np.zeros(n, np.int32), pr["mass"], ob["pos"], ob["quat"],
                                    pr["size"], pr["radius"], np.zeros(n, np.float32))
    blob = checkers.encode_snapshot(1234, "Mixed", ref)
    assert blob == checkers.encode_snapshot(1234, "Mixed", mine)
    assert len(blob) == 24 + 5 + 64 * n
    assert checkers.snapshot_json(1234, "Mixed", ref) == checkers.snapshot_json(1234, "Mixed", mine)
    dec = checkers.decode_snapshot(blob)
    assert dec["frame"] == 1234 and dec["scene"] == "Mixed" and [b["id"] for b in dec["bodies"]] == list(range(n))
    assert all(np.array_equal(b["pos"], f["pos"]) and b["material"] == f["material"]
               for b, f in zip(dec["bodies"], ref))


def test_round_snapshot_matches_reference_world():
    """Snapshot of a world with round bodies: shape codes, sphere/cylinder/capsule materials,
    shape radius and half length as the reference's SimWorld reports them."""
    sc = scenes.round_mix(150, seed=41, cols=5)
    o = checkers.World(sc, "oracle", order_mode=0)
    r = checkers.World(sc, "ref")
    o.step(20)
    r.step(20)
    wb = r.world_bodies()
    n = sc.n_bodies
    ref = checkers.snapshot_fields(np.arange(n), wb["shape"], wb["mass"], wb["pos"], wb["quat"], wb["size"],
                                   wb["radius"], wb["half_length"])
    ob, pr = o.bodies(), o.body_props()
    shape = np.asarray(sc.shape, np.int32)[::-1]
    dims = np.asarray(sc.dims, np.float32)[::-1]
    rnd = shape != 0
    radius = np.where(rnd, dims[:, 0], pr["radius"]).astype(np.float32)
    half = np.where(rnd, dims[:, 1], 0).astype(np.float32)
    mine = checkers.snapshot_fields(n - 1 - np.arange(n), shape, pr["mass"], ob["pos"], ob["quat"], pr["size"],
                                    radius, half)
    assert {b["shape"] for b in ref} == {0, 1, 2, 3}
    assert checkers.encode_snapshot(7, "Round", ref) == checkers.encode_snapshot(7, "Round", mine)
    assert checkers.snapshot_json(7, "Round", ref) == checkers.snapshot_json(7, "Round", mine)


def test_narrowphase_random_pairs():
    import make_golden

    cases = make_golden.narrowphase_cases(n_random=300, seed=99)
    for i in range(cases[0].shape[0]):
        a = checkers.collide_boxes("oracle", *(c[i] for c in cases))
        b = checkers.collide_boxes("ref", *(c[i] for c in cases))
        assert a[0] == b[0] and np.array_equal(a[1], b[1]), i
        assert np.array_equal(bits(a[2]), bits(b[2])) and np.array_equal(bits(a[3]), bits(b[3])), i


def _greedy_order(w, n, sc):
    """Sequential greedy colouring in list order, computed independently in Python."""
    m, j = w.manifolds(), w.joints()
    mass = w.body_props()["mass"]
    adj = [[] for _ in range(n)]
    deg = np.zeros(n, int)
    sp = sc.ftype == scenes.FORCE_SPRING
    springs = [(n - 1 - a, n - 1 - b) for a, b in zip(sc.fa[sp], sc.fb[sp])]
    for a, b in [tuple(x) for x in m["ab"]] + [tuple(x) for x in j["ab"]] + springs:
        if a >= 0:
            deg[a] += 1
        deg[b] += 1
        if a >= 0 and mass[a] > 0 and mass[b] > 0:
            adj[a].append(b)
            adj[b].append(a)
    col = -np.ones(n, int)
    for v in range(n):
        if mass[v] <= 0 or deg[v] == 0:
            continue
        used = {col[u] for u in adj[v] if col[u] >= 0}
        c = 0
        while c in used:
            c += 1
        col[v] = c
    return np.array([v for c in range(col.max() + 1) for v in range(n) if col[v] == c], np.int32)


def test_colour_mode_1_is_greedy_list_order():
    """Jones-Plassmann with list-index priority equals sequential greedy colouring."""
    for sc in (scenes.reference_pyramid(16), scenes.bridge(), scenes.mixed_drop(1500, 10, 12, 0.05,
                                                                               extent=(24, 24, 16), seed=5)):
        o = checkers.World(sc, "oracle", order_mode=1)
        for _ in range(20):
            o.prepare()
            assert np.array_equal(o.solve_order(), _greedy_order(o, sc.n_bodies, sc)), sc.name
            o.iterate()
            o.finish()
