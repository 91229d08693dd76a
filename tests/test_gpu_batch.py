"""Batched worlds: many independent worlds in one context, stepped by one launch sequence
per step. Every world must evolve bit for bit as the oracle evolves it alone (each world
keeps its own broadphase grid, colouring and force order)."""
import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import World, scenes

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def per_world(arr, ws, w):
    return arr[ws[w]:ws[w + 1]]


@pytest.mark.parametrize("mode", [scenes.BROADPHASE_GRID, scenes.BROADPHASE_SAP])
def test_uneven_batch_matches_each_world_alone(gpu, mode):
    worlds = scenes.batched_worlds(24, seed=11, lo=8, hi=160)
    for sc in worlds:
        sc.params.broadphase = mode  # one sweep axis (or grid) per world
    g = World(worlds)
    oracles = [checkers.World(sc, "oracle", order_mode=1) for sc in worlds]
    ws = g.world_start
    for step in range(1, 41):
        g.step(1)
        for o in oracles:
            o.step(1)
        if step % 10:
            continue
        b = g.bodies()
        col, _ = g.colours()
        m = g.manifolds()
        for w, o in enumerate(oracles):
            ob = o.bodies()
            for k in ("pos", "quat", "vel", "angvel"):
                assert np.array_equal(bits(per_world(b[k], ws, w)), bits(ob[k])), (step, w, k)
            oc, _ = o.colours()
            assert np.array_equal(per_world(col, ws, w), oc), (step, w, "colours")
            sel = (m["ab"][:, 0] >= ws[w]) & (m["ab"][:, 0] < ws[w + 1])
            om = o.manifolds()
            assert np.array_equal(m["ab"][sel] - ws[w], om["ab"]), (step, w, "pairs")
            assert np.array_equal(m["keys"][sel], om["keys"]), (step, w, "keys")
            assert np.array_equal(bits(m["contact"][sel]), bits(om["contact"])), (step, w, "contacts")
    g.close()


def test_batch_of_identical_worlds_is_identical(gpu):
    """The same scene repeated: every copy ends bit-identical (no cross-world coupling)."""
    sc = scenes.stack_grid(4, 4, 6, seed=5)
    g = World([sc] * 5)
    g.step(30)
    b = g.bodies()["pos"].reshape(5, sc.n_bodies, 3)
    for w in range(1, 5):
        assert np.array_equal(bits(b[0]), bits(b[w]))
    g.close()


def test_batch_with_round_worlds(gpu):
    """Box-only and round-shape worlds in one batch: the round kernel instances serve every
    world, and each world still evolves as the oracle evolves it alone."""
    worlds = [scenes.round_mix(120, seed=31, cols=4), scenes.stack_grid(3, 3, 5, seed=7),
              scenes.sphere_pour(200, seed=17), scenes.pyramid(8)]
    g = World(worlds)
    oracles = [checkers.World(sc, "oracle", order_mode=1) for sc in worlds]
    ws = g.world_start
    for step in range(1, 31):
        g.step(1)
        for o in oracles:
            o.step(1)
        if step % 10:
            continue
        b = g.bodies()
        for w, o in enumerate(oracles):
            ob = o.bodies()
            for k in ("pos", "quat", "vel", "angvel"):
                assert np.array_equal(bits(per_world(b[k], ws, w)), bits(ob[k])), (step, w, k)
    g.close()
