"""The sorted-Morton LBVH broadphase mode (AVBD_BROADPHASE_LBVH) against the oracle's
uniform grid (solver.cpp:284-486): the tree only generates each grid entry's binned
candidates, so the new pairs, their creation order and everything after them equal the
grid's bit for bit. Checked after every step on stacks, drop piles with jointed chains and
springs, round shapes, a sphere pour, the grid's cell-cap path, a batch of worlds, and the
full 65,536-box benchmark scene."""
import copy

import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import World, scenes
from test_gpu_parity import assert_same_state

pytestmark = pytest.mark.gpu


def lbvh_world(sc):
    g = World(sc)
    p = copy.copy(sc.params)
    p.broadphase = scenes.BROADPHASE_LBVH
    g.set_params(p)
    return g


def lockstep_lbvh(sc, steps, every=1, sync=True):
    g = lbvh_world(sc)
    o = checkers.World(sc, "oracle", order_mode=1)
    for s in range(1, steps + 1):
        g.step(1, sync=sync)
        o.step(1)
        if s % every == 0 or s == steps:
            assert_same_state(g, o, f"{sc.name} (lbvh) step {s}")
    st = g.stats()
    g.close()
    return st


SCENES = {
    "stacks": lambda: scenes.stack_grid(6, 6, 8, seed=3),
    "stacks4096": lambda: scenes.stack_grid(16, 16, 16, seed=1),
    "mixed": lambda: scenes.mixed_drop(3000, 20, 12, 0.05, extent=(30, 30, 20), seed=5),
    "round_mix": lambda: scenes.round_mix(600, seed=11, cols=8),
    "sphere_pour": lambda: scenes.sphere_pour(1000),
    "pyramid20": lambda: scenes.pyramid(20),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_lbvh_equals_grid(gpu, name):
    st = lockstep_lbvh(SCENES[name](), 40)
    assert st["manifold_count"] > 0


def test_lbvh_device_steps_pile_up(gpu):
    """Unsynchronised device-resident steps in LBVH mode, checked every 10."""
    lockstep_lbvh(scenes.mixed_drop(3000, 20, 12, 0.05, extent=(30, 30, 20), seed=5), 60, every=10, sync=False)


def test_lbvh_grid_cell_cap_path(gpu):
    """A box flung at 30 km/s: the grid rescales its cells on the host; the tree follows."""
    sc = scenes.stack_grid(4, 4, 4, seed=12)
    sc.vel[5] = (3.0e4, 3.0e4, 3.0e4)
    lockstep_lbvh(sc, 20)


def test_lbvh_batch(gpu):
    worlds = [scenes.stack_grid(3, 3, 5, seed=1), scenes.rope(12),
              scenes.mixed_drop(400, 4, 8, 0.05, extent=(12, 12, 10), seed=2), scenes.round_mix(200, seed=4, cols=4)]
    grid = World(worlds)
    lb = World(worlds)
    p = copy.copy(worlds[0].params)
    p.broadphase = scenes.BROADPHASE_LBVH
    lb.set_params(p)
    for s in range(1, 31):
        grid.step(1)
        lb.step(1)
        if s % 5 == 0:
            bg, bl = grid.bodies(), lb.bodies()
            for k in bg:
                assert np.array_equal(bg[k].view(np.uint32), bl[k].view(np.uint32)), (s, k)
            mg, ml = grid.manifolds(), lb.manifolds()
            assert np.array_equal(mg["ab"], ml["ab"]) and np.array_equal(mg["seq"], ml["seq"]), s
    grid.close()
    lb.close()


@pytest.mark.slow
def test_lbvh_benchmark_scene(gpu):
    """The 65,536-box scene, 5 steps, bit-exact against the oracle's grid."""
    lockstep_lbvh(scenes.stack_grid(64, 64, 16, seed=1), 5)
