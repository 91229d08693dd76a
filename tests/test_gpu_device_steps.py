"""Device-resident steps (AVBD_STEP_DEVICE, the default) against host-counted steps
(AVBD_STEP_HOST) and the oracle.

A device-resident step keeps its counts (manifolds, sequence numbers, colours) on the GPU
and issues all its launches without waiting. When a step cannot run as issued (new pairs
beyond the manifold buffers, a joint broken in the previous step, the grid's cell-count
cap) it stops on the device before changing anything, and the next call that waits for
the device redoes it on the host. Both forms give the same bits; these tests let steps
pile up unsynchronised between checkpoints so that stops and redos happen mid-queue."""
import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import World, scenes
from test_gpu_parity import assert_same_state, bits

pytestmark = pytest.mark.gpu

SCENES = {
    "stacks": lambda: scenes.stack_grid(6, 6, 8, seed=3),
    "mixed": lambda: scenes.mixed_drop(3000, 20, 12, 0.05, extent=(30, 30, 20), seed=5),
    "breakable": lambda: scenes.breakable(),
    "bridge": lambda: scenes.bridge(),
    "round_mix": lambda: scenes.round_mix(600, seed=11, cols=8),
    "sphere_pour": lambda: scenes.sphere_pour(1000),
}


def same_world(a: World, b: World, where: str):
    ba, bb = a.bodies(), b.bodies()
    for k in ba:
        assert np.array_equal(bits(ba[k]), bits(bb[k])), f"{where}: {k}"
    ma, mb = a.manifolds(), b.manifolds()
    for k in ("ab", "seq", "n", "keys", "stick"):
        assert np.array_equal(ma[k], mb[k]), f"{where}: manifold {k}"
    assert np.array_equal(bits(ma["contact"]), bits(mb["contact"])), f"{where}: contact rows"
    ja, jb = a.joints(), b.joints()
    assert np.array_equal(ja["ab"], jb["ab"]) and np.array_equal(bits(ja["state"]), bits(jb["state"])), where
    ca, na = a.colours()
    cb, nb = b.colours()
    assert na == nb and np.array_equal(ca, cb), f"{where}: colouring"


@pytest.mark.parametrize("name", sorted(SCENES))
def test_device_steps_equal_host_steps(gpu, name):
    sc = SCENES[name]()
    host = World(sc)
    host.set_step_mode(World.STEP_HOST)
    dev = World(sc)
    for s in range(1, 61):
        host.step(1)
        dev.step(1, sync=False)
        if s % 10 == 0:
            same_world(host, dev, f"{name} step {s}")
    st = dev.stats()
    assert st["device_steps"] >= 60
    assert host.stats()["device_steps"] == 0
    if name == "breakable":
        # a joint broke: the step after it stopped on the device and was redone on the host
        assert st["redone_steps"] > 0
    host.close()
    dev.close()


def test_small_manifold_headroom_redoes_steps_and_stays_exact(gpu):
    """With room for a single new manifold per step, the steps that create contacts stop on
    the device (together with every step queued after them) and are redone on the host;
    the world still equals the oracle bit for bit."""
    sc = scenes.stack_grid(6, 6, 8, seed=3)
    g = World(sc)
    g.set_manifold_headroom(1)
    o = checkers.World(sc, "oracle", order_mode=1)
    for s in range(1, 41):
        g.step(1, sync=False)
        o.step(1)
        if s % 5 == 0:
            assert_same_state(g, o, f"headroom step {s}")
    st = g.stats()
    assert st["redone_steps"] > 0 and st["device_steps"] >= 40
    g.close()


def test_batch_device_steps_equal_host_steps(gpu):
    """A batch of uneven worlds (stacks, chains, drop piles, round bodies) in both forms."""
    worlds = [scenes.stack_grid(3, 3, 5, seed=1), scenes.rope(12), scenes.mixed_drop(400, 4, 8, 0.05,
                                                                                     extent=(12, 12, 10), seed=2),
              scenes.round_mix(200, seed=4, cols=4), scenes.breakable()]
    host = World(worlds)
    host.set_step_mode(World.STEP_HOST)
    dev = World(worlds)
    for s in range(1, 41):
        host.step(1)
        dev.step(1, sync=False)
        if s % 8 == 0:
            same_world(host, dev, f"batch step {s}")
    host.close()
    dev.close()


def test_autotune_after_device_steps(gpu):
    """The autotuner times the per-colour primal on the last colouring, whose ranges a
    device-resident step hands to the host when it is confirmed; the world is unchanged by
    the trials and keeps stepping bit-exactly."""
    sc = scenes.stack_grid(6, 6, 8, seed=3)
    g = World(sc)
    o = checkers.World(sc, "oracle", order_mode=1)
    g.step(4)
    o.step(4)
    assert g.stats()["redone_steps"] == 0 and g.stats()["device_steps"] == 4
    best, us = g.autotune(2)
    assert len(us) == len(World.primal_variants()) and all(x > 0 for x in us)
    assert_same_state(g, o, "after autotune")
    for s in range(1, 6):
        g.step(1)
        o.step(1)
        assert_same_state(g, o, f"after autotune, step {s}")
    g.close()


def test_page_locked_caller_arrays(gpu):
    """Body state read into and written from page-locked caller arrays (direct DMA) equals
    the staged path for ordinary arrays, bit for bit, through a write / step / read loop."""
    import torch

    sc = scenes.stack_grid(6, 6, 8, seed=3)
    a, b = World(sc), World(sc)
    a.step(3)
    b.step(3)
    ref = a.bodies()
    keep = {k: torch.empty(v.shape, dtype=torch.float32, pin_memory=True) for k, v in ref.items()}
    pinned = {k: t.numpy() for k, t in keep.items()}
    b.bodies(out=pinned)
    for k in ref:
        assert np.array_equal(bits(pinned[k]), bits(ref[k])), k
    for s in range(5):
        plain = {k: v.copy() for k, v in ref.items()}
        plain["vel"][3] += np.float32(0.01)
        pinned["vel"][3] += np.float32(0.01)
        a.write_bodies(pos=plain["pos"], quat=plain["quat"], vel=plain["vel"], angvel=plain["angvel"],
                       prevvel=plain["prevvel"])
        b.write_bodies(pos=pinned["pos"], quat=pinned["quat"], vel=pinned["vel"], angvel=pinned["angvel"],
                       prevvel=pinned["prevvel"])
        a.step(1, sync=False)
        b.step(1, sync=False)
        ref = a.bodies()
        b.bodies(out=pinned)
        for k in ref:
            assert np.array_equal(bits(pinned[k]), bits(ref[k])), (s, k)
    a.close()
    b.close()
