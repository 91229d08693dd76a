"""Failure paths of the step, made to happen without faulting the GPU.

* Bounded waits: the colouring's grid barrier and the iteration kernel's grid barriers
  and partner waits poll at most a set number of times (avbd_set_wait_limits). With a
  limit of one poll a multi-block launch cannot pass its first barrier, so the wait runs
  out: the kernel records it and every block returns. The step reports AVBD_ERR_STATE,
  the context latches (AVBD_ERR_LATCHED on the next step), and after avbd_clear_error,
  the default limits and a reload the same context steps bit-exactly again.
* Non-finite state: a NaN position or an infinite velocity written between steps makes
  the next step refuse to run (AVBD_ERR_STATE) before it changes anything, in both step
  forms; after the state is repaired the world continues bit-exactly.

The reference has no counterpart: its CPU solver never waits and propagates NaN silently
(its GPU lane reports failures on stderr and falls back to the CPU,
avbd_gpu_solver.cpp:2152-2170)."""
import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import World, _lib, scenes
from test_gpu_parity import assert_same_state, bits

pytestmark = pytest.mark.gpu

MODES = {"device": World.STEP_DEVICE, "host": World.STEP_HOST}


def step_status(w: World) -> int:
    """Status of one step as the caller sees it: the step call, or the wait after it."""
    rc = w.lib.avbd_step(w.h, 1)
    if rc == _lib.AVBD_OK:
        rc = w.lib.avbd_synchronize(w.h)
    return rc


def recovers_bit_exact(w: World, sc, steps=10):
    """After clear_error, default limits and a reload: lockstep with a fresh oracle."""
    w.clear_error()
    w.set_wait_limits(0, 0)
    w.reload()
    o = checkers.World(sc, "oracle", order_mode=1)
    for s in range(1, steps + 1):
        w.step(1)
        o.step(1)
        assert_same_state(w, o, f"after recovery, step {s}")


@pytest.mark.parametrize("mode", sorted(MODES))
def test_iteration_wait_expiry_fails_latches_and_recovers(gpu, mode):
    sc = scenes.stack_grid(8, 8, 8, seed=3)  # 512 boxes, several colours, 148 blocks
    w = World(sc)
    w.set_step_mode(MODES[mode])
    w.step(3)
    w.set_wait_limits(0, 1)
    assert step_status(w) == _lib.AVBD_ERR_STATE
    assert "iteration kernel wait expired" in w.last_error()
    assert w.lib.avbd_step(w.h, 1) == _lib.AVBD_ERR_LATCHED
    recovers_bit_exact(w, sc)
    w.close()


@pytest.mark.parametrize("mode", sorted(MODES))
def test_colouring_wait_expiry_fails_latches_and_recovers(gpu, mode):
    sc = scenes.stack_grid(8, 8, 8, seed=3)  # more than 256 bodies: a multi-block colouring
    w = World(sc)
    w.set_step_mode(MODES[mode])
    w.step(3)
    w.set_wait_limits(1, 0)
    assert step_status(w) == _lib.AVBD_ERR_STATE
    assert "colouring did not finish" in w.last_error()
    assert w.lib.avbd_step(w.h, 1) == _lib.AVBD_ERR_LATCHED
    recovers_bit_exact(w, sc)
    w.close()


def test_wait_expiry_in_a_world_with_joints(gpu):
    """Worlds with joints take a grid barrier after every colour: that barrier runs out."""
    sc = scenes.mixed_drop(3000, 20, 12, 0.05, extent=(30, 30, 20), seed=5)
    w = World(sc)
    w.step(2)
    w.set_wait_limits(0, 1)
    assert step_status(w) == _lib.AVBD_ERR_STATE
    recovers_bit_exact(w, sc, steps=5)
    w.close()


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("field", ["pos", "vel"])
def test_non_finite_state_is_refused_before_anything_changes(gpu, mode, field):
    sc = scenes.stack_grid(6, 6, 8, seed=3)
    w = World(sc)
    w.set_step_mode(MODES[mode])
    o = checkers.World(sc, "oracle", order_mode=1)
    w.step(5)
    o.step(5)
    before, mbefore = w.bodies(), w.manifolds()
    bad = before[field].copy()
    bad[7, 2] = np.nan if field == "pos" else np.inf
    w.write_bodies(**{field: bad})
    assert step_status(w) == _lib.AVBD_ERR_STATE
    assert "non-finite" in w.last_error()
    assert w.lib.avbd_step(w.h, 1) == _lib.AVBD_ERR_LATCHED
    w.clear_error()
    after, mafter = w.bodies(), w.manifolds()
    for k in before:
        want = bad if k == field else before[k]
        assert np.array_equal(bits(after[k]), bits(want)), k
    for k in ("ab", "seq", "n", "keys"):
        assert np.array_equal(mafter[k], mbefore[k]), k
    assert np.array_equal(bits(mafter["contact"]), bits(mbefore["contact"]))
    w.write_bodies(**{field: before[field]})
    for s in range(1, 11):
        w.step(1)
        o.step(1)
        assert_same_state(w, o, f"after repair, step {s}")
    w.close()
