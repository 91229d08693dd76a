"""CPU checks of the differentiable step's test infrastructure: the oracle's frozen-branch
tape, the FP64 replay, the FP64 reference adjoint and the VJP primitives they share with
the CUDA adjoint (avbd_demo3d_b200/csrc/avbd_diff.h)."""
from __future__ import annotations

import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import scenes


def _dynamic_mask(w, th):
    n = w.n
    d = w.body_props()["mass"] > 0
    m = np.zeros(th.size, bool)
    m[:3 * n] = np.repeat(d, 3)
    m[3 * n:6 * n] = np.repeat(d, 3)
    m[6 * n:7 * n] = d
    m[7 * n:] = True
    return m


def _recorded(scene, steps):
    w = checkers.World(scene, "oracle", order_mode=1)
    w.tape_begin()
    w.step(steps)
    return w


def _target(w, seed=0):
    b, p = w.bodies(), w.body_props()
    d = p["mass"] > 0
    com = (p["mass"][d, None] * b["pos"][d]).sum(0) / p["mass"][d].sum()
    return com + np.random.default_rng(seed).uniform(-1, 1, 3)


def test_vjp_primitives_match_central_differences():
    # rotate, qdiff, qstep, the 6x6 solve with contact rows, the dual update, warm start
    # and C0, each on random inputs; h = 1e-6 central differences
    assert checkers.adjoint_selftest() < 1e-4


def test_replay_tracks_the_fp32_run():
    w = _recorded(scenes.tower(3, 3, 4, seed=4), 40)
    assert w.tape_steps() == 40
    th = w.adj_theta0()
    _, pos = w.adj_loss(th, np.zeros(3))
    # same branches, double precision: the FP32 and FP64 trajectories stay close
    assert np.abs(pos - w.bodies()["pos"]).max() < 1e-4


@pytest.mark.parametrize("shape,steps", [((2, 2, 3), 30), ((3, 3, 4), 60)])
def test_reference_adjoint_matches_finite_differences(shape, steps):
    w = _recorded(scenes.tower(*shape, seed=4), steps)
    th = w.adj_theta0()
    target = _target(w)
    loss, g = w.adj_gradient(th, target)
    assert loss == pytest.approx(w.adj_loss(th, target)[0], rel=1e-12)
    rng = np.random.default_rng(1)
    dirs = rng.standard_normal((8, th.size)) * _dynamic_mask(w, th)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    fd = w.adj_fd(th, target, dirs, h=1e-4)
    ad = dirs @ g
    assert np.abs(ad - fd).max() <= 1e-5 * np.abs(fd).max()
    # each parameter block on its own
    n = w.n
    for sl in (slice(0, 3 * n), slice(3 * n, 6 * n), slice(6 * n, 7 * n), slice(7 * n, None)):
        d = np.zeros((1, th.size))
        d[0, sl] = rng.standard_normal(th[sl].size)
        d *= _dynamic_mask(w, th)
        d /= np.linalg.norm(d)
        f = w.adj_fd(th, target, d, h=1e-4)[0]
        a = float(d[0] @ g)
        # the friction block is small (most contacts stick): FD round-off ~1e-10 of the loss
        assert abs(a - f) <= 1e-4 * abs(f) + 1e-9


def test_static_parameters_have_no_gradient():
    w = _recorded(scenes.tower(2, 2, 2, seed=4), 10)
    th = w.adj_theta0()
    _, g = w.adj_gradient(th, _target(w))
    n = w.n
    static = w.body_props()["mass"] == 0
    assert static.any()
    assert np.all(g[:3 * n].reshape(n, 3)[static] == 0)
    assert np.all(g[6 * n:7 * n][static] == 0)


def test_pairs_are_sorted_and_carry_the_nominal_friction():
    w = _recorded(scenes.tower(2, 2, 3, seed=4), 5)
    lohi, mu = w.adj_pairs()
    keys = lohi[:, 0].astype(np.int64) << 32 | lohi[:, 1]
    assert np.all(np.diff(keys) > 0) and np.all(lohi[:, 0] < lohi[:, 1])
    f = w.body_props()["friction"]
    np.testing.assert_array_equal(mu, np.sqrt(f[lohi[:, 0]] * f[lohi[:, 1]]).astype(np.float32))


def test_tape_refuses_joints():
    w = checkers.World(scenes.rope(8), "oracle", order_mode=1)
    with pytest.raises(ValueError):
        w.tape_begin()
