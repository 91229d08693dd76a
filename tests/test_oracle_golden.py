"""The CPU oracle against golden fixtures produced by the reference solver itself
(tests/golden/make_golden.py). Everything is compared bit for bit."""
import hashlib
import os

import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def digest(b):
    h = hashlib.sha256()
    for k in ("pos", "quat", "vel", "angvel", "prevvel"):
        h.update(np.ascontiguousarray(b[k]).tobytes())
    return np.frombuffer(h.digest(), dtype=np.uint8)


def test_pyramid_600_steps_bit_exact():
    g = np.load(os.path.join(GOLDEN, "pyramid20_ref.npz"))
    w = checkers.World(scenes.pyramid(20), "oracle")
    for s in range(1, 601):
        w.step(1)
        b = w.bodies()
        assert np.array_equal(digest(b), g["digests"][s - 1]), f"state digest differs at step {s}"
        assert np.array_equal(w.counters()[[0, 1, 2, 3, 4, 5]], g["counters"][s - 1]), f"counters differ at {s}"
        if s in (1, 10, 60, 120, 600):
            for k in ("pos", "quat", "vel", "angvel", "prevvel"):
                assert np.array_equal(bits(b[k]), bits(g[f"s{s}_{k}"])), (s, k)


def test_narrowphase_fixtures():
    g = np.load(os.path.join(GOLDEN, "narrowphase_ref.npz"))
    n_cases = g["pA"].shape[0]
    kinds = {"face": 0, "edge": 0, "none": 0}
    for i in range(n_cases):
        n, keys, rA, rB, basis = checkers.collide_boxes("oracle", g["pA"][i], g["qA"][i], g["sA"][i], g["pB"][i],
                                                        g["qB"][i], g["sB"][i])
        assert n == g["n"][i], i
        assert np.array_equal(keys, g["keys"][i]), i
        assert np.array_equal(bits(rA), bits(g["rA"][i])), i
        assert np.array_equal(bits(rB), bits(g["rB"][i])), i
        if n:
            assert np.array_equal(bits(basis), bits(g["basis"][i])), i
            kinds["edge" if (keys[0] >> 24) == 2 else "face"] += 1
        else:
            kinds["none"] += 1
    # the fixture exercises every branch
    assert kinds["face"] > 50 and kinds["edge"] > 5 and kinds["none"] > 5, kinds


@pytest.mark.parametrize("name", ["rope", "springs", "bridge", "breakable", "boxbox", "rotboxbox", "cluster",
                                  "stacks", "mixed"])
@pytest.mark.parametrize("order", ["list", "colour"])
def test_scene_60_steps(name, order):
    import make_golden  # noqa: E402  (tests/golden on sys.path below)

    g = np.load(os.path.join(GOLDEN, "scenes60_ref.npz"))
    sc = make_golden.golden_scenes()[name]
    w = checkers.World(sc, "oracle", order_mode=1 if order == "colour" else 0)
    w.step(60)
    b, m, j = w.bodies(), w.manifolds(), w.joints()
    p = f"{name}_{order}_"
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(bits(b[k]), bits(g[p + k])), k
    assert np.array_equal(m["ab"], g[p + "man_ab"])
    assert np.array_equal(m["n"], g[p + "man_n"])
    assert np.array_equal(m["keys"], g[p + "man_keys"])
    assert np.array_equal(bits(m["contact"]), bits(g[p + "man_contact"]))
    assert np.array_equal(bits(j["state"]), bits(g[p + "joint_state"]))
    assert np.array_equal(j["broken"], g[p + "joint_broken"])
