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


@pytest.mark.parametrize("mode", [scenes.BROADPHASE_ALL_PAIRS, scenes.BROADPHASE_SAP])
def test_other_broadphase_modes(mode):
    sc = scenes.stack_grid(5, 5, 6, seed=25)
    sc.params.broadphase = mode
    lockstep(sc, 40, False)


def test_narrowphase_random_pairs():
    import make_golden

    cases = make_golden.narrowphase_cases(n_random=300, seed=99)
    for i in range(cases[0].shape[0]):
        a = checkers.collide_boxes("oracle", *(c[i] for c in cases))
        b = checkers.collide_boxes("ref", *(c[i] for c in cases))
        assert a[0] == b[0] and np.array_equal(a[1], b[1]), i
        assert np.array_equal(bits(a[2]), bits(b[2])) and np.array_equal(bits(a[3]), bits(b[3])), i
