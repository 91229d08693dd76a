"""The double-precision build of the reference (oracle/make_fp64.py + ref64_driver.cpp),
the yardstick that every result's error is stated against.

The single-precision solve is chaotic: its distance from the FP64 solve grows to about a
centimetre within ten steps on the 210-box pyramid and then stays there, for the
reference's own CPU solver as much as for this build. The GPU equals the oracle swept in
colour order bit for bit (the -m gpu parity tests), so the oracle's error against FP64
here is the GPU's."""
import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import scenes

pytestmark = pytest.mark.skipif(not (checkers.ref_available() and checkers.ref64_available()),
                                reason="reference libraries not built (make -C oracle ref ref64)")


def test_fp64_build_is_double_and_starts_where_fp32_does():
    sc = scenes.pyramid(20)
    r64 = checkers.Fp64Reference(sc)
    assert r64.lib.ref64_is_double() == 1
    b = r64.bodies()
    assert b["pos"].dtype == np.float64
    # before the first step: the single-precision reference's state, widened exactly
    r = checkers.World(sc, "ref")
    b32 = r.bodies()
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(b[k], b32[k].astype(np.float64)), k
    r.close()
    r64.close()


def test_pyramid_fp32_vs_fp64_matches_the_survey_probe():
    """FP32 reference against its FP64 build on the 210-box benchmark pyramid: 6.0e-7 m
    after one step, about 1.1e-2 m at step 10 and 1.3e-2 m at step 60 (the figures measured
    when the reference was surveyed)."""
    sc = scenes.pyramid(20)
    r, r64 = checkers.World(sc, "ref"), checkers.Fp64Reference(sc)
    got = {}
    done = 0
    for m in (1, 10, 60):
        r.step(m - done)
        r64.step(m - done)
        done = m
        got[m] = checkers.pose_error(r.bodies(), r64.bodies())
    assert 1e-8 < got[1][0] < 2e-6, got
    assert 3e-3 < got[10][0] < 3e-2, got
    assert 3e-3 < got[60][0] < 3e-2, got


def test_colour_order_solve_error_against_fp64_is_the_references_own():
    """Over the pyramid's 600 steps, the colour-order solve (what the GPU computes, bit for
    bit) is as far from FP64 as the reference's own list-order FP32 solve is: within 2x +
    1 mm at every checkpoint. Prints the figures (AVBD_ERR lines)."""
    sc = scenes.pyramid(20)
    o = checkers.World(sc, "oracle", order_mode=1)
    r, r64 = checkers.World(sc, "ref"), checkers.Fp64Reference(sc)
    done = 0
    for m in (10, 60, 600):
        for w in (o, r, r64):
            w.step(m - done)
        done = m
        gp, gq = checkers.pose_error(o.bodies(), r64.bodies())
        rp, rq = checkers.pose_error(r.bodies(), r64.bodies())
        print(f"AVBD_ERR pyramid20 step {m} | colour_order_vs_fp64 pos {gp:.3e} m rot {gq:.3e} rad | "
              f"ref32_vs_fp64 pos {rp:.3e} m rot {rq:.3e} rad")
        assert gp <= 2 * rp + 1e-3, (m, gp, rp)
