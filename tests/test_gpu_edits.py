"""Joint edits between steps on the GPU (SimulationHost's drag: a world-anchored joint added,
its anchor moved every step, deleted; simulation_host.cpp:242-274), against the oracle doing
the same edits, bit for bit after every step. The oracle's edits are themselves checked
against the reference in test_oracle_vs_ref.py."""
import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import World, scenes
from avbd_demo3d_b200 import _lib
from test_gpu_parity import assert_same_state

pytestmark = pytest.mark.gpu


def drag_script(w, props, steps=60):
    """beginDrag on the last dynamic body (stiffness 5000, 0), updateDrag every step, a
    body-body joint added at step 20 and deleted at step 40, releaseDrag, ten free steps."""
    b = int(np.flatnonzero(props["mass"] > 0)[-1])
    pos = w.bodies()["pos"][b].astype(np.float64)
    h = w.add_joint(-1, b, pos.astype(np.float32), np.array([0.1, -0.05, 0.2], np.float32), 5000.0, 0.0)
    link = None
    for s in range(steps):
        w.set_joint_anchor(h, (pos + np.array([0.05 * s, 0.02 * s, 0.04 * s])).astype(np.float32))
        if s == 20:
            link = w.add_joint(b, b - 1, [0.0, 0.5, 0.0], [0.0, -0.5, 0.0], float("inf"), 100.0, 1e4)
        if s == 40:
            w.remove_joint(link)
        w.step(1)
        yield s, h, link
    w.remove_joint(h)
    for s in range(10):
        w.step(1)
        yield steps + s, h, link


@pytest.mark.parametrize("name", ["mixed", "stacks"])
def test_drag_edits_bit_exact(gpu, name):
    sc = (scenes.mixed_drop(1200, 8, 10, 0.1, extent=(20, 20, 14), seed=31) if name == "mixed"
          else scenes.stack_grid(4, 4, 6, seed=33))
    g = World(sc)
    o = checkers.World(sc, "oracle", order_mode=1)
    g.step(20)
    o.step(20)
    assert_same_state(g, o, "before the drag")
    props = o.body_props()
    for (sg, hg, lg), (so, ho, lo) in zip(drag_script(g, props), drag_script(o, props)):
        assert sg == so and hg == ho and lg == lo, "sequence numbers of the added joints differ"
        assert_same_state(g, o, f"{name} drag step {sg}")
    assert g.next_seq() > hg
    g.close()


def test_edit_errors_leave_the_world_unchanged(gpu):
    sc = scenes.mixed_drop(400, 6, 6, 0.1, extent=(14, 14, 10), seed=35)
    g = World(sc)
    g.step(5)
    before_j, before_b = g.joints(), g.bodies()
    lib, h = g.lib, g.h

    def rejected(fn, *args):
        with pytest.raises(_lib.AvbdError):
            fn(*args)
        lib.avbd_clear_error(h)

    seq = int(before_j["seq"][0])
    rejected(g.remove_joint, g.next_seq() + 7)                  # names no joint
    st = before_j["state28"][:1].copy()
    rejected(g.write_joints, before_j["ab"][:1][:, ::-1], before_j["seq"][:1], st)  # bodies differ
    rejected(g.write_joints, np.repeat(before_j["ab"][:1], 2, 0), [seq, seq], np.repeat(st, 2, 0))  # repeated
    # a sequence number below the next one would not make the joint the newest force
    rejected(g._edit_joints, "avbd_add_joints", np.array([[-1, 3]], np.int32), np.array([seq], np.int64), st)
    rejected(g._edit_joints, "avbd_add_joints", np.array([[3, 3]], np.int32), np.array([g.next_seq()], np.int64), st)
    after_j, after_b = g.joints(), g.bodies()
    for k in ("ab", "seq", "state28", "broken"):
        assert np.array_equal(before_j[k], after_j[k]), k
    for k in before_b:
        assert np.array_equal(before_b[k], after_b[k]), k
    g.step(1)
    g.close()


def test_joints_stay_inside_their_world(gpu):
    """In a batch, a joint between two worlds is refused; one inside a world is accepted and
    leaves the other worlds' results unchanged."""
    scs = [scenes.pyramid(6), scenes.pyramid(5)]
    g = World(scs)
    solo = World(scs[1])
    ws = g.world_start
    with pytest.raises(_lib.AvbdError):
        g.add_joint(int(ws[0]), int(ws[1]), [0, 0, 0], [0, 0, 0])
    g.lib.avbd_clear_error(g.h)
    b = int(ws[0]) + int(np.flatnonzero(g.props["mass"][ws[0]:ws[1]] > 0)[0])
    g.add_joint(-1, b, g.bodies()["pos"][b], [0, 0, 0], 5000.0, 0.0)
    g.step(30)
    solo.step(30)
    bg, bs = g.bodies(), solo.bodies()
    for k in bs:
        assert np.array_equal(bg[k][ws[1]:ws[2]], bs[k]), k
    g.close()
    solo.close()
