"""Generate the golden fixtures from the REFERENCE solver compiled from its own sources.

Run in a checkout that has the reference (it needs oracle/_ref/libavbd_ref.so):
    make -C oracle ref && python tests/golden/make_golden.py

Fixtures written next to this script:
  pyramid20_ref.npz      the 210-box benchmark pyramid, 600 reference steps: a SHA-256 of
                         the body state after every step, full states at a few steps, and
                         per-step counters (pair checks, hits, manifolds, contacts)
  narrowphase_ref.npz    box-box contacts (count, feature keys, local offsets, basis) of the
                         reference's collideBoxes on seeded random pairs and probe layouts
  scenes60_ref.npz       state after 60 steps for joint, spring, fracture, probe, stack and
                         mixed-drop scenes, in list order and in colour order (colour-order
                         runs relink the reference's body list into the oracle's sweep order)
"""
from __future__ import annotations

import hashlib
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from avbd_demo3d_b200 import scenes  # noqa: E402
import checkers  # noqa: E402


def state_digest(b: dict) -> bytes:
    h = hashlib.sha256()
    for k in ("pos", "quat", "vel", "angvel", "prevvel"):
        h.update(np.ascontiguousarray(b[k]).tobytes())
    return h.digest()


def golden_scenes():
    return {
        "rope": scenes.rope(20),
        "springs": scenes.spring_chain(8),
        "bridge": scenes.bridge(),
        "breakable": scenes.breakable(),
        "boxbox": scenes.box_box_probe(),
        "rotboxbox": scenes.rotated_box_box_probe(),
        "cluster": scenes.box_cluster_probe(),
        "stacks": scenes.stack_grid(6, 6, 8, seed=3),
        "mixed": scenes.mixed_drop(1500, 10, 12, 0.05, extent=(24, 24, 16), seed=5),
    }


def narrowphase_cases(n_random: int = 400, seed: int = 11):
    """(pA, qA, sA, pB, qB, sB) rows: seeded random overlapping/near pairs, axis-aligned,
    edge-on and nested layouts."""
    rs = scenes.Stream(seed)
    rows = []
    for _ in range(n_random):
        sA = rs.log_uniform(3, 0.1, 2.0)
        sB = rs.log_uniform(3, 0.1, 2.0)
        qA = rs.unit_quaternions(1)[0]
        qB = rs.unit_quaternions(1)[0]
        d = rs.unit_quaternions(1)[0][:3]
        d = d / max(np.linalg.norm(d), 1e-9)
        reach = 0.5 * (np.linalg.norm(sA) + np.linalg.norm(sB))
        dist = reach * rs.uniform(1, 0.2, 1.05)[0]
        pA = rs.uniform(3, -3, 3)
        rows.append((pA, qA, sA, pA + d * dist, qB, sB))
    ident = np.array([0, 0, 0, 1.0])
    yaw = lambda a: np.array([0, 0, math.sin(a / 2), math.cos(a / 2)])
    tilt = lambda a: np.array([math.sin(a / 2), 0, 0, math.cos(a / 2)])
    fixed = [
        ((0, 0, 0.5), ident, (1, 1, 1), (0, 0, -0.5), ident, (100, 100, 1)),  # resting on ground
        ((0, 0, 1.0), ident, (1, 1, 1), (0.2, 0.1, 0.0), ident, (1, 1, 1)),  # stacked, offset
        ((-0.2, 0, 4), ident, (0.9, 0.65, 1.0), (0.45, 0, 4), ident, (0.9, 0.65, 1.0)),  # Box Box probe
        ((-0.18, 0, 4), yaw(0.55), (1.1, 0.65, 1.0), (0.42, 0.03, 4), yaw(-0.35), (1.1, 0.65, 1.0)),  # rotated probe
        ((0, 0, 0), tilt(math.pi / 4), (1, 1, 1), (0, 0, 1.2), yaw(math.pi / 4), (1, 1, 1)),  # edge on edge
        ((0, 0, 0), ident, (2, 2, 2), (0.1, 0.1, 0.1), yaw(0.3), (0.5, 0.5, 0.5)),  # nested
        ((0, 0, 0), ident, (1, 1, 1), (1.0, 0, 0), ident, (1, 1, 1)),  # exactly touching faces
        ((0, 0, 0), ident, (1, 1, 1), (1.0, 1.0, 1.0), ident, (1, 1, 1)),  # touching corners
    ]
    rows += [tuple(np.asarray(x, dtype=np.float64) for x in r) for r in fixed]
    arr = lambda i, w: np.array([r[i] for r in rows], dtype=np.float32).reshape(len(rows), w)
    return arr(0, 3), arr(1, 4), arr(2, 3), arr(3, 3), arr(4, 4), arr(5, 3)


def run_pyramid(kind: str):
    sc = scenes.pyramid(20)
    w = checkers.World(sc, kind)
    digests, counters, snaps = [], [], {}
    for s in range(1, 601):
        w.step(1)
        b = w.bodies()
        digests.append(np.frombuffer(state_digest(b), dtype=np.uint8))
        counters.append(w.counters()[[0, 1, 2, 3, 4, 5]])
        if s in (1, 10, 60, 120, 600):
            for k, v in b.items():
                snaps[f"s{s}_{k}"] = v
    return np.stack(digests), np.stack(counters), snaps


def run_scene(sc, kind: str, colour: bool, steps: int = 60):
    w = checkers.World(sc, kind)
    o = checkers.World(sc, "oracle", order_mode=1) if colour else None
    for _ in range(steps):
        if colour:
            o.prepare()
            w.prepare()
            w.iterate_ordered(o.solve_order())
            o.iterate()
            o.finish()
            w.finish()
        else:
            w.step(1)
    b = w.bodies()
    m = w.manifolds()
    j = w.joints()
    return {"pos": b["pos"], "quat": b["quat"], "vel": b["vel"], "angvel": b["angvel"], "man_ab": m["ab"],
            "man_n": m["n"], "man_keys": m["keys"], "man_contact": m["contact"], "joint_state": j["state"],
            "joint_broken": j["broken"]}


def main():
    if not checkers.ref_available():
        raise SystemExit("the reference library is not built: make -C oracle ref")
    digests, counters, snaps = run_pyramid("ref")
    np.savez_compressed(os.path.join(HERE, "pyramid20_ref.npz"), digests=digests, counters=counters, **snaps)

    cases = narrowphase_cases()
    out = {"n": [], "keys": [], "rA": [], "rB": [], "basis": []}
    for i in range(cases[0].shape[0]):
        n, keys, rA, rB, basis = checkers.collide_boxes("ref", *(c[i] for c in cases))
        for k, v in zip(out, (n, keys, rA, rB, basis)):
            out[k].append(v)
    np.savez_compressed(os.path.join(HERE, "narrowphase_ref.npz"), pA=cases[0], qA=cases[1], sA=cases[2],
                        pB=cases[3], qB=cases[4], sB=cases[5], **{k: np.array(v) for k, v in out.items()})

    res = {}
    for name, sc in golden_scenes().items():
        for colour in (False, True):
            for k, v in run_scene(sc, "ref", colour).items():
                res[f"{name}_{'colour' if colour else 'list'}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "scenes60_ref.npz"), **res)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
