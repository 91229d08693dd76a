"""Pair and contact injection (avbd_step_external) against the reference's own
Solver::stepCpuReferenceWithExternalBroadphase (solver.cpp:939-957): the reference compiled
from its own sources runs prepareStep with the same injected pairs and contacts
(broadphaseExternalPairs, solver.cpp:579-626; Manifold::initialize's lookup,
manifold.cpp:110-117), then sweeps its bodies in the GPU's colour order. Bodies, manifolds
(pairs, creation order, feature keys, contact rows) and the pair counters must match bit for
bit after every step.

The injected lists are built to reach every rule: shuffled pairs in both orientations,
repeated pairs (a later copy is constrained by the manifold an earlier one made), pairs
naming one body twice or no body, pairs whose spheres do not touch; contact entries copied
from live manifolds with moved anchors and some renamed feature keys, entries for pairs
without a manifold (which make one), lookup-only entries (decreasing dense ids), and two
entries for one ordered pair (the later wins)."""
import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import World, scenes
from avbd_demo3d_b200.solver import box_properties
from test_gpu_parity import bits

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not checkers.ref_available(), reason="reference library not built")]


def candidate_pairs(sc, pos, rng):
    n = sc.n_bodies
    radius = box_properties(sc.size, sc.density)[2][::-1]
    d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=2)
    i, j = np.nonzero(np.triu(d < 1.3 * (radius[:, None] + radius[None, :]), 1))
    pairs = np.stack([i, j], 1)
    flip = rng.random(len(pairs)) < 0.5
    pairs[flip] = pairs[flip][:, ::-1]
    extra = [pairs[rng.integers(len(pairs), size=max(1, len(pairs) // 10))],  # repeats
             pairs[rng.integers(len(pairs), size=max(1, len(pairs) // 10))][:, ::-1],  # reversed repeats
             np.array([[3, 3], [-1, 2], [n + 5, 1], [0, n]])]  # skipped: one body twice, no body
    pairs = np.concatenate([pairs] + extra).astype(np.int32)
    return pairs[rng.permutation(len(pairs))]


def orthobasis(nrm):
    t = np.cross(nrm, [0.0, 0.0, 1.0]) if abs(nrm[2]) < 0.9 else np.cross(nrm, [1.0, 0.0, 0.0])
    t /= np.linalg.norm(t)
    return np.concatenate([nrm, t, np.cross(nrm, t)]).astype(np.float32)


def contact_entries(w, sc, pos, rng):
    """Entries copied from a third of the live manifolds (anchors moved by up to 1 mm, some
    feature keys renamed) plus entries for close pairs with no manifold, each in a random
    orientation; one ordered pair given twice."""
    n = sc.n_bodies
    m = w.manifolds()
    live = np.nonzero(m["n"] > 0)[0]
    pick = live[rng.random(len(live)) < 0.33]
    ab, num, basis, keys, contact, stick = [], [], [], [], [], []
    for k in pick:
        a, b = m["ab"][k]
        c = m["contact"][k].copy()
        c[:, 0:6] += rng.uniform(-1e-3, 1e-3, (8, 6)).astype(np.float32)
        kk = m["keys"][k].copy()
        kk[rng.random(8) < 0.25] += 7  # a renamed feature: no warm start from the old contact
        swap = rng.random() < 0.5
        ab.append((b, a) if swap else (a, b))
        num.append(m["n"][k])
        basis.append(m["basis"][k])
        keys.append(kk)
        contact.append(c)
        stick.append(m["stick"][k])
    have = {tuple(sorted(p)) for p in m["ab"].tolist()}
    radius = box_properties(sc.size, sc.density)[2][::-1]
    made = 0
    for a in rng.permutation(n):
        for b in rng.permutation(n)[:20]:
            if a == b or (min(a, b), max(a, b)) in have or made >= 6:
                continue
            d = pos[a] - pos[b]
            if np.linalg.norm(d) > 1.2 * (radius[a] + radius[b]):
                continue
            nrm = d / np.linalg.norm(d)
            c = np.zeros((8, 15), np.float32)
            c[0, 0:3] = -0.1 * nrm
            c[0, 3:6] = 0.1 * nrm
            c[0, 9:12] = (5.0, 3.0, 3.0)  # penalty seed
            ab.append((a, b))
            num.append(1)
            basis.append(orthobasis(nrm))
            keys.append(np.array([0x01020304] + [0] * 7, np.int32))
            contact.append(c)
            stick.append(np.zeros(8, np.int32))
            made += 1
    if ab:  # the same ordered pair twice: the later entry is the one used
        ab.append(ab[0])
        num.append(num[0])
        basis.append(basis[0])
        k2 = keys[0].copy()
        k2[0] += 1
        keys.append(k2)
        contact.append(contact[0])
        stick.append(stick[0])
    ab = np.array(ab, np.int32).reshape(-1, 2)
    # a manifold is made only for entries whose dense ids increase (list indices decrease)
    creates = (ab[:, 0] > ab[:, 1]).astype(np.int32)
    return {"ab": ab, "n": np.array(num, np.int32), "basis": np.array(basis, np.float32).reshape(-1, 9),
            "keys": np.array(keys, np.int32).reshape(-1, 8), "contact": np.array(contact, np.float32).reshape(-1, 8, 15),
            "stick": np.array(stick, np.int32).reshape(-1, 8), "creates": creates}


def same_as_reference(g, r, where):
    bg, br = g.bodies(), r.bodies()
    for k in ("pos", "quat", "vel", "angvel", "prevvel"):
        assert np.array_equal(bits(bg[k]), bits(br[k])), f"{where}: {k} (max |d| {np.abs(bg[k] - br[k]).max():.3e})"
    mg, mr = g.manifolds(), r.manifolds()
    assert np.array_equal(mg["ab"], mr["ab"]), f"{where}: manifold pairs / creation order"
    assert np.array_equal(mg["n"], mr["n"]) and np.array_equal(mg["keys"], mr["keys"]), f"{where}: feature keys"
    assert np.array_equal(bits(mg["contact"]), bits(mr["contact"])), f"{where}: contact rows"
    assert np.array_equal(bits(mg["basis"]), bits(mr["basis"])), f"{where}: contact basis"
    st, c = g.stats(), r.counters()
    assert (st["pair_checks"], st["sphere_hits"], st["constrained_hits"]) == (c[0], c[1], c[2]), where


@pytest.mark.parametrize("with_contacts", [False, True])
def test_external_pairs_and_contacts_match_the_reference(gpu, with_contacts):
    sc = scenes.stack_grid(4, 4, 6, seed=3)
    g = World(sc)
    r = checkers.World(sc, "ref")
    rng = np.random.default_rng(11 + with_contacts)
    # a few ordinary steps first, so that the injected lists meet live manifolds
    for s in range(1, 6):
        g.step(1)
        r.prepare()
        r.iterate_ordered(g.solve_order())
        r.finish()
    same_as_reference(g, r, "before injection")
    for s in range(1, 31):
        pos = g.bodies()["pos"].astype(np.float64)
        pairs = candidate_pairs(sc, pos, rng)
        entries = contact_entries(g, sc, pos, rng) if with_contacts else None
        g.step_external(pairs, entries)
        r.prepare_external(pairs, entries)
        r.iterate_ordered(g.solve_order())
        r.finish()
        same_as_reference(g, r, f"external step {s}")
    # and back to the grid broadphase
    for s in range(1, 6):
        g.step(1)
        r.prepare()
        r.iterate_ordered(g.solve_order())
        r.finish()
        same_as_reference(g, r, f"after injection, step {s}")
    g.close()
