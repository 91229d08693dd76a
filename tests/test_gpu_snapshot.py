"""Viewer-bridge snapshots written from the device state (avbd_snapshot_binary / _json)
against the test restatement of makeSnapshotBinary / makeSnapshotJson on the oracle's state
(viewer_bridge.cpp:748-842), whose fields are pinned to the reference's SimWorld in
test_oracle_vs_ref.py."""
import json

import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import World, _lib, scenes

pytestmark = pytest.mark.gpu


def oracle_fields(o, n, ids):
    ob, pr = o.bodies(), o.body_props()
    return checkers.snapshot_fields(ids, np.zeros(n, np.int32), pr["mass"], ob["pos"], ob["quat"], pr["size"],
                                    pr["radius"], np.zeros(n, np.float32))


def test_snapshots_match_the_restatement(gpu):
    sc = scenes.mixed_drop(1200, 8, 10, 0.1, extent=(20, 20, 14), seed=31)
    n = sc.n_bodies
    g = World(sc)
    o = checkers.World(sc, "oracle", order_mode=1)
    g.step(15)
    o.step(15)
    name = 'Mixed "drop"\n\ttest'
    fields = oracle_fields(o, n, n - 1 - np.arange(n))
    blob = g.snapshot_binary(42, name)
    assert blob == checkers.encode_snapshot(42, name, fields)
    text = g.snapshot_json(42, name)
    assert text == checkers.snapshot_json(42, name, fields)
    doc = json.loads(text)
    assert doc["frame"] == 42 and doc["scene"] == name and len(doc["bodies"]) == n
    # caller-given dense ids (a permutation with gaps): records in ascending id order
    ids = np.random.default_rng(5).permutation(n).astype(np.int32) * 3 + 1
    blob = g.snapshot_binary(7, "ids", body_id=ids)
    assert blob == checkers.encode_snapshot(7, "ids", oracle_fields(o, n, ids))
    dec = checkers.decode_snapshot(blob)
    assert [b["id"] for b in dec["bodies"]] == sorted(ids.tolist())
    g.close()


def test_snapshot_buffer_checks(gpu):
    g = World(scenes.pyramid(5))
    size = len(g.snapshot_binary(0, "p"))
    assert size == 24 + 1 + 64 * g.n
    import ctypes
    small = (ctypes.c_uint8 * (size - 1))()
    need = ctypes.c_int64()
    rc = g.lib.avbd_snapshot_binary(g.h, 0, b"p", None, small, size - 1, ctypes.byref(need))
    assert rc == _lib.AVBD_ERR_CAPACITY and need.value == size
    g.lib.avbd_clear_error(g.h)
    bad = np.full(g.n, -1, np.int32)
    with pytest.raises(_lib.AvbdError):
        g.snapshot_binary(0, "p", body_id=bad)
    g.lib.avbd_clear_error(g.h)
    g.step(1)
    g.close()


def test_round_world_snapshot(gpu):
    """Spheres, capsules and cylinders in the snapshot: shape code, material id, shape
    radius and half length from the device's shape table."""
    sc = scenes.round_mix(180, seed=43, cols=5)
    n = sc.n_bodies
    g = World(sc)
    o = checkers.World(sc, "oracle", order_mode=1)
    g.step(12)
    o.step(12)
    ob, pr = o.bodies(), o.body_props()
    shape = np.asarray(sc.shape, np.int32)[::-1]
    dims = np.asarray(sc.dims, np.float32)[::-1]
    rnd = shape != 0
    fields = checkers.snapshot_fields(n - 1 - np.arange(n), shape, pr["mass"], ob["pos"], ob["quat"], pr["size"],
                                      np.where(rnd, dims[:, 0], pr["radius"]).astype(np.float32),
                                      np.where(rnd, dims[:, 1], 0).astype(np.float32))
    assert {f["shape"] for f in fields} == {0, 1, 2, 3}
    assert g.snapshot_binary(3, "Round") == checkers.encode_snapshot(3, "Round", fields)
    assert g.snapshot_json(3, "Round") == checkers.snapshot_json(3, "Round", fields)
    g.close()
