"""Seeded scene generators: deterministic, in range, non-overlapping where promised."""
import numpy as np

from avbd_demo3d_b200 import scenes


def test_stream_deterministic_and_uniform():
    a = scenes.Stream(7).uniform(10000)
    b = scenes.Stream(7).uniform(10000)
    assert np.array_equal(a, b)
    assert 0.0 <= a.min() and a.max() < 1.0 and abs(a.mean() - 0.5) < 0.01
    q = scenes.Stream(3).unit_quaternions(1000)
    assert np.allclose(np.linalg.norm(q, axis=1), 1.0)


def test_pyramid_layout():
    sc = scenes.pyramid(20)
    assert sc.n_bodies == 211 and sc.density[0] == 0 and (sc.density[1:] == 1).all()
    assert sc.params.gravity == np.float32(-9.81) or abs(sc.params.gravity + 9.81) < 1e-6


def test_stack_grid_benchmark_shape():
    sc = scenes.stack_grid(64, 64, 16, seed=1)
    assert sc.n_bodies == 65537
    half = sc.size[1:] / 2
    assert half.min() >= 0.25 and half.max() <= 0.75
    assert sc.density[1:].min() >= 0.5 and sc.density[1:].max() <= 2.0
    assert sc.friction[1:].min() >= 0.3 and sc.friction[1:].max() <= 0.8
    # vertical contact: each box rests on the one below (gap within float rounding)
    z = sc.pos[1:, 2].reshape(64 * 64, 16)
    hz = half[:, 2].reshape(64 * 64, 16)
    gaps = (z[:, 1:] - hz[:, 1:]) - (z[:, :-1] + hz[:, :-1])
    assert np.abs(gaps).max() < 1e-5
    assert np.abs(z[:, 0] - hz[:, 0]).max() < 1e-6


def test_mixed_drop_constraints_and_spacing():
    sc = scenes.mixed_drop(3000, 20, 12, 0.05, extent=(40, 40, 20), seed=5)
    assert sc.n_bodies == 3001
    assert (sc.ftype == scenes.FORCE_JOINT).sum() == 20 * 11
    n_springs = (sc.ftype == scenes.FORCE_SPRING).sum()
    assert n_springs == int(round((3000 - 240) * 0.05)) // 2
    # bounding spheres of non-linked bodies do not overlap at spawn (check a sample)
    pos, r = sc.pos[1:].astype(np.float64), np.linalg.norm(sc.size[1:] / 2, axis=1)
    rng = np.random.default_rng(0)
    for i in rng.choice(3000, 200, replace=False):
        d = np.linalg.norm(pos - pos[i], axis=1)
        clash = np.nonzero(d < r + r[i] - 1e-4)[0]
        clash = clash[clash != i]
        # only links of the same chain (12 boxes each, the first 240 bodies) may overlap
        assert all(i < 240 and j < 240 and i // 12 == j // 12 for j in clash), (i, clash)


def test_round_scenes_and_mass_properties():
    """round_mix / sphere_pour carry every shape code, and the mass, moment and bounding
    radius the device world is loaded with (solver.round_properties, float32 formulas of
    rigid.cpp:44-90) equal the C oracle's bit for bit."""
    import checkers
    from avbd_demo3d_b200.solver import box_properties, round_properties

    for sc in (scenes.round_mix(240, seed=11, cols=6), scenes.sphere_pour(240)):
        shape = np.asarray(sc.shape)
        assert sc.dims.shape == (sc.n_bodies, 2) and shape.shape == (sc.n_bodies,)
        assert set(np.unique(shape)) <= {scenes.SHAPE_BOX, scenes.SHAPE_SPHERE, scenes.SHAPE_CAPSULE,
                                         scenes.SHAPE_CYLINDER}
        mass, moment, radius = box_properties(sc.size, sc.density)
        round_properties(sc.shape, sc.dims, sc.density, mass, moment, radius)
        o = checkers.World(sc, "oracle")
        pr = o.body_props()  # list order: creation order reversed
        for mine, theirs in ((mass, pr["mass"]), (moment, pr["moment"]), (radius, pr["radius"])):
            assert np.array_equal(np.asarray(mine, np.float32)[::-1].view(np.uint32),
                                  np.asarray(theirs, np.float32).view(np.uint32))
    assert {1, 2, 3} <= set(np.unique(scenes.round_mix(240, seed=11, cols=6).shape))
