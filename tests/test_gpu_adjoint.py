"""GPU adjoint of the step (avbd_adjoint_forward / avbd_adjoint_backward over the C ABI)
against the FP64 reference adjoint and FP64 central finite differences of the
frozen-branch replay, both recorded from the oracle's bit-identical FP32 run.

The loss is the squared distance of the dynamic bodies' centre of mass after T steps to a
seeded target; parameters are the constructor velocities v0 (velocity and previous
velocity), angular velocities w0, masses and per-pair friction coefficients."""
from __future__ import annotations

import numpy as np
import pytest

import checkers
from avbd_demo3d_b200 import World, scenes

pytestmark = pytest.mark.gpu


def _com_and_grad(pos, mass, target):
    d = mass > 0
    mass = mass.astype(np.float64)
    M = float(mass[d].sum())
    com = (mass[d, None] * pos[d]).sum(0) / M
    r = com - target
    dpos = np.zeros_like(pos, dtype=np.float64)
    dpos[d] = 2.0 * r[None, :] * (mass[d, None] / M)
    dmass = np.zeros(len(mass))
    dmass[d] = 2.0 * ((pos[d] - com) @ r) / M
    return float(r @ r), com, dpos, dmass


def _gpu_gradient(scene, steps, every, target):
    w = World(scene, device=0)
    w.adjoint_forward(steps, every)
    b = w.bodies()
    lohi, mu = w.adjoint_pairs()
    props = _masses(scene)
    # the loss of the differentiated map: at the double-precision replay's final state
    final = w.adjoint_replay_state()
    assert np.abs(final["pos"] - b["pos"]).max() < 1e-3
    loss, com, dpos, dmass = _com_and_grad(final["pos"], props, target)
    g = w.adjoint_backward(d_pos=dpos)
    after = w.bodies()
    n = w.n
    theta_grad = np.concatenate([(g["vel"] + g["prevvel"]).ravel(), g["angvel"].ravel(), g["mass"] + dmass,
                                 g["pair_friction"]])
    return w, loss, theta_grad, lohi, mu, b, after, g, n


def _masses(scene):
    from avbd_demo3d_b200.solver import box_properties
    m, _, _ = box_properties(scene.size, scene.density)
    return np.ascontiguousarray(m[::-1])  # list order


def _reference(scene, steps):
    w = checkers.World(scene, "oracle", order_mode=1)
    w.tape_begin()
    w.step(steps)
    return w


def _target(scene, seed=7):
    m = _masses(scene)
    pos = np.ascontiguousarray(scene.pos[::-1]).astype(np.float64)
    d = m > 0
    com = (m[d, None] * pos[d]).sum(0) / m[d].sum()
    return com + np.random.default_rng(seed).uniform(-1, 1, 3)


def _dirs(w_ref, th, k, seed=1):
    n = w_ref.n
    d = w_ref.body_props()["mass"] > 0
    mask = np.zeros(th.size, bool)
    mask[:3 * n] = np.repeat(d, 3)
    mask[3 * n:6 * n] = np.repeat(d, 3)
    mask[6 * n:7 * n] = d
    mask[7 * n:] = True
    dirs = np.random.default_rng(seed).standard_normal((k, th.size)) * mask
    return dirs / np.linalg.norm(dirs, axis=1, keepdims=True)


def test_adjoint_forward_is_the_plain_step(gpu):
    sc = scenes.tower(3, 3, 4, seed=4)
    a = World(sc, device=0)
    a.adjoint_forward(40, 10)
    b = World(sc, device=0)
    b.step(40)
    ref = _reference(sc, 40)
    ga, gb, gr = a.bodies(), b.bodies(), ref.bodies()
    for k in ("pos", "quat", "vel", "angvel", "prevvel"):
        np.testing.assert_array_equal(ga[k].view(np.uint32), gb[k].view(np.uint32))
        np.testing.assert_array_equal(ga[k].view(np.uint32), gr[k].view(np.uint32))


def test_tape_matches_the_oracle_record(gpu):
    """Every branch outcome the GPU tapes from its FP32 step equals the outcome the oracle
    recorded while taking the same (bit-identical) step."""
    sc = scenes.tower(3, 3, 4, seed=4)
    steps = 25
    w = World(sc, device=0)
    w.adjoint_forward(steps, 10)
    ref = _reference(sc, steps)
    for s in range(steps):
        g, r = w.adjoint_tape(s), ref.tape_step(s)
        assert g["nMan"] == r["nMan"]
        np.testing.assert_array_equal(g["body_flags"], r["body_flags"])
        np.testing.assert_array_equal(g["src"], r["src"])
        rf = r["flags"].astype(np.uint32)
        packed = rf[..., 2] | (rf[..., 0] << 12) | (rf[..., 1] << 14)
        np.testing.assert_array_equal(g["flags"], packed.astype(np.uint16))


def test_backward_restores_the_state_and_stepping_continues(gpu):
    sc = scenes.tower(3, 3, 4, seed=4)
    target = _target(sc)
    w, _, _, _, _, before, after, _, _ = _gpu_gradient(sc, 30, 10, target)
    for k in ("pos", "quat", "vel", "angvel", "prevvel"):
        np.testing.assert_array_equal(before[k].view(np.uint32), after[k].view(np.uint32))
    w.step(5)
    plain = World(sc, device=0)
    plain.step(35)
    np.testing.assert_array_equal(w.bodies()["pos"].view(np.uint32), plain.bodies()["pos"].view(np.uint32))


@pytest.mark.parametrize("shape,steps,every", [((2, 2, 3), 30, 10), ((3, 3, 4), 60, 7)])
def test_gradient_matches_reference_adjoint_and_fd(gpu, shape, steps, every):
    sc = scenes.tower(*shape, seed=4)
    target = _target(sc)
    _, loss, g, lohi, mu, _, _, _, n = _gpu_gradient(sc, steps, every, target)
    ref = _reference(sc, steps)
    rlohi, rmu = ref.adj_pairs()
    np.testing.assert_array_equal(lohi, rlohi)
    np.testing.assert_array_equal(mu, rmu)
    th = ref.adj_theta0()
    rloss, rg = ref.adj_gradient(th, target)
    # the same map in double precision; the GPU sums each body's rows in lane groups
    assert loss == pytest.approx(rloss, rel=1e-10)
    # the same frozen-branch map in double precision; only summation orders differ
    assert np.linalg.norm(g - rg) <= 1e-6 * np.linalg.norm(rg)
    n = len(g) - len(mu)
    for sl in (slice(0, 3 * (n // 7)), slice(3 * (n // 7), 6 * (n // 7)), slice(6 * (n // 7), n)):
        assert np.linalg.norm(g[sl] - rg[sl]) <= 1e-6 * np.linalg.norm(rg[sl])
    dirs = _dirs(ref, th, 8)
    fd = ref.adj_fd(th, target, dirs, h=1e-4)
    ad = dirs @ g
    assert np.abs(ad - fd).max() <= 1e-3 * np.abs(fd).max()


def test_tower_1000_gradient_within_1e3_of_fd(gpu):
    """The 1,000-box tower (10 x 10 stacks x 10 high), 120 steps, 10 iterations, a checkpoint
    every 10 steps; 32 seeded unit directions, FP64 central differences with h = 1e-4."""
    sc = scenes.tower(10, 10, 10, seed=4)
    target = _target(sc)
    _, loss, g, lohi, mu, _, _, _, n = _gpu_gradient(sc, 120, 10, target)
    ref = _reference(sc, 120)
    th = ref.adj_theta0()
    rlohi, _ = ref.adj_pairs()
    np.testing.assert_array_equal(lohi, rlohi)
    dirs = _dirs(ref, th, 32)
    fd = ref.adj_fd(th, target, dirs, h=1e-4)
    ad = dirs @ g
    rel = np.abs(ad - fd) / np.abs(fd)
    assert rel.max() <= 1e-3, rel.max()
    _, rg = ref.adj_gradient(th, target)
    assert np.linalg.norm(g - rg) <= 1e-6 * np.linalg.norm(rg)


def test_torch_autograd_function(gpu):
    """The forward / backward pair as a torch.autograd.Function (test harness only)."""
    torch = pytest.importorskip("torch")
    sc = scenes.tower(2, 2, 3, seed=4)
    target = _target(sc)
    masses = _masses(sc)

    class TowerLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, v0, w0):
            w = World(sc, device=0)
            b = w.bodies()
            w.write_bodies(vel=v0.detach().cpu().numpy(), angvel=w0.detach().cpu().numpy(),
                           prevvel=v0.detach().cpu().numpy())
            w.adjoint_forward(20, 5)
            pos = w.adjoint_replay_state()["pos"]
            loss, _, dpos, _ = _com_and_grad(pos, masses, target)
            ctx.world, ctx.dpos = w, dpos
            return torch.tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            g = ctx.world.adjoint_backward(d_pos=ctx.dpos * float(gout))
            return (torch.from_numpy(g["vel"] + g["prevvel"]), torch.from_numpy(g["angvel"]))

    w0 = World(sc, device=0).bodies()
    v = torch.tensor(w0["vel"], dtype=torch.float64, requires_grad=True)
    om = torch.tensor(w0["angvel"], dtype=torch.float64, requires_grad=True)
    loss = TowerLoss.apply(v, om)
    loss.backward()
    ref = _reference(sc, 20)
    th = ref.adj_theta0()
    _, rg = ref.adj_gradient(th, target)
    n = ref.n
    np.testing.assert_allclose(v.grad.numpy().ravel(), rg[:3 * n], rtol=1e-7, atol=1e-12)
    np.testing.assert_allclose(om.grad.numpy().ravel(), rg[3 * n:6 * n], rtol=1e-7, atol=1e-12)


def test_adjoint_rejects_joints(gpu):
    from avbd_demo3d_b200._lib import AvbdError
    w = World(scenes.rope(6), device=0)
    with pytest.raises(AvbdError):
        w.adjoint_forward(5, 5)


def test_backward_needs_forward(gpu):
    from avbd_demo3d_b200._lib import AvbdError
    w = World(scenes.tower(2, 2, 2, seed=4), device=0)
    with pytest.raises(AvbdError):
        w.adjoint_backward()
