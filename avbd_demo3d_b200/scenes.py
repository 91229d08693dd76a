"""Seeded synthetic scenes for the AVBD step, described in creation order.

A scene is what the reference's scene builders (source/scenes.h) produce through the
public constructors: bodies via ``new Rigid(solver, size, density, friction, pos, vel)``
(rigid.cpp:24-42) with the orientation assigned right after construction (scenes.h:45),
then joints ``new Joint(solver, a, b, rA, rB, stiffnessLin, stiffnessAng, fracture)``
(joint.cpp:25-33) and springs ``new Spring(solver, a, b, rA, rB, stiffness, rest)``
(spring.cpp:14-25) in the listed order. Creation order matters: it fixes the solver's
body list (newest first) and every body's force list, hence the summation order.

Random draws come from a counter-based SplitMix64 stream, so the same seed gives the
same float32 inputs in every consumer (the CUDA path, the C oracle, the reference).
Values are drawn in float64 and rounded once to float32.

Up is +z. Grounds are static boxes (density 0) whose top face is at z = 0.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

F32 = np.float32

SHAPE_BOX, SHAPE_SPHERE, SHAPE_CAPSULE, SHAPE_CYLINDER = 0, 1, 2, 3

FORCE_JOINT = 1
FORCE_SPRING = 2
FORCE_IGNORE = 3

BROADPHASE_ALL_PAIRS = 0
BROADPHASE_GRID = 1
BROADPHASE_SAP = 2
BROADPHASE_LBVH = 3  # the grid's pairs, candidates from a sorted-Morton LBVH (GPU only)

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_MIX1 = np.uint64(0xBF58476D1CE4E5B9)
_MIX2 = np.uint64(0x94D049BB133111EB)


class Stream:
    """Counter-based SplitMix64: draw k of seed s is mix(s + (k + 1) * golden)."""

    def __init__(self, seed: int):
        self.seed = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        self.count = 0

    def bits(self, n: int) -> np.ndarray:
        k = np.arange(self.count + 1, self.count + 1 + n, dtype=np.uint64)
        self.count += n
        with np.errstate(over="ignore"):
            z = self.seed + k * _GOLDEN
            z = (z ^ (z >> np.uint64(30))) * _MIX1
            z = (z ^ (z >> np.uint64(27))) * _MIX2
            z = z ^ (z >> np.uint64(31))
        return z

    def uniform(self, n: int, lo=0.0, hi=1.0) -> np.ndarray:
        """n float64 draws in [lo, hi) from the top 24 bits."""
        u = (self.bits(n) >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)
        return lo + (hi - lo) * u

    def log_uniform(self, n: int, lo: float, hi: float) -> np.ndarray:
        return np.exp(self.uniform(n, math.log(lo), math.log(hi)))

    def unit_quaternions(self, n: int) -> np.ndarray:
        """Shoemake's uniform random rotations, xyzw."""
        u1, u2, u3 = self.uniform(n), self.uniform(n), self.uniform(n)
        a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
        t2, t3 = 2.0 * np.pi * u2, 2.0 * np.pi * u3
        return np.stack([a * np.sin(t2), a * np.cos(t2), b * np.sin(t3), b * np.cos(t3)], axis=1)


@dataclasses.dataclass
class Params:
    """Solver parameters (solver.h:348-357; defaults of solver.cpp:909-932 except where set)."""

    dt: float = float(F32(1.0) / F32(60.0))
    gravity: float = -10.0
    iterations: int = 10
    alpha: float = 0.99
    betaLin: float = 10000.0
    betaAng: float = 100.0
    gamma: float = 0.999
    broadphase: int = BROADPHASE_GRID


def baseline_params(**kw) -> Params:
    """The benchmark parameter set: g -9.81, dt 1/60, 10 iterations, alpha 0.99,
    gamma 0.99, penalty ramp 1e5 (angular ramp at the default 100)."""
    p = Params(gravity=-9.81, alpha=0.99, gamma=0.99, betaLin=1e5, betaAng=100.0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@dataclasses.dataclass
class Scene:
    name: str
    size: np.ndarray  # (n, 3) full widths
    density: np.ndarray  # (n,)
    friction: np.ndarray  # (n,)
    pos: np.ndarray  # (n, 3)
    vel: np.ndarray  # (n, 3)
    quat: np.ndarray  # (n, 4) xyzw
    ftype: np.ndarray  # (m,)
    fa: np.ndarray  # (m,) creation index of body A, -1 = world
    fb: np.ndarray  # (m,)
    frA: np.ndarray  # (m, 3)
    frB: np.ndarray  # (m, 3)
    fparam: np.ndarray  # (m, 3)
    params: Params
    # round bodies (Rigid::makeSphere / makeCapsule / makeCylinder, rigid.cpp:44-90): shape per
    # body (SHAPE_*), dims = (radius, half length); None when every body is a box
    shape: np.ndarray | None = None  # (n,) int32
    dims: np.ndarray | None = None  # (n, 2)

    @property
    def n_bodies(self) -> int:
        return int(self.size.shape[0])

    @property
    def n_forces(self) -> int:
        return int(self.ftype.shape[0])


class SceneBuilder:
    def __init__(self, name: str, params: Params):
        self.name = name
        self.params = params
        self.b = {k: [] for k in ("size", "density", "friction", "pos", "vel", "quat", "shape", "dims")}
        self.f = {k: [] for k in ("ftype", "fa", "fb", "frA", "frB", "fparam")}

    def body(self, size, density, friction, pos, vel=(0, 0, 0), quat=(0, 0, 0, 1)) -> int:
        self.b["size"].append(np.asarray(size, dtype=F32).reshape(3))
        self.b["density"].append(F32(density))
        self.b["friction"].append(F32(friction))
        self.b["pos"].append(np.asarray(pos, dtype=F32).reshape(3))
        self.b["vel"].append(np.asarray(vel, dtype=F32).reshape(3))
        self.b["quat"].append(np.asarray(quat, dtype=F32).reshape(4))
        self.b["shape"].append(SHAPE_BOX)
        self.b["dims"].append(np.zeros(2, F32))
        return len(self.b["size"]) - 1

    def round_body(self, shape, radius, half_length, density, friction, pos, vel=(0, 0, 0), quat=(0, 0, 0, 1)) -> int:
        """Rigid::makeSphere / makeCapsule / makeCylinder (rigid.cpp:44-90); size holds the
        shape's bounding widths as the constructor gives them."""
        r, h = F32(radius), F32(half_length)
        d = F32(r * F32(2.0))
        height = {SHAPE_SPHERE: d, SHAPE_CAPSULE: F32(F32(h * F32(2.0)) + d), SHAPE_CYLINDER: F32(h * F32(2.0))}[shape]
        i = self.body((d, d, height), density, friction, pos, vel, quat)
        self.b["shape"][i] = shape
        self.b["dims"][i] = np.array([r, h if shape != SHAPE_SPHERE else 0.0], F32)
        return i

    def sphere(self, radius, density, friction, pos, vel=(0, 0, 0), quat=(0, 0, 0, 1)) -> int:
        return self.round_body(SHAPE_SPHERE, radius, 0.0, density, friction, pos, vel, quat)

    def capsule(self, radius, half_length, density, friction, pos, vel=(0, 0, 0), quat=(0, 0, 0, 1)) -> int:
        return self.round_body(SHAPE_CAPSULE, radius, half_length, density, friction, pos, vel, quat)

    def cylinder(self, radius, half_length, density, friction, pos, vel=(0, 0, 0), quat=(0, 0, 0, 1)) -> int:
        return self.round_body(SHAPE_CYLINDER, radius, half_length, density, friction, pos, vel, quat)

    def bodies(self, size, density, friction, pos, vel=None, quat=None) -> np.ndarray:
        n = len(size)
        first = len(self.b["size"])
        vel = np.zeros((n, 3)) if vel is None else vel
        quat = np.tile(np.array([0, 0, 0, 1.0]), (n, 1)) if quat is None else quat
        self.b["size"].extend(np.asarray(size, dtype=F32))
        self.b["density"].extend(np.asarray(density, dtype=F32).reshape(n))
        self.b["friction"].extend(np.asarray(friction, dtype=F32).reshape(n))
        self.b["pos"].extend(np.asarray(pos, dtype=F32))
        self.b["vel"].extend(np.asarray(vel, dtype=F32))
        self.b["quat"].extend(np.asarray(quat, dtype=F32))
        self.b["shape"].extend([SHAPE_BOX] * n)
        self.b["dims"].extend(np.zeros((n, 2), F32))
        return np.arange(first, first + n)

    def joint(self, a, b, rA, rB, stiffness_lin=math.inf, stiffness_ang=0.0, fracture=math.inf):
        self._force(FORCE_JOINT, a, b, rA, rB, (stiffness_lin, stiffness_ang, fracture))

    def spring(self, a, b, rA, rB, stiffness, rest=-1.0):
        self._force(FORCE_SPRING, a, b, rA, rB, (stiffness, rest, 0.0))

    def ignore_collision(self, a, b):
        self._force(FORCE_IGNORE, a, b, (0, 0, 0), (0, 0, 0), (0, 0, 0))

    def _force(self, t, a, b, rA, rB, p):
        self.f["ftype"].append(t)
        self.f["fa"].append(-1 if a is None else int(a))
        self.f["fb"].append(int(b))
        self.f["frA"].append(np.asarray(rA, dtype=F32).reshape(3))
        self.f["frB"].append(np.asarray(rB, dtype=F32).reshape(3))
        self.f["fparam"].append(np.asarray(p, dtype=F32).reshape(3))

    def build(self) -> Scene:
        def arr(x, shape, dt):
            return np.ascontiguousarray(np.array(x, dtype=dt).reshape(shape))

        n = len(self.b["size"])
        m = len(self.f["ftype"])
        return Scene(
            name=self.name,
            size=arr(self.b["size"], (n, 3), F32),
            density=arr(self.b["density"], (n,), F32),
            friction=arr(self.b["friction"], (n,), F32),
            pos=arr(self.b["pos"], (n, 3), F32),
            vel=arr(self.b["vel"], (n, 3), F32),
            quat=arr(self.b["quat"], (n, 4), F32),
            ftype=arr(self.f["ftype"], (m,), np.int32),
            fa=arr(self.f["fa"], (m,), np.int32),
            fb=arr(self.f["fb"], (m,), np.int32),
            frA=arr(self.f["frA"], (m, 3), F32),
            frB=arr(self.f["frB"], (m, 3), F32),
            fparam=arr(self.f["fparam"], (m, 3), F32),
            params=self.params,
            shape=arr(self.b["shape"], (n,), np.int32) if any(self.b["shape"]) else None,
            dims=arr(self.b["dims"], (n, 2), F32) if any(self.b["shape"]) else None,
        )


# ---------------------------------------------------------------------------
# Benchmark workloads
# ---------------------------------------------------------------------------


def pyramid(rows: int = 20, params: Params | None = None) -> Scene:
    """Pyramid of 1 m boxes, rows touching: row r holds rows - r boxes at
    x = i*1.01 + r*0.5 - rows/2, z = r + 0.5 (layout of scenePyramid, scenes.h:59-68),
    density 1, friction 0.5, on a static 100x100x1 ground with its top at z = 0.
    rows = 20 gives the 210-box benchmark pyramid."""
    s = SceneBuilder(f"pyramid{rows}", params or baseline_params())
    s.body((100, 100, 1), 0.0, 0.5, (0, 0, -0.5))
    half = F32(rows) / F32(2.0)
    for r in range(rows):
        for i in range(rows - r):
            x = F32(i) * F32(1.01) + F32(r) * F32(0.5) - half
            s.body((1, 1, 1), 1.0, 0.5, (x, 0.0, F32(r) + F32(0.5)))
    return s.build()


def stack_grid(nx: int = 64, ny: int = 64, height: int = 16, seed: int = 1, pitch: float = 2.0,
               params: Params | None = None) -> Scene:
    """nx*ny stacks of `height` boxes on a static ground (200x200x1 at the benchmark size).
    Per box, in draw order: half-extents U[0.25,0.75] (x, y, z), density U[0.5,2],
    horizontal jitter U[-0.05,0.05] (x, y), friction U[0.3,0.8]. Boxes touch vertically.
    64x64x16 = 65,536 boxes is the large benchmark scene."""
    s = SceneBuilder(f"stacks{nx}x{ny}x{height}", params or baseline_params())
    extent = max(200.0, pitch * max(nx, ny) + 8.0)
    s.body((extent, extent, 1), 0.0, 0.5, (0, 0, -0.5))
    n = nx * ny * height
    rs = Stream(seed)
    draws = rs.uniform(n * 7).reshape(n, 7)
    half = F32(0.25 + 0.5 * draws[:, 0:3]).astype(np.float64)
    density = 0.5 + 1.5 * draws[:, 3]
    jitter = -0.05 + 0.1 * draws[:, 4:6]
    friction = 0.3 + 0.5 * draws[:, 6]
    half = half.reshape(ny, nx, height, 3)
    zc = np.cumsum(2.0 * half[..., 2], axis=2) - half[..., 2]
    gy, gx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    cx = ((gx - (nx - 1) / 2.0) * pitch)[..., None] + jitter.reshape(ny, nx, height, 2)[..., 0]
    cy = ((gy - (ny - 1) / 2.0) * pitch)[..., None] + jitter.reshape(ny, nx, height, 2)[..., 1]
    pos = np.stack([cx, cy, zc], axis=-1).reshape(n, 3)
    s.bodies(2.0 * half.reshape(n, 3), density, friction, pos)
    return s.build()


def rope(n: int = 20, params: Params | None = None) -> Scene:
    """Chain of 1x0.5x0.5 boxes linked by ball joints, first link static
    (layout of sceneRope, scenes.h:70-83)."""
    s = SceneBuilder(f"rope{n}", params or baseline_params())
    s.body((100, 100, 1), 0.0, 0.5, (0, 0, -20))
    prev = None
    for i in range(n):
        cur = s.body((1, 0.5, 0.5), 0.0 if i == 0 else 1.0, 0.5, (float(i), 0.0, 10.0))
        if prev is not None:
            s.joint(prev, cur, (0.5, 0, 0), (-0.5, 0, 0))
        prev = cur
    return s.build()


def spring_chain(n: int = 8, params: Params | None = None) -> Scene:
    """Alternating soft/stiff springs between boxes, end links static
    (layout of sceneSpringsRatio, scenes.h:113-128)."""
    s = SceneBuilder(f"springs{n}", params or baseline_params())
    s.body((100, 100, 1), 0.0, 0.5, (0, 0, -10))
    prev = None
    for i in range(n):
        x = (i - (n - 1) * 0.5) * 3.0
        cur = s.body((1, 0.75, 0.75), 0.0 if i in (0, n - 1) else 1.0, 0.5, (x, 0.0, 12.0))
        if prev is not None:
            s.spring(prev, cur, (0.5, 0, 0), (-0.5, 0, 0), 10.0 if i % 2 == 0 else 10000.0, 3.0)
        prev = cur
    return s.build()


def _quat_rotate(q: np.ndarray, v: np.ndarray) -> np.ndarray:
    u = q[..., :3]
    t = 2.0 * np.cross(u, v)
    return v + q[..., 3:4] * t + np.cross(u, t)


def mixed_drop(n_boxes: int = 200_000, n_chains: int = 2048, chain_len: int = 48, spring_frac: float = 0.05,
               extent=(200.0, 200.0, 100.0), seed: int = 2, params: Params | None = None) -> Scene:
    """Boxes dropped from a seeded volume [-X/2,X/2]x[-Y/2,Y/2]x[1,1+Z] with half-extents
    log-uniform in [0.1,1] and uniform random orientations; bounding spheres do not
    overlap at spawn (rejection sampling). n_chains chains of chain_len boxes (part of
    n_boxes) share one orientation per chain and are linked by ball joints at touching
    face centres; spring_frac of the remaining boxes are paired by springs with
    stiffness log-uniform in [1e2,1e5] and rest length = initial distance.
    The defaults are the 200,000-box mixed-constraint benchmark scene."""
    s = SceneBuilder(f"mixed{n_boxes}", params or baseline_params())
    X, Y, Z = extent
    s.body((X + 20.0, Y + 20.0, 1), 0.0, 0.5, (0, 0, -0.5))
    rs = Stream(seed)
    cell = 2.0 * math.sqrt(3.0)  # >= twice the largest bounding radius
    grid: dict[tuple, list] = {}
    centers, radii = [], []

    def free(c, r):
        k = (int(c[0] // cell), int(c[1] // cell), int(c[2] // cell))
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get((k[0] + dx, k[1] + dy, k[2] + dz), ()):
                        d = c - centers[j]
                        if d @ d < (r + radii[j]) ** 2:
                            return False
        return True

    def insert(c, r):
        centers.append(c)
        radii.append(r)
        grid.setdefault((int(c[0] // cell), int(c[1] // cell), int(c[2] // cell)), []).append(len(centers) - 1)

    lo = np.array([-X / 2, -Y / 2, 1.0])
    hi = np.array([X / 2, Y / 2, 1.0 + Z])
    spec_size, spec_pos, spec_quat = [], [], []
    chain_links = []
    n_chain_boxes = n_chains * chain_len
    # chains first
    for c in range(n_chains):
        while True:
            half = F32(rs.log_uniform(chain_len * 3, 0.1, 1.0)).astype(np.float64).reshape(chain_len, 3)
            q = rs.unit_quaternions(1)[0]
            start = rs.uniform(3) * (hi - lo) + lo
            axis = _quat_rotate(q, np.array([1.0, 0.0, 0.0]))
            offs = np.cumsum(2.0 * half[:, 0]) - half[:, 0]
            p = start[None, :] + offs[:, None] * axis[None, :]
            r = np.sqrt((half * half).sum(axis=1))
            if np.any(p - r[:, None] < lo - [0, 0, 0.5]) or np.any(p + r[:, None] > hi + [0, 0, 0.5]):
                continue
            if all(free(p[k], r[k]) for k in range(chain_len)):
                break
        # links of one chain touch each other: insert after the test
        base = len(spec_size)
        for k in range(chain_len):
            insert(p[k], r[k])
            spec_size.append(2.0 * half[k])
            spec_pos.append(p[k])
            spec_quat.append(q)
        for k in range(1, chain_len):
            chain_links.append((base + k - 1, base + k, half[k - 1, 0], half[k, 0]))
    # loose boxes
    n_loose = n_boxes - n_chain_boxes
    while len(spec_size) < n_boxes:
        m = n_boxes - len(spec_size)
        half = F32(rs.log_uniform(m * 3, 0.1, 1.0)).astype(np.float64).reshape(m, 3)
        q = rs.unit_quaternions(m)
        p = rs.uniform(m * 3).reshape(m, 3) * (hi - lo) + lo
        r = np.sqrt((half * half).sum(axis=1))
        for k in range(m):
            if free(p[k], r[k]):
                insert(p[k], r[k])
                spec_size.append(2.0 * half[k])
                spec_pos.append(p[k])
                spec_quat.append(q[k])
    density = rs.uniform(n_boxes, 0.5, 2.0)
    friction = rs.uniform(n_boxes, 0.3, 0.8)
    quat = np.array(spec_quat)
    quat = quat / np.linalg.norm(quat, axis=1, keepdims=True)
    s.bodies(np.array(spec_size), density, friction, np.array(spec_pos), quat=quat)
    for (a, b, ha, hb) in chain_links:
        s.joint(1 + a, 1 + b, (ha, 0.0, 0.0), (-hb, 0.0, 0.0))
    n_spring_boxes = int(round(n_loose * spring_frac)) // 2 * 2
    if n_spring_boxes:
        pick = rs.bits(n_loose)
        order = np.argsort(pick[:n_loose], kind="stable")[:n_spring_boxes]
        loose_ids = 1 + n_chain_boxes + order
        stiff = rs.log_uniform(n_spring_boxes // 2, 1e2, 1e5)
        for k in range(n_spring_boxes // 2):
            s.spring(int(loose_ids[2 * k]), int(loose_ids[2 * k + 1]), (0, 0, 0), (0, 0, 0), stiff[k], -1.0)
    return s.build()


def round_mix(n: int = 600, seed: int = 11, cols: int = 10, params: Params | None = None) -> Scene:
    """Mixed primitives dropped onto a static ground slab: spheres, capsules, cylinders and
    boxes in equal shares (shape drawn per body), radii U[0.2, 0.5], half lengths U[0.1, 0.5],
    box widths U[0.4, 1.0], density U[0.5, 2], friction U[0.3, 0.8], uniform random
    orientations, placed on a jittered cols x cols x (n / cols^2) lattice of 1.4 m pitch
    from z = 1.5 with small random velocities; plus four static cylinders lying on the ground
    and a raised static slab, so every shape pair of the narrowphase meets (round-round,
    round-box and its static-slab and swept-sphere paths, cylinder-box and cylinder-cylinder)."""
    rs = Stream(seed)
    b = SceneBuilder(f"round_mix{n}", params or baseline_params())
    b.body((100, 100, 1), 0.0, 0.5, (0, 0, -0.5))
    half = cols * 1.4 / 2.0
    for k in range(4):  # static cylinders lying on the ground along x
        b.cylinder(0.3, 2.0, 0.0, 0.6, (-half + 1.0 + k * (2.0 * half - 2.0) / 3.0, 0.0, 0.3),
                   quat=(0.0, 0.70710677, 0.0, 0.70710677))
    b.body((4.0, 4.0, 0.2), 0.0, 0.5, (half + 3.0, 0.0, 1.0))  # raised static slab
    shape = (rs.uniform(n) * 4.0).astype(np.int64).clip(0, 3)
    radius = rs.uniform(n, 0.2, 0.5)
    halfl = rs.uniform(n, 0.1, 0.5)
    width = rs.uniform(3 * n, 0.4, 1.0).reshape(n, 3)
    density = rs.uniform(n, 0.5, 2.0)
    friction = rs.uniform(n, 0.3, 0.8)
    quat = rs.unit_quaternions(n)
    jitter = rs.uniform(3 * n, -0.1, 0.1).reshape(n, 3)
    vel = rs.uniform(3 * n, -0.5, 0.5).reshape(n, 3)
    for i in range(n):
        cx, cy, cz = i % cols, (i // cols) % cols, i // (cols * cols)
        pos = (cx * 1.4 - half + 0.7 + jitter[i, 0], cy * 1.4 - half + 0.7 + jitter[i, 1], 1.5 + cz * 1.4 + jitter[i, 2])
        if shape[i] == SHAPE_BOX:
            b.body(width[i], density[i], friction[i], pos, vel[i], quat[i])
        else:
            b.round_body(int(shape[i]), radius[i], halfl[i], density[i], friction[i], pos, vel[i], quat[i])
    return b.build()


def sphere_pour(n: int = 2000, seed: int = 13, params: Params | None = None) -> Scene:
    """Spheres (radius U[0.15, 0.3]) streamed in from a seeded column above a row of static
    standing cylinders on a static ground: many sphere-sphere and sphere-static contacts,
    rolling friction on the ground and the cylinders."""
    rs = Stream(seed)
    b = SceneBuilder(f"sphere_pour{n}", params or baseline_params())
    b.body((100, 100, 1), 0.0, 0.5, (0, 0, -0.5))
    for k in range(5):
        b.cylinder(0.4, 0.6, 0.0, 0.8, (-4.0 + 2.0 * k, 0.0, 0.6))
    radius = rs.uniform(n, 0.15, 0.3)
    side = int(math.ceil(n ** (1.0 / 3.0)))
    jitter = rs.uniform(3 * n, -0.05, 0.05).reshape(n, 3)
    for i in range(n):
        x, y, z = i % side, (i // side) % side, i // (side * side)
        pos = (x * 0.65 - side * 0.325 + jitter[i, 0], y * 0.65 - side * 0.325 + jitter[i, 1], 2.0 + z * 0.65)
        b.sphere(radius[i], 1.0, 0.45, pos, (1.1, 0.0, -1.5))
    return b.build()


def tower(nx: int = 10, ny: int = 10, height: int = 10, seed: int = 4, params: Params | None = None) -> Scene:
    """The 1,000-box tower: stacks built like stack_grid on one 10x10 footprint."""
    return stack_grid(nx, ny, height, seed=seed, params=params)


# ---------------------------------------------------------------------------
# Small scenes covering the reference's box-only probe and constraint scenes
# ---------------------------------------------------------------------------


def _zquat(angle: float):
    return (0.0, 0.0, math.sin(angle * 0.5), math.cos(angle * 0.5))


def box_box_probe(params: Params | None = None) -> Scene:
    """Two overlapping boxes above a ground slab (layout of sceneBoxBoxContactProbe, scenes.h:618-626)."""
    s = SceneBuilder("boxboxprobe", params or Params())
    s.body((24, 24, 1), 0.0, 0.7, (0, 0, 0))
    s.body((0.9, 0.65, 1.0), 1.0, 0.7, (-0.2, 0.0, 4.0))
    s.body((0.9, 0.65, 1.0), 1.0, 0.7, (0.45, 0.0, 4.0))
    return s.build()


def rotated_box_box_probe(params: Params | None = None) -> Scene:
    """Two yawed, overlapping boxes (layout of sceneRotatedBoxBoxContactProbe, scenes.h:628-640)."""
    s = SceneBuilder("rotatedboxboxprobe", params or Params())
    s.body((24, 24, 1), 0.0, 0.7, (0, 0, 0))
    s.body((1.1, 0.65, 1.0), 1.0, 0.7, (-0.18, 0.0, 4.0), quat=_zquat(0.55))
    s.body((1.1, 0.65, 1.0), 1.0, 0.7, (0.42, 0.03, 4.0), quat=_zquat(-0.35))
    return s.build()


def box_cluster_probe(params: Params | None = None) -> Scene:
    """3x3 cluster of yawed boxes (layout of sceneBoxClusterContactProbe, scenes.h:642-660)."""
    s = SceneBuilder("boxclusterprobe", params or Params())
    s.body((24, 24, 1), 0.0, 0.7, (0, 0, 0))
    sp = F32(0.78)
    for y in range(3):
        for x in range(3):
            p = (F32(x - 1) * sp + (F32(0.10) if y & 1 else F32(0.0)), F32(y - 1) * sp * F32(0.85), 4.0)
            s.body((0.9, 0.75, 1.0), 1.0, 0.7, p, quat=_zquat(0.10 * (x - y)))
    return s.build()


def bridge(n: int = 40, params: Params | None = None) -> Scene:
    """Plank bridge with two ball joints per link, boxes dropped on it
    (layout of sceneBridge, scenes.h:990-1021)."""
    s = SceneBuilder(f"bridge{n}", params or Params())
    s.body((100, 100, 1), 0.0, 0.5, (0, 0, 0))
    prev = None
    for i in range(n):
        cur = s.body((1.0, 4.0, 0.5), 0.0 if i in (0, n - 1) else 1.0, 0.5, (F32(i) - F32(n / 2.0), 0.0, 10.0))
        if prev is not None:
            s.joint(prev, cur, (0.5, 2.0, 0), (-0.5, 2.0, 0), math.inf, 0.0)
            s.joint(prev, cur, (0.5, -2.0, 0), (-0.5, -2.0, 0), math.inf, 0.0)
        prev = cur
    for x in range(n // 4):
        for y in range(n // 8):
            s.body((1, 1, 1), 1.0, 0.5, (F32(x) - F32(n / 8.0), 0.0, F32(y) + F32(12.0)))
    return s.build()


def breakable(n: int = 10, m: int = 5, break_force: float = 90.0, params: Params | None = None) -> Scene:
    """Beam of boxes held by rigid joints (linear and angular) with a fracture threshold,
    loaded by falling boxes (layout of sceneBreakable, scenes.h:1023-1052)."""
    s = SceneBuilder(f"breakable{n}", params or Params())
    s.body((100, 100, 1), 0.0, 0.5, (0, 0, 0))
    prev = None
    for i in range(n + 1):
        cur = s.body((1, 1, 0.5), 1.0, 0.5, (F32(i) - F32(n / 2.0), 0.0, 6.0))
        if prev is not None:
            s.joint(prev, cur, (0.5, 0, 0), (-0.5, 0, 0), math.inf, math.inf, break_force)
        prev = cur
    s.body((1, 1, 5), 0.0, 0.5, (-n / 2.0, 0, 2.5))
    s.body((1, 1, 5), 0.0, 0.5, (n / 2.0, 0, 2.5))
    for i in range(m):
        s.body((2, 1, 1), 1.0, 0.5, (0, 0, F32(i) * F32(2.0) + F32(8.0)))
    return s.build()


def reference_pyramid(size: int = 16, params: Params | None = None) -> Scene:
    """The reference's Pyramid scene (scenePyramid, scenes.h:59-68): 16 rows of 1x0.5x0.5
    boxes at x = i*1.01 + r*0.5 - 8, z = r*0.85 + 0.5 on a static ground at z = -0.5,
    with the solver's default parameters."""
    s = SceneBuilder(f"refpyramid{size}", params or Params())
    s.body((100, 100, 1), 0.0, 0.5, (0.0, 0.0, -0.5))
    half = F32(size) / F32(2.0)
    for r in range(size):
        for i in range(size - r):
            x = F32(i) * F32(1.01) + F32(r) * F32(0.5) - half
            s.body((1, 0.5, 0.5), 1.0, 0.5, (x, 0.0, F32(r) * F32(0.85) + F32(0.5)))
    return s.build()


# ---------------------------------------------------------------------------
# Batched uneven worlds
# ---------------------------------------------------------------------------


def _world_stack(b: SceneBuilder, n: int, rs: Stream):
    """Columns of random height 1..16 on a 2 m pitch until n boxes (stack-grid distributions)."""
    heights = []
    left = n
    while left > 0:
        h = int(min(left, 1 + int(rs.uniform(1)[0] * 16)))
        heights.append(h)
        left -= h
    cols = len(heights)
    side = int(math.ceil(math.sqrt(cols)))
    d = rs.uniform(n * 7).reshape(n, 7)
    half = F32(0.25 + 0.5 * d[:, 0:3]).astype(np.float64)
    pos = np.zeros((n, 3))
    k = 0
    for c, h in enumerate(heights):
        gx, gy = c % side, c // side
        z = 0.0
        for _ in range(h):
            pos[k] = ((gx - (side - 1) / 2.0) * 2.0 - 0.05 + 0.1 * d[k, 4],
                      (gy - (side - 1) / 2.0) * 2.0 - 0.05 + 0.1 * d[k, 5], z + half[k, 2])
            z += 2.0 * half[k, 2]
            k += 1
    b.bodies(2.0 * half, 0.5 + 1.5 * d[:, 3], 0.3 + 0.5 * d[:, 6], pos)


def _world_chain(b: SceneBuilder, n: int, rs: Stream):
    """One chain of n boxes linked by ball joints at touching face centres, first link
    anchored to the world, laid out horizontally above the ground (links' half-extents
    log-uniform in [0.1,1], one random yaw for the chain)."""
    half = F32(rs.log_uniform(n * 3, 0.1, 1.0)).astype(np.float64).reshape(n, 3)
    yaw = rs.uniform(1, 0.0, 2.0 * math.pi)[0]
    q = np.array([0.0, 0.0, math.sin(yaw / 2), math.cos(yaw / 2)])
    axis = np.array([math.cos(yaw), math.sin(yaw), 0.0])
    offs = np.cumsum(2.0 * half[:, 0]) - half[:, 0]
    start = np.array([0.0, 0.0, 2.0 + half[:, 1:].max() * 2.0])
    pos = start[None, :] + (offs - offs.mean())[:, None] * axis[None, :]
    first = b.bodies(2.0 * half, rs.uniform(n, 0.5, 2.0), rs.uniform(n, 0.3, 0.8), pos,
                     quat=np.tile(q, (n, 1)))
    b.joint(None, int(first[0]), pos[0] - axis * half[0, 0], (-half[0, 0], 0, 0))
    for k in range(1, n):
        b.joint(int(first[k - 1]), int(first[k]), (half[k - 1, 0], 0, 0), (-half[k, 0], 0, 0))


def _world_pile(b: SceneBuilder, n: int, rs: Stream):
    """n boxes with log-uniform half-extents and random orientations dropped from a volume:
    jittered lattice points spaced beyond two bounding radii, so nothing overlaps at spawn."""
    half = F32(rs.log_uniform(n * 3, 0.1, 1.0)).astype(np.float64).reshape(n, 3)
    q = rs.unit_quaternions(n)
    side = int(math.ceil(n ** (1.0 / 3.0)))
    idx = np.arange(n)
    lattice = np.stack([idx % side, (idx // side) % side, idx // (side * side)], axis=1).astype(np.float64)
    spacing = 3.6
    jitter = rs.uniform(n * 3, -0.05, 0.05).reshape(n, 3)
    pos = (lattice - (side - 1) / 2.0) * spacing + jitter
    pos[:, 2] += (side - 1) / 2.0 * spacing + 2.0
    b.bodies(2.0 * half, rs.uniform(n, 0.5, 2.0), rs.uniform(n, 0.3, 0.8), pos,
             quat=q / np.linalg.norm(q, axis=1, keepdims=True))


def batched_worlds(n_worlds: int = 4096, seed: int = 3, lo: int = 8, hi: int = 2048,
                   params: Params | None = None) -> list:
    """Independent worlds with box counts log-uniform in [lo, hi]; each is, with equal
    probability, a random-height stack field, a jointed chain or a drop pile (the mixed-scene
    distributions), on its own static ground. 4,096 worlds is the batched benchmark."""
    rs = Stream(seed)
    counts = np.floor(np.exp(rs.uniform(n_worlds, math.log(lo), math.log(hi)))).astype(int)
    kinds = (rs.uniform(n_worlds) * 3).astype(int)
    worlds = []
    for w in range(n_worlds):
        b = SceneBuilder(f"world{w}", params or baseline_params())
        n = int(counts[w])
        extent = 40.0 + 4.0 * math.sqrt(n)
        if kinds[w] == 1:
            extent = max(extent, 4.0 * n)  # a chain lying down needs room
        b.body((extent, extent, 1), 0.0, 0.5, (0, 0, -0.5))
        wr = Stream(seed * 1000003 + w)
        (_world_stack, _world_chain, _world_pile)[kinds[w]](b, n, wr)
        worlds.append(b.build())
    return worlds
