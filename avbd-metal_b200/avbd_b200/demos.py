"""Seeded scene builders: the reference's demo recipes that the solver
configurations are derived from (Sources/PhysicsAVBD/Demos/*.swift) and the
synthetic benchmark scenes built on them.

Randomness comes from SplitMix64 (Sources/SimCore/Math/Random.swift), so a
(recipe, seed) pair always produces the same scene.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi
from .scene import PhysicsScene, SceneJoint, SceneSpring, SceneTet, SceneTri

f32 = np.float32
MASK64 = (1 << 64) - 1


class SplitMix64:
    """SplitMix64 (Random.swift:3-21)."""

    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def next_float(self) -> float:
        """Uniform in [0, 1) with 24 random bits (Random.swift:17-20)."""
        return float(f32(self.next() >> 40) / f32(1 << 24))

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * self.next_float()

    def normal(self) -> float:
        """Standard normal by Box-Muller over two draws."""
        u1 = max(self.next_float(), 1.0 / (1 << 24))
        u2 = self.next_float()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def add_ground(s: PhysicsScene, friction: float = 0.7) -> int:
    """Demos.addGround (Demos.swift:191-196): static 200x200x2 box at z=-1."""
    return s.add_body((200, 200, 2), 0.0, friction, (0, 0, -1))


def stack(height: int) -> PhysicsScene:
    """Demos.stack (Demos.swift:214-222)."""
    s = PhysicsScene("stack")
    add_ground(s)
    for i in range(height):
        s.add_body((1, 1, 1), 1.0, 0.7, (0, 0, 0.5 + i))
    return s


def add_soft_block(s: PhysicsScene, center, nx: int, ny: int, nz: int, spacing: float,
                   mu: float = 3000, lam: float = 30000, mass_per_node: float = 0.05,
                   friction: float = 0.8, self_collision: bool = False,
                   jitter=None, exclusion_joints: bool = True):
    """Demos.addSoftBlock (Demos5.swift:76-145): particle lattice, 5 tets per
    cell (parity-alternated), inert lattice-neighbour exclusion joints.

    `jitter(i, j, k) -> (dx, dy, dz)` optionally perturbs the spawn pose (and
    therefore the rest shape) of each node."""
    sp = f32(spacing)
    half = np.array([nx - 1, ny - 1, nz - 1], dtype=np.float32) * sp / f32(2)
    c = np.array(center, dtype=np.float32)
    ids = np.full((nx, ny, nz), -1, dtype=np.int64)
    flat = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                p = c + np.array([i, j, k], dtype=np.float32) * sp - half
                if jitter is not None:
                    p = p + np.array(jitter(i, j, k), dtype=np.float32)
                b = s.add_particle(float(sp * f32(0.32)), mass_per_node, friction, tuple(p))
                ids[i, j, k] = b
                flat.append(b)

    def tet(a, b, c_, d):
        s.add_tet(SceneTet((int(a), int(b), int(c_), int(d)), mu, lam, self_collision))

    for i in range(nx - 1):
        for j in range(ny - 1):
            for k in range(nz - 1):
                c000, c100 = ids[i, j, k], ids[i + 1, j, k]
                c010, c110 = ids[i, j + 1, k], ids[i + 1, j + 1, k]
                c001, c101 = ids[i, j, k + 1], ids[i + 1, j, k + 1]
                c011, c111 = ids[i, j + 1, k + 1], ids[i + 1, j + 1, k + 1]
                if (i + j + k) % 2 == 0:
                    tet(c000, c100, c010, c001)
                    tet(c110, c100, c010, c111)
                    tet(c101, c100, c001, c111)
                    tet(c011, c010, c001, c111)
                    tet(c100, c010, c001, c111)
                else:
                    tet(c100, c000, c110, c101)
                    tet(c010, c000, c110, c011)
                    tet(c001, c000, c101, c011)
                    tet(c111, c110, c101, c011)
                    tet(c000, c110, c101, c011)
    if exclusion_joints:
        offs = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
        for i in range(nx):
            for j in range(ny):
                for k in range(nz):
                    a = int(ids[i, j, k])
                    for di, dj, dk in offs:
                        if i + di < nx and j + dj < ny and k + dk < nz:
                            s.add_joint(SceneJoint(a, int(ids[i + di, j + dj, k + dk]),
                                                   (0, 0, 0), (0, 0, 0), 0.0, 0.0))
    return flat


def add_cloth_grid(s: PhysicsScene, positions, thickness: float, mass_per_node: float,
                   friction: float = 0.7, structural_k: float = 5000.0, hard_rods: bool = True,
                   shear_k: float = 60.0, bend_k: float = 8.0, membrane_mu: float = 300.0,
                   membrane_bend: float = 5e-4, pinned=()):
    """Demos7.addClothGrid (Demos7.swift:17-84): a particle grid with
    structural rods (hard AL rods by default: `structural_k` is their penalty
    cap), StVK membranes with mu = lambda = `membrane_mu` and Bergou bending
    on alternating diagonals.  `pinned` lists (i, j) nodes given zero mass."""
    nu, nv = len(positions), len(positions[0])
    pinned = set(pinned)
    grid = []
    for i in range(nu):
        row = []
        for j in range(nv):
            m = 0.0 if (i, j) in pinned else mass_per_node
            row.append(s.add_particle(thickness, m, friction, tuple(positions[i][j])))
        grid.append(row)

    def link(a, b, k, hard=False):
        s.add_spring(SceneSpring(a, b, (0, 0, 0), (0, 0, 0), k, hard=hard))

    for i in range(nu):
        for j in range(nv):
            if i + 1 < nu:
                link(grid[i][j], grid[i + 1][j], structural_k, hard_rods)
            if j + 1 < nv:
                link(grid[i][j], grid[i][j + 1], structural_k, hard_rods)
            if membrane_mu <= 0:
                if i + 1 < nu and j + 1 < nv:
                    link(grid[i][j], grid[i + 1][j + 1], shear_k)
                    link(grid[i + 1][j], grid[i][j + 1], shear_k)
                if i + 2 < nu:
                    link(grid[i][j], grid[i + 2][j], bend_k)
                if j + 2 < nv:
                    link(grid[i][j], grid[i][j + 2], bend_k)
    for i in range(nu - 1):
        for j in range(nv - 1):
            v00, v10 = grid[i][j], grid[i + 1][j]
            v01, v11 = grid[i][j + 1], grid[i + 1][j + 1]

            def tri(a, b, c):
                s.add_tri(SceneTri((a, b, c), membrane_mu, membrane_mu, membrane_bend))

            if (i + j) % 2 == 0:
                tri(v00, v10, v11)
                tri(v00, v11, v01)
            else:
                tri(v00, v10, v01)
                tri(v10, v11, v01)
    return grid


def drape_scene(res: int = 28, friction: float = 0.6, membrane_mu: float = 300.0,
                bend: float = 5e-4, obstacle: str = "sphere") -> PhysicsScene:
    """Demos7.drape (Demos7.swift:270-301): a res x res sheet of 2.8 m falls
    onto a static sphere of diameter 1.1 m above the ground.  `obstacle`
    "capsule" (a horizontal static capsule, met by the capsule's three
    feature spheres) or "torus" (a flat static ring, met only by
    particle-torus contacts) replaces the sphere."""
    s = PhysicsScene("drape")
    st = s.settings
    st.iterations, st.beta_lin, st.particle_damping, st.cloth_viscosity = 10, 20000.0, 1.5, 0.25
    add_ground(s, friction=friction)
    if obstacle == "sphere":
        s.add_sphere(1.1, 0.0, friction, (0.0, 0.0, 1.0))
    elif obstacle == "capsule":
        s.add_capsule(1.2, 0.4, 0.0, friction, (0.0, 0.0, 1.0), rotation=quat_axis_angle(math.pi / 2, (0, 1, 0)))
    elif obstacle == "torus":
        s.add_torus(0.5, 0.2, 0.0, friction, (0.0, 0.0, 1.2))
    else:
        raise ValueError(f"unknown obstacle {obstacle!r}")
    n = max(20, res)
    size = f32(2.8)
    spacing = size / f32(n - 1)
    r = min(f32(0.05), f32(0.3) * spacing)
    pos = [[(float(f32(i) * spacing - size / f32(2)), float(f32(j) * spacing - size / f32(2)), 1.75)
            for j in range(n)] for i in range(n)]
    add_cloth_grid(s, pos, float(r), 0.008, friction, membrane_mu=membrane_mu, membrane_bend=bend)
    return s


# ---------------------------------------------------------------------------
# Synthetic benchmark scenes (one per solver configuration)
# ---------------------------------------------------------------------------

def rigid_stack_scene(seed: int = 1, count: int = 20) -> PhysicsScene:
    """Rigid stack: `count` unit cubes (density 1000) with 1e-3 m gaps on a
    static ground, friction 0.5, lateral jitter U(+-1e-3) from the seed;
    dt 1/60, 10 iterations, beta 1e5, alpha 0.95, gamma 0.99, g = -9.81."""
    rng = SplitMix64(seed)
    s = PhysicsScene("rigid-stack")
    add_ground(s, friction=0.5)
    for i in range(count):
        jx = rng.uniform(-1e-3, 1e-3)
        jy = rng.uniform(-1e-3, 1e-3)
        s.add_body((1, 1, 1), 1000.0, 0.5, (jx, jy, 0.5 + i * (1.0 + 1e-3)))
    st = s.settings
    st.dt, st.gravity, st.iterations = 1.0 / 60.0, -9.81, 10
    st.beta_lin, st.alpha, st.gamma = 1.0e5, 0.95, 0.99
    return s


def soft_cube_scene(seed: int = 2, n: int = 24, iterations: int = 20,
                    exclusion_joints: bool = True) -> PhysicsScene:
    """Soft cube: n^3-vertex lattice of a 1 m cube, 5 tets per cell, Stable
    Neo-Hookean E=1e5 Pa, nu=0.4, density 1000 (lumped node mass), dropped
    from 0.5 m onto the ground, friction 0.4, dt 1/60, static palette; rest
    positions perturbed by N(0, 1e-4 m) from the seed."""
    rng = SplitMix64(seed)
    E, nu, rho = 1.0e5, 0.4, 1000.0
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    spacing = 1.0 / (n - 1)
    s = PhysicsScene("soft-cube")
    add_ground(s, friction=0.4)
    noise = {}

    def jitter(i, j, k):
        v = (rng.normal() * 1e-4, rng.normal() * 1e-4, rng.normal() * 1e-4)
        noise[(i, j, k)] = v
        return v

    add_soft_block(s, (0.0, 0.0, 1.0), n, n, n, spacing, mu=mu, lam=lam,
                   mass_per_node=rho * 1.0 / (n ** 3), friction=0.4, jitter=jitter,
                   exclusion_joints=exclusion_joints)
    st = s.settings
    st.dt, st.gravity, st.iterations = 1.0 / 60.0, -9.81, iterations
    return s


def cloth_sphere_scene(seed: int = 3, n: int = 256, iterations: int = 30,
                       hard_rods: bool = True) -> PhysicsScene:
    """Cloth with self-contact: an n x n sheet of 2 m side (spacing 2/(n-1)),
    membrane mu = lambda = 1e4, Bergou bending 1e-3, particle (contact) radius
    2e-3 m, areal density 0.1 kg/m^2, two corners of one edge pinned, held
    0.1 m above a static sphere of radius 0.5 m (centre z = 1) over the ground;
    in-plane noise U(+-1e-4 m) from the seed.  Hard structural rods
    (penalty cap 5000) as in addClothGrid.  Planar-DAT is selected
    automatically (shell-only scene); dt 1/120, `iterations` iterations."""
    rng = SplitMix64(seed)
    s = PhysicsScene("cloth-sphere")
    st = s.settings
    st.dt, st.iterations, st.beta_lin = 1.0 / 120.0, iterations, 20000.0
    st.particle_damping, st.cloth_viscosity = 1.5, 0.25
    add_ground(s, friction=0.5)
    s.add_sphere(1.0, 0.0, 0.5, (0.0, 0.0, 1.0))
    side = f32(2.0)
    spacing = side / f32(n - 1)
    pos = []
    for i in range(n):
        row = []
        for j in range(n):
            x = f32(i) * spacing - side / f32(2) + f32(rng.uniform(-1e-4, 1e-4))
            y = f32(j) * spacing - side / f32(2) + f32(rng.uniform(-1e-4, 1e-4))
            row.append((float(x), float(y), 1.6))
        pos.append(row)
    mass = float(f32(0.1) * side * side / f32(n * n))
    add_cloth_grid(s, pos, 2e-3, mass, 0.5, hard_rods=hard_rods, membrane_mu=1e4,
                   membrane_bend=1e-3, pinned=((0, 0), (0, n - 1)))
    return s


def batched_worlds_scene(worlds: int = 4096, seed: int = 4, pitch: float = 1.6, first_world: int = 0,
                         collision_groups: bool = True):
    """Batched articulated worlds packed into one scene, one collision group
    per world (the reference's vector-environment layout,
    RL/PushTEnv.swift:114-180): each world is a planar serial chain of 3-7
    box links (0.25 x 0.06 x 0.06 m, density 500) lying on the ground plane,
    joined by hinges about +z with implicit position-PD motors (effort 2 N m,
    kp 50, kd 1), the first link hinged to the world, plus a welded T block
    (bar 0.2 x 0.05 x 0.05 m, stem 0.05 x 0.15 x 0.05 m) at a seeded pose;
    friction 0.5, dt 1/60, 8 iterations.  Returns (scene, motor joint ids,
    world offsets): offsets[e] is the first body of world e (ragged).

    World w draws from its own stream SplitMix64((seed << 32) + w), so a shard
    [first_world, first_world + worlds) builds exactly the worlds that a
    single scene of all worlds would contain.  collision_groups=False leaves
    every collider in group 0, for avbd_create_batched to assign the groups
    from the world offsets."""
    s = PhysicsScene("batched-worlds")
    cols = int(math.ceil(math.sqrt(worlds)))
    rows = int(math.ceil(worlds / cols))
    hx, hy = 0.5 * (cols - 1) * pitch, 0.5 * (rows - 1) * pitch
    s.add_body((2 * (hx + pitch), 2 * (hy + pitch), 2.0), 0.0, 0.5, (0.0, 0.0, -1.0))
    motors, offsets = [], []
    link = (0.25, 0.06, 0.06)
    for e in range(worlds):
        rng = SplitMix64((seed << 32) + first_world + e)
        g = e + 1 if collision_groups else 0
        cx, cy = (e % cols) * pitch - hx, (e // cols) * pitch - hy
        offsets.append(len(s.bodies))
        n = 3 + int(rng.next_float() * 5)
        base = (cx - 0.6, cy - 0.3, 0.03)
        prev = -1
        for k in range(n):
            pos = (base[0] + 0.25 * k + 0.125, base[1], base[2])
            b = s.add_body(link, 500.0, 0.5, pos, collision_group=g)
            anchor_a = (base[0], base[1], base[2]) if prev < 0 else (0.125, 0.0, 0.0)
            motors.append(len(s.joints))
            s.add_joint(SceneJoint(prev, b, anchor_a, (-0.125, 0.0, 0.0), stiffness_ang=float("inf"),
                                   hinge_axis=(0.0, 0.0, 1.0), motor_torque=2.0, motor_stiffness=50.0,
                                   motor_damping=1.0))
            prev = b
        yaw = (rng.next_float() - 0.5) * 2.0 * math.pi
        qz = (0.0, 0.0, math.sin(0.5 * yaw), math.cos(0.5 * yaw))
        cyaw, syaw = math.cos(yaw), math.sin(yaw)
        bc = (cx + 0.25 + 0.2 * rng.next_float(), cy + 0.25 + 0.2 * rng.next_float(), 0.025)

        def rot(v):
            return (cyaw * v[0] - syaw * v[1], syaw * v[0] + cyaw * v[1], v[2])
        ob, os_ = rot((0.0, 0.05, 0.0)), rot((0.0, -0.05, 0.0))
        bar = s.add_body((0.2, 0.05, 0.05), 500.0, 0.5, (bc[0] + ob[0], bc[1] + ob[1], bc[2]), rotation=qz,
                         collision_group=g)
        stem = s.add_body((0.05, 0.15, 0.05), 500.0, 0.5, (bc[0] + os_[0], bc[1] + os_[1], bc[2]), rotation=qz,
                          collision_group=g)
        s.add_joint(SceneJoint(bar, stem, (0.0, -0.025, 0.0), (0.0, 0.075, 0.0), stiffness_ang=float("inf")))
        s.add_joint(SceneJoint(bar, stem, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 0.0, 0.0))
    st = s.settings
    st.dt, st.iterations, st.gravity = 1.0 / 60.0, 8, -9.81
    return s, motors, offsets


def single_tet_scene() -> PhysicsScene:
    """SoftBodyTests.testTetVolumePreservation (SoftBodyTests.swift:53-69)."""
    s = PhysicsScene("tet1")
    s.settings.iterations = 20
    p0 = s.add_particle(0.05, 0.1, position=(0, 0, 3))
    p1 = s.add_particle(0.05, 0.1, position=(0.5, 0, 3))
    p2 = s.add_particle(0.05, 0.1, position=(0, 0.5, 3))
    p3 = s.add_particle(0.05, 0.1, position=(0, 0, 3.5))
    s.add_joint(SceneJoint(-1, p0, (0, 0, 3), (0, 0, 0)))
    s.add_tet(SceneTet((p0, p1, p2, p3), 2000, 20000))
    return s


def particle_rod_chain_scene() -> PhysicsScene:
    """SoftBodyTests.testParticleRodChainInextensible (SoftBodyTests.swift:27-51)."""
    s = PhysicsScene("pc")
    s.settings.iterations = 20
    prev = -1
    for k in range(12):
        p = s.add_particle(0.05, 0.02, position=(k * 0.25, 0, 4))
        if k == 0:
            s.add_joint(SceneJoint(-1, p, (0, 0, 4), (0, 0, 0)))
        else:
            s.add_spring(SceneSpring(prev, p, (0, 0, 0), (0, 0, 0), 1e5, hard=True))
        prev = p
    return s


def pinned_soft_block_scene(n: int = 10) -> PhysicsScene:
    """A soft block hanging from world joints at its four top corners: every
    particle a 3-DOF body, some carrying joints (general primal path)."""
    s = PhysicsScene("pinned-soft-block")
    add_ground(s, friction=0.5)
    ids = add_soft_block(s, (0.0, 0.0, 2.0), n, n, n, 0.08, mu=2e4, lam=8e4,
                         mass_per_node=0.01, friction=0.5, exclusion_joints=False)
    grid = np.array(ids).reshape(n, n, n)
    for i in (0, n - 1):
        for j in (0, n - 1):
            b = int(grid[i, j, n - 1])
            p = s.bodies[b].position
            s.add_joint(SceneJoint(-1, b, p, (0, 0, 0)))
    s.settings.iterations = 12
    return s


def box_field_scene(count: int = 700, seed: int = 4) -> PhysicsScene:
    """`count` small boxes on the ground in a loose grid (rigid, dynamic coloring)."""
    rng = SplitMix64(seed)
    s = PhysicsScene("box-field")
    add_ground(s, friction=0.6)
    side = int(math.ceil(math.sqrt(count)))
    for i in range(count):
        x, y = (i % side) * 0.5, (i // side) * 0.5
        s.add_body((0.3, 0.3, 0.3), 500.0, 0.6, (x, y, 0.16 + rng.uniform(0.0, 0.05)))
    return s


def mixed_scene(seed: int = 5, cubes: int = 64, cube_n: int = 10, boxes: int = 256, cloth_n: int = 128,
                iterations: int = 20, cube_size: float = 0.3, pitch: float = 0.5) -> PhysicsScene:
    """Mixed scene: `cubes` soft cubes of cube_n^3 vertices (Stable
    Neo-Hookean E=5e4 Pa, nu=0.45, density 1000, side `cube_size`) on a
    square grid of pitch `pitch`, `boxes` rigid boxes with edges U(0.1, 0.4) m
    above them, and a cloth_n x cloth_n sheet (membrane mu = lambda = 1e4,
    Bergou bending 1e-3, contact radius 5e-3 m, areal density 0.1 kg/m^2)
    covering the field from above, all falling together onto the ground;
    dt 1/60.  Tets and cloth together select isotropic OGC truncation; every
    soft surface, the cloth and the boxes meet through vertex-triangle,
    edge-edge and rigid-triangle contacts.  Positions and box sizes come
    from the seed."""
    rng = SplitMix64(seed)
    s = PhysicsScene("mixed")
    st = s.settings
    st.dt, st.gravity, st.iterations = 1.0 / 60.0, -9.81, iterations
    add_ground(s, friction=0.5)
    E, nu, rho = 5.0e4, 0.45, 1000.0
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    g = int(math.ceil(math.sqrt(cubes)))
    extent = g * pitch
    node_mass = rho * cube_size ** 3 / cube_n ** 3
    for c in range(cubes):
        cx = (c % g) * pitch - extent / 2 + pitch / 2 + rng.uniform(-0.02, 0.02)
        cy = (c // g) * pitch - extent / 2 + pitch / 2 + rng.uniform(-0.02, 0.02)
        cz = cube_size / 2 + 0.05 + rng.uniform(0.0, 0.1)
        add_soft_block(s, (cx, cy, cz), cube_n, cube_n, cube_n, cube_size / (cube_n - 1), mu=mu, lam=lam,
                       mass_per_node=node_mass, friction=0.5, exclusion_joints=False)
    bg = int(math.ceil(math.sqrt(boxes)))
    bpitch = extent / bg
    for b in range(boxes):
        size = (rng.uniform(0.1, 0.4), rng.uniform(0.1, 0.4), rng.uniform(0.1, 0.4))
        bx = (b % bg) * bpitch - extent / 2 + bpitch / 2
        by = (b // bg) * bpitch - extent / 2 + bpitch / 2
        s.add_body(size, 500.0, 0.5, (bx, by, cube_size + 0.45 + rng.uniform(0.0, 0.2)))
    if cloth_n >= 2:
        side = f32(extent)
        spacing = side / f32(cloth_n - 1)
        z = cube_size + 1.2
        pos = [[(float(f32(i) * spacing - side / f32(2)), float(f32(j) * spacing - side / f32(2)), z)
                for j in range(cloth_n)] for i in range(cloth_n)]
        mass = float(f32(0.1) * side * side / f32(cloth_n * cloth_n))
        add_cloth_grid(s, pos, 5e-3, mass, 0.5, hard_rods=True, membrane_mu=1e4, membrane_bend=1e-3)
    return s


def two_cubes_scene(n: int = 5, iterations: int = 10) -> PhysicsScene:
    """Two soft cubes, one dropped onto the other: vertex-triangle contacts
    between separate soft surfaces (isotropic OGC)."""
    s = PhysicsScene("two-cubes")
    add_ground(s, friction=0.5)
    for z in (0.16, 0.52):
        add_soft_block(s, (0.03 * (z > 0.3), 0.0, z), n, n, n, 0.3 / (n - 1), mu=3000.0, lam=30000.0,
                       mass_per_node=0.05, friction=0.5, exclusion_joints=False)
    s.settings.iterations = iterations
    return s


# ---------------------------------------------------------------------------
# Tori, capsules and convex hulls
# ---------------------------------------------------------------------------

def quat_axis_angle(angle: float, axis) -> tuple:
    """Unit quaternion (x, y, z, w) of a rotation by `angle` about `axis`."""
    a = np.asarray(axis, dtype=np.float64)
    a = a / np.linalg.norm(a)
    h = 0.5 * angle
    return tuple(float(f32(x)) for x in (*(a * math.sin(h)), math.cos(h)))


def quat_mul(a, b) -> tuple:
    """Hamilton product a * b of (x, y, z, w) quaternions, normalised."""
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    q = np.array([aw * bx + ax * bw + ay * bz - az * by,
                  aw * by - ax * bz + ay * bw + az * bx,
                  aw * bz + ax * by - ay * bx + az * bw,
                  aw * bw - ax * bx - ay * by - az * bz])
    q /= np.linalg.norm(q)
    return tuple(float(f32(x)) for x in q)


Q_X90 = quat_axis_angle(math.pi / 2, (1, 0, 0))


def torus_rest_scene() -> PhysicsScene:
    """A torus dropped flat onto a static slab comes to rest lying flat, its
    centre one tube radius up (TorusAndMachineTests.swift:7-15)."""
    s = PhysicsScene("torus-rest")
    s.add_body((100, 100, 2), 0.0, 0.5, (0, 0, -1))
    s.add_torus(0.45, 0.12, 1.0, 0.5, (0, 0, 2))
    return s


def linked_tori_scene() -> PhysicsScene:
    """Two interlocked rings, the upper one pinned to the world, carrying a
    1 kg box on the lower one (TorusAndMachineTests.swift:17-30).  The box is
    the last body."""
    s = PhysicsScene("linked-tori")
    t1 = s.add_torus(0.45, 0.12, 1.0, 0.4, (0, 0, 6), rotation=Q_X90)
    t2 = s.add_torus(0.45, 0.12, 1.0, 0.4, (0, 0, 5.34),
                     rotation=quat_mul(quat_axis_angle(math.pi / 2, (0, 0, 1)), Q_X90))
    s.add_joint(SceneJoint(-1, t1, (0, 0, 6.4), (0.45, 0, 0)))
    w = s.add_body((0.5, 0.5, 0.5), 8.0, 0.5, (0, 0, 4.4))
    s.add_joint(SceneJoint(t2, w, (0.45, 0, 0), (0, 0, 0.45)))
    return s


def ring_catch_scene() -> PhysicsScene:
    """A ball dropped into a static upright ring stays in it
    (TorusAndMachineTests.swift:32-41)."""
    s = PhysicsScene("ring-catch")
    s.add_body((100, 100, 2), 0.0, 0.5, (0, 0, -1))
    s.add_torus(0.6, 0.15, 0.0, 0.5, (0, 0, 1.5), rotation=Q_X90)
    s.add_sphere(0.7, 1.0, 0.5, (0, 0, 1.52))
    return s


def bearing_scene() -> PhysicsScene:
    """A torus hub hanging on a static capsule axle settles at the analytic
    offset (major - minor) - axle radius below it
    (TorusAndMachineTests.swift:88-102)."""
    s = PhysicsScene("bearing")
    s.settings.iterations = 20
    s.settings.beta_lin = 20000.0
    s.add_capsule(2.0, 0.11, 0.0, 0.02, (0, 0, 3), rotation=Q_X90)
    s.add_torus(0.27, 0.115, 1.5, 0.02, (0, 0, 3), rotation=Q_X90)
    return s


def hull_box_scene() -> PhysicsScene:
    """A body whose only collider is an 8-vertex convex hull (a unit cube)
    rests on box terrain (GPUSolverTests.swift:537-571).  Body 1 is the hull
    body."""
    s = PhysicsScene("hull-box")
    s.settings.dt = 1.0 / 120.0
    s.settings.gravity = -9.81
    s.settings.iterations = 20
    s.add_body((20, 20, 0.2), 0.0, 1.0, (0, 0, -0.1))
    body = s.add_body((1, 1, 1), 0.0, 1.0, (0, 0, 2), mass=1.0, diagonal_inertia=(1 / 6, 1 / 6, 1 / 6),
                      collision_enabled=False)
    hull = [(x, y, z) for z in (-0.5, 0.5) for y in (-0.5, 0.5) for x in (-0.5, 0.5)]
    s.add_convex_collider(body, hull, friction=1.0)
    return s


def capsule_foot_scene() -> PhysicsScene:
    """A foot of three capsule colliders with material anchors, held by a
    500 N/m spring to a world point (GPUSolverTests.swift:577-620): under a
    load below the Coulomb limit it must not creep.  Joint 0 is the spring;
    body 1 the foot."""
    s = PhysicsScene("capsule-foot")
    s.settings.dt = 1.0 / 120.0
    s.settings.iterations = 20
    s.add_body((20, 8, 0.2), 0.0, 1.1, (0, 0, -0.1))
    foot = s.add_body((0.35, 0.2, 0.2), 0.0, 1.1, (0, 0, 0.36), mass=5.0, diagonal_inertia=(0.08, 0.12, 0.08),
                      collision_enabled=False)
    along_x = quat_axis_angle(math.pi / 2, (0, 1, 0))
    for y in (-0.07, 0.07):
        s.add_collider(foot, (0.24, 0.035, 0), friction=1.1, local_position=(0, y, -0.31),
                       local_rotation=along_x, shape=abi.SHAPE_CAPSULE)
    s.add_collider(foot, (0.14, 0.035, 0), friction=1.1, local_position=(0.14, 0, -0.31),
                   local_rotation=Q_X90, shape=abi.SHAPE_CAPSULE)
    s.add_joint(SceneJoint(-1, foot, (0, 0, 0.36), (0, 0, 0), stiffness_lin=500.0, stiffness_ang=0.0))
    return s


def chainmail_scene(rings: int = 6, drops: int = 3) -> PhysicsScene:
    """Demos2.chainmail (Demos2.swift:318-430): a sheet of interlinked tori
    hung on welded peg posts, with spheres and boxes dropped on it."""
    s = PhysicsScene("chainmail")
    st = s.settings
    st.iterations, st.beta_lin, st.lambda_max = 15, 20000.0, 1500.0
    add_ground(s, friction=0.6)
    R, r, sheet_z, pitch = 0.45, 0.15, 8.0, 1.15
    n = rings
    extent = float(f32(n - 1) * f32(pitch) / f32(2))
    mid = (n - 1) // 2
    inf = float("inf")

    def add_post(x, y):
        seg_h, cross = 1.6, 0.22
        peg_z, top_z = sheet_z - 0.3, sheet_z + 1.0
        prev = s.add_body((cross, cross, seg_h), 0.0, 0.4, (x, y, seg_h / 2))
        z = seg_h
        while z < top_z:
            h = min(seg_h, top_z - z)
            seg = s.add_body((cross, cross, h), 4.0, 0.4, (x, y, z + h / 2))
            s.add_joint(SceneJoint(prev, seg, (0, 0, s.bodies[prev].size[2] / 2), (0, 0, -h / 2),
                                   stiffness_lin=inf, stiffness_ang=inf))
            prev = seg
            z += h
        host = prev
        for axis in range(2):
            size = (1.1, 0.14, 0.14) if axis == 0 else (0.14, 1.1, 0.14)
            peg = s.add_body(size, 2.0, 0.5, (x, y, peg_z))
            seg_c = s.bodies[host].position[2]
            s.add_joint(SceneJoint(host, peg, (0, 0, peg_z - seg_c), (0, 0, 0), stiffness_lin=inf,
                                   stiffness_ang=inf))
            off = (0.4, 0, 0) if axis == 0 else (0, 0.4, 0)
            s.add_joint(SceneJoint(host, peg, (off[0], off[1], peg_z - seg_c), off, stiffness_lin=inf,
                                   stiffness_ang=inf))

    cells = set()
    for j in range(n):
        for i in range(n):
            corner = (i in (0, n - 1)) and (j in (0, n - 1))
            edge_mid = (i == mid and j in (0, n - 1)) or (j == mid and i in (0, n - 1))
            if corner or edge_mid:
                cells.add(j * n + i)
    for cell in sorted(cells):
        i, j = cell % n, cell // n
        add_post(i * pitch - extent, j * pitch - extent)
    q_y = quat_mul(quat_axis_angle(math.pi / 2, (0, 0, 1)), Q_X90)
    for j in range(n):
        for i in range(n):
            cx, cy = i * pitch - extent, j * pitch - extent
            s.add_torus(R, r, 1.0, 0.3, (cx, cy, sheet_z))
            if i + 1 < n:
                s.add_torus(R, r, 1.0, 0.3, (cx + pitch / 2, cy, sheet_z), rotation=Q_X90)
            if j + 1 < n:
                s.add_torus(R, r, 1.0, 0.3, (cx, cy + pitch / 2, sheet_z), rotation=q_y)
    rng = SplitMix64(11)
    for k in range(drops):
        sz = 0.9 + rng.next_float() * 0.7
        pos = ((rng.next_float() - 0.5) * n * pitch * 0.4, (rng.next_float() - 0.5) * n * pitch * 0.4,
               sheet_z + 4 + k * 2)
        if k % 2 == 0:
            s.add_sphere(sz, 1.0, 0.5, pos)
        else:
            s.add_body((sz, sz, sz), 1.0, 0.5, pos)
    return s


def shapes_scene(seed: int = 6, count: int = 512, pitch: float = 1.3) -> PhysicsScene:
    """A seeded pile of capsules, tori, spheres, boxes and convex-hull
    bodies (octahedra) dropped onto the ground in a square grid of columns:
    every narrowphase shape pair except hull/round (which produces no
    contact) occurs."""
    s = PhysicsScene("shapes")
    add_ground(s, friction=0.6)
    rng = SplitMix64(seed)
    side = max(1, int(math.ceil(math.sqrt(count / 4))))
    octa = [(0.35, 0, 0), (-0.35, 0, 0), (0, 0.35, 0), (0, -0.35, 0), (0, 0, 0.35), (0, 0, -0.35)]
    for k in range(count):
        col, layer = k % (side * side), k // (side * side)
        x = (col % side - 0.5 * (side - 1)) * pitch + rng.uniform(-0.1, 0.1)
        y = (col // side - 0.5 * (side - 1)) * pitch + rng.uniform(-0.1, 0.1)
        z = 0.6 + 1.1 * layer
        q = quat_axis_angle(rng.uniform(0.0, math.pi), (rng.uniform(-1, 1), rng.uniform(-1, 1), 1.0))
        kind = rng.next() % 5
        if kind == 0:
            s.add_capsule(rng.uniform(0.3, 0.7), rng.uniform(0.12, 0.2), 1.0, 0.5, (x, y, z), rotation=q)
        elif kind == 1:
            s.add_torus(rng.uniform(0.25, 0.4), rng.uniform(0.08, 0.12), 1.0, 0.5, (x, y, z), rotation=q)
        elif kind == 2:
            s.add_sphere(rng.uniform(0.3, 0.6), 1.0, 0.5, (x, y, z))
        elif kind == 3:
            s.add_body((rng.uniform(0.3, 0.6), rng.uniform(0.3, 0.6), rng.uniform(0.3, 0.6)), 1.0, 0.5, (x, y, z),
                       rotation=q)
        else:
            b = s.add_body((0.7, 0.7, 0.7), 0.0, 0.5, (x, y, z), rotation=q, mass=0.3,
                           diagonal_inertia=(0.02, 0.02, 0.02), collision_enabled=False)
            s.add_convex_collider(b, octa, friction=0.5)
    return s


# ---------------------------------------------------------------------------
# Push-T vector environment (RL/PushTEnv.swift)
# ---------------------------------------------------------------------------

PUSHT_TIP_HEIGHT = 0.42
PUSHT_PUSHER_FORCE = 60.0
PUSHT_PITCH = 7.0


def _qrot(q, v):
    u = np.asarray(q[:3], np.float64)
    t = 2.0 * np.cross(u, v)
    return np.asarray(v, np.float64) + q[3] * t + np.cross(u, t)


def pusht_scene(num_envs: int = 16, seed: int = 1):
    """PushTEnv.init(numEnvs:seed:) with the grid layout
    (RL/PushTEnv.swift:114-183, buildOne :194-246): one collision group per
    environment, each with a vertical capsule pusher tip driven by a soft
    world joint (the drag joint, moved with set_joint_world_anchors) plus an
    angular weld, a T block of two welded boxes at a seeded pose, and a
    fence.  Returns (scene, envs): envs[e] is a dict with the body ids
    (tip, bar, stem), the drag joint, the centre and the goal."""
    s = PhysicsScene("pusht")
    st = s.settings
    st.iterations, st.beta_lin, st.lambda_max = 16, 20000.0, 600.0
    cols = int(math.ceil(math.sqrt(num_envs)))
    rows = int(math.ceil(num_envs / cols))
    hx, hy = 0.5 * (cols - 1) * PUSHT_PITCH, 0.5 * (rows - 1) * PUSHT_PITCH
    s.add_body((2 * (hx + 3.5), 2 * (hy + 3.5), 2.0), 0.0, 1.3, (0.0, 0.0, -1.0))
    rng = SplitMix64(seed)
    inf = float("inf")
    envs = []
    for e in range(num_envs):
        c = np.array([(e % cols) * PUSHT_PITCH - hx, (e // cols) * PUSHT_PITCH - hy, 0.0])
        g = e + 1
        tip = s.add_body((0.7, 0.09, 0.0), 1.2, 0.35, tuple(c + (1.4, 0.0, PUSHT_TIP_HEIGHT)),
                         shape=abi.SHAPE_CAPSULE, collision_group=g)
        drag = len(s.joints)
        s.add_joint(SceneJoint(-1, tip, tuple(c + (1.4, 0.0, PUSHT_TIP_HEIGHT)), (0, 0, 0),
                               stiffness_lin=PUSHT_PUSHER_FORCE / 0.08, stiffness_ang=0.0))
        s.add_joint(SceneJoint(-1, tip, (0, 0, 0), (0, 0, 0), stiffness_lin=0.0, stiffness_ang=inf))
        ang = rng.next_float() * 2.0 * math.pi
        rad = 0.55 + rng.next_float() * 1.0
        byaw = (rng.next_float() - 0.5) * 2.0 * math.pi
        q = quat_axis_angle(byaw, (0, 0, 1))
        block = c + (math.cos(ang) * rad, math.sin(ang) * rad, 0.0)
        pbar = block + _qrot(q, (0.0, 0.125, 0.0)) + (0, 0, 0.09)
        pstem = block + _qrot(q, (0.0, -0.325, 0.0)) + (0, 0, 0.09)
        bar = s.add_body((1.0, 0.25, 0.18), 3.0, 1.1, tuple(pbar), rotation=q, collision_group=g)
        stem = s.add_body((0.25, 0.65, 0.18), 3.0, 1.1, tuple(pstem), rotation=q, collision_group=g)
        mid = (np.asarray(s.bodies[bar].position) + np.asarray(s.bodies[stem].position)) * 0.5
        qi = (-q[0], -q[1], -q[2], q[3])
        s.add_joint(SceneJoint(bar, stem, tuple(_qrot(qi, mid - np.asarray(s.bodies[bar].position))),
                               tuple(_qrot(qi, mid - np.asarray(s.bodies[stem].position))),
                               stiffness_lin=inf, stiffness_ang=inf))
        s.add_joint(SceneJoint(bar, stem, (0, 0, 0), (0, 0, 0), stiffness_lin=0.0, stiffness_ang=0.0))
        for sgn in (-1.0, 1.0):
            s.add_body((6.4, 0.12, 0.45), 0.0, 0.4, tuple(c + (0.0, sgn * 3.2, 0.22)), collision_group=g)
            s.add_body((0.12, 6.4, 0.45), 0.0, 0.4, tuple(c + (sgn * 3.2, 0.0, 0.22)), collision_group=g)
        envs.append(dict(tip=tip, bar=bar, stem=stem, drag_joint=drag, center=(float(c[0]), float(c[1])),
                         goal_pos=(0.85, 0.85), goal_yaw=0.0))
    return s, envs


def pusht_env_table(envs, half_window: float = 3.25):
    """PushTEnvGPU records of a batch (RL/PushTEnv.swift:569-575) as a
    ctypes array: the window covers the whole arena."""
    out = (abi.PushTEnv * len(envs))()
    for t, r in zip(out, envs):
        t.ids[:] = [r["tip"], r["bar"], r["stem"], 0]
        t.frame[:] = [r["center"][0], r["center"][1], r["goal_pos"][0], r["goal_pos"][1]]
        t.goal[:] = [r["goal_yaw"], half_window, 0.0, 0.0]
    return out


def pusht_tip_anchors(envs, targets):
    """World anchor points of the drag joints for env-local tip targets
    (setTipTarget, RL/PushTEnv.swift:258-262): targets clamped to +-3.02 m."""
    t = np.clip(np.asarray(targets, np.float64).reshape(-1, 2), -3.02, 3.02)
    pts = [(r["center"][0] + t[i, 0], r["center"][1] + t[i, 1], PUSHT_TIP_HEIGHT) for i, r in enumerate(envs)]
    return [r["drag_joint"] for r in envs], np.asarray(pts, np.float32)


def skin_bindings_for_tets(scene, per_tet: int = 1, seed: int = 9):
    """Render-skin bindings for a tet scene: `per_tet` points inside each
    tet (random barycentric weights), bound to its four vertices with a
    seeded rest normal; zero inverses (computed from the rest pose on
    upload)."""
    rng = np.random.default_rng(seed)
    out = []
    for t in scene.tets:
        for _ in range(per_tet):
            w = rng.dirichlet(np.ones(4)).astype(np.float32)
            b = abi.SkinBinding()
            b.ids[:] = list(t.ids)
            b.weights[:] = [float(x) for x in w]
            n = rng.normal(size=3)
            b.rest_normal[:] = [float(n[0]), float(n[1]), float(n[2]), 0.0]
            out.append(b)
    return out


SCENES = {
    "rigid-stack": rigid_stack_scene,
    "soft-cube": soft_cube_scene,
    "cloth-sphere": cloth_sphere_scene,
    "mixed": mixed_scene,
}
