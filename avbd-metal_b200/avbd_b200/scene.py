"""Back-end-neutral scene description: the Python mirror of the reference's
`PhysicsScene` / `SimSettings` (Sources/SimCore/Scenes/Scene.swift:34-752).

Field names and defaults follow the reference.  Arithmetic that the reference
performs in Float (e.g. the particle density of `addParticle`, Scene.swift:723-737)
is done here in numpy float32 in the same order, so the scene handed to the
solver is the scene the reference would build.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from . import abi

f32 = np.float32
INF = float("inf")


@dataclass
class SimSettings:
    """SimSettings (Scene.swift:485-545); render-only fields omitted."""
    dt: float = 1.0 / 60.0
    gravity: float = -10.0
    iterations: int = 10
    collision_margin: float = 0.01
    friction_combine_mode: int = 0
    alpha: float = 0.99
    beta_lin: float = 10000.0
    beta_ang: float = 100.0
    gamma: float = 0.999
    lambda_max: float = 1.0e6
    rod_decay_pow: float = 0.0
    particle_damping: float = 0.0
    rigid_linear_damping: float = 0.0
    rigid_angular_damping: float = 0.0
    cloth_viscosity: float = 0.0

    def to_c(self) -> abi.Settings:
        s = abi.Settings()
        s.dt = f32(self.dt)
        s.gravity = self.gravity
        s.iterations = int(self.iterations)
        s.collision_margin = self.collision_margin
        s.friction_combine_mode = int(self.friction_combine_mode)
        s.alpha = self.alpha
        s.beta_lin = self.beta_lin
        s.beta_ang = self.beta_ang
        s.gamma = self.gamma
        s.lambda_max = self.lambda_max
        s.rod_decay_pow = self.rod_decay_pow
        s.particle_damping = self.particle_damping
        s.rigid_linear_damping = self.rigid_linear_damping
        s.rigid_angular_damping = self.rigid_angular_damping
        s.cloth_viscosity = self.cloth_viscosity
        return s


def _qrot32(q, v):
    """Rotate v by the unit quaternion q = (x, y, z, w), in float32."""
    u = np.asarray(q[:3], dtype=np.float32)
    w = np.float32(q[3])
    v = np.asarray(v, dtype=np.float32)
    t = np.float32(2) * np.cross(u, v)
    return (v + w * t + np.cross(u, t)).astype(np.float32)


def _vec(v, n=3):
    return tuple(float(f32(x)) for x in v)[:n]


@dataclass
class SceneBody:
    size: Tuple[float, float, float]
    density: float
    friction: float
    position: Tuple[float, float, float]
    rotation: Tuple[float, float, float, float] = (0.0, 0.0, 0.0, 1.0)  # x, y, z, w
    velocity: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    shape: int = abi.SHAPE_BOX
    dynamic_friction: Optional[float] = None
    mass: Optional[float] = None
    diagonal_inertia: Optional[Tuple[float, float, float]] = None
    gravity_scale: float = 1.0
    is_particle: bool = False

    @property
    def is_dynamic(self) -> bool:
        if self.mass is not None:
            return self.mass > 0
        return self.density > 0


@dataclass
class SceneCollider:
    body: int
    size: Tuple[float, float, float]
    friction: float
    dynamic_friction: Optional[float] = None
    local_position: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    local_rotation: Tuple[float, float, float, float] = (0.0, 0.0, 0.0, 1.0)
    shape: int = abi.SHAPE_BOX
    collision_group: int = 0
    collides_with_shared: bool = True
    collision_enabled: bool = True
    world_round_anchor: bool = False
    hull_vertices: Optional[List[Tuple[float, float, float]]] = None  # centred, collider frame


@dataclass
class SceneJoint:
    body_a: int
    body_b: int
    r_a: Tuple[float, float, float]
    r_b: Tuple[float, float, float]
    stiffness_lin: float = INF
    stiffness_ang: float = 0.0
    fracture: float = INF
    fracture_linear: bool = False
    hinge_axis: Optional[Tuple[float, float, float]] = None
    motor_target: float = 0.0
    motor_torque: float = 0.0
    motor_rate: float = 0.0
    motor_stiffness: float = 0.0
    motor_damping: float = 0.0
    motor_mode: int = abi.MOTOR_IMPLICIT_POSITION_PD
    armature: float = 0.0
    limit_lo: float = 1.0
    limit_hi: float = -1.0


@dataclass
class SceneSpring:
    body_a: int
    body_b: int
    r_a: Tuple[float, float, float]
    r_b: Tuple[float, float, float]
    stiffness: float
    rest: float = -1.0
    hard: bool = False


@dataclass
class SceneTet:
    ids: Tuple[int, int, int, int]
    mu: float
    lam: float
    self_collision: bool = False


@dataclass
class SceneTri:
    ids: Tuple[int, int, int]
    mu: float = 0.0
    lam: float = 0.0
    bend: float = 0.0


@dataclass
class SceneSpinner:
    body: int
    axis: Tuple[float, float, float]
    omega: float


class PhysicsScene:
    """PhysicsScene (Scene.swift:547-752)."""

    def __init__(self, name: str = "scene"):
        self.name = name
        self.bodies: List[SceneBody] = []
        self.colliders: List[SceneCollider] = []
        self.joints: List[SceneJoint] = []
        self.springs: List[SceneSpring] = []
        self.tets: List[SceneTet] = []
        self.tris: List[SceneTri] = []
        self.exclusions: List[Tuple[int, int]] = []
        self.spinners: List[SceneSpinner] = []
        self.settings = SimSettings()

    # -- builders mirroring Scene.swift ----------------------------------
    def add_body(self, size, density, friction, position, rotation=(0, 0, 0, 1),
                 velocity=(0, 0, 0), shape=abi.SHAPE_BOX, dynamic_friction=None,
                 mass=None, diagonal_inertia=None, gravity_scale=1.0,
                 collision_group=0, collision_enabled=True) -> int:
        """addBody (Scene.swift:565-591): one body plus its own collider."""
        if shape == abi.SHAPE_SPHERE:
            size = (size[0], size[0], size[0])
        if (mass is None) != (diagonal_inertia is None):
            raise ValueError("explicit mass and diagonal inertia must be supplied together")
        self.bodies.append(SceneBody(
            size=_vec(size), density=density, friction=friction, position=_vec(position),
            rotation=_vec(rotation, 4), velocity=_vec(velocity), shape=shape,
            dynamic_friction=dynamic_friction, mass=mass,
            diagonal_inertia=diagonal_inertia, gravity_scale=gravity_scale))
        b = len(self.bodies) - 1
        if collision_enabled:
            self.colliders.append(SceneCollider(
                body=b, size=self.bodies[b].size, friction=friction,
                dynamic_friction=dynamic_friction, shape=shape,
                collision_group=collision_group,
                world_round_anchor=(shape != abi.SHAPE_BOX)))
        return b

    def add_collider(self, body, size, friction=None, dynamic_friction=None,
                     local_position=(0, 0, 0), local_rotation=(0, 0, 0, 1),
                     shape=abi.SHAPE_BOX, collision_group=0,
                     collides_with_shared=True, collision_enabled=True) -> int:
        """addCollider (Scene.swift:611-637)."""
        if not 0 <= body < len(self.bodies):
            raise ValueError("collider owner out of range")
        if shape == abi.SHAPE_SPHERE:
            size = (size[0], size[0], size[0])
        b = self.bodies[body]
        self.colliders.append(SceneCollider(
            body=body, size=_vec(size), friction=b.friction if friction is None else friction,
            dynamic_friction=(dynamic_friction if dynamic_friction is not None
                              else (b.dynamic_friction if b.dynamic_friction is not None
                                    else b.friction)),
            local_position=_vec(local_position), local_rotation=_vec(local_rotation, 4),
            shape=shape, collision_group=collision_group,
            collides_with_shared=collides_with_shared,
            collision_enabled=collision_enabled, world_round_anchor=False))
        return len(self.colliders) - 1

    def add_convex_collider(self, body, vertices, friction=None, dynamic_friction=None,
                            local_position=(0, 0, 0), local_rotation=(0, 0, 0, 1),
                            collision_group=0, collides_with_shared=True,
                            collision_enabled=True) -> int:
        """addConvexCollider (Scene.swift:645-676): 4...64 cooked hull
        vertices in the collider frame; the collider becomes the vertices'
        tight box, its origin moved to the box centre without changing the
        geometry.  The narrowphase contacts hulls against boxes only."""
        v = np.asarray(vertices, dtype=np.float32).reshape(-1, 3)
        if not 4 <= len(v) <= 64:
            raise ValueError("convex collider requires 4...64 cooked hull vertices")
        if not np.isfinite(v).all():
            raise ValueError("convex collider vertices must be finite")
        lo, hi = v.min(axis=0), v.max(axis=0)
        center = (lo + hi) * np.float32(0.5)
        centered = v - center
        q = np.asarray(local_rotation, dtype=np.float32)
        shift = _qrot32(q, center)
        lp = np.asarray(local_position, dtype=np.float32) + shift
        c = self.add_collider(body, tuple(float(x) for x in hi - lo), friction=friction,
                              dynamic_friction=dynamic_friction, local_position=tuple(float(x) for x in lp),
                              local_rotation=local_rotation, shape=abi.SHAPE_BOX,
                              collision_group=collision_group, collides_with_shared=collides_with_shared,
                              collision_enabled=collision_enabled)
        self.colliders[c].hull_vertices = [tuple(float(x) for x in row) for row in centered]
        return c

    def add_sphere(self, diameter, density, friction, position, velocity=(0, 0, 0)) -> int:
        return self.add_body((diameter, diameter, diameter), density, friction, position,
                             velocity=velocity, shape=abi.SHAPE_SPHERE)

    def add_capsule(self, length, radius, density, friction, position, rotation=(0, 0, 0, 1),
                    velocity=(0, 0, 0)) -> int:
        """addCapsule (Scene.swift:687-694): axis along local z, size
        (length, radius, 0)."""
        return self.add_body((length, radius, 0.0), density, friction, position, rotation=rotation,
                             velocity=velocity, shape=abi.SHAPE_CAPSULE)

    def add_torus(self, major, minor, density, friction, position, rotation=(0, 0, 0, 1),
                  velocity=(0, 0, 0)) -> int:
        """addTorus (Scene.swift:696-703): axis along local z, size
        (major, minor, 0)."""
        return self.add_body((major, minor, 0.0), density, friction, position, rotation=rotation,
                             velocity=velocity, shape=abi.SHAPE_TORUS)

    def add_particle(self, radius, mass, friction=0.5, position=(0, 0, 0),
                     velocity=(0, 0, 0)) -> int:
        """addParticle (Scene.swift:720-737): density chosen in Float so the
        sphere volume formula reproduces `mass`."""
        r = f32(radius)
        vol = f32(4.0) / f32(3.0) * f32(math.pi) * r * r * r
        density = f32(mass) / vol
        d = float(r * f32(2))
        self.bodies.append(SceneBody(
            size=(d, d, d), density=float(density), friction=friction,
            position=_vec(position), velocity=_vec(velocity), shape=abi.SHAPE_SPHERE,
            is_particle=True))
        b = len(self.bodies) - 1
        self.colliders.append(SceneCollider(
            body=b, size=(d, d, d), friction=friction, shape=abi.SHAPE_SPHERE,
            world_round_anchor=True))
        return b

    def add_joint(self, j: SceneJoint) -> None:
        if j.hinge_axis is not None:
            a = np.asarray(j.hinge_axis, dtype=np.float32)
            j.hinge_axis = tuple(float(x) for x in a / np.float32(np.sqrt(np.float32(a @ a))))
        self.joints.append(j)

    def add_spring(self, s: SceneSpring) -> None:
        self.springs.append(s)

    def add_tet(self, t: SceneTet) -> None:
        self.tets.append(t)

    def add_tri(self, t: SceneTri) -> None:
        self.tris.append(t)

    def add_collision_exclusion(self, a: int, b: int) -> None:
        self.exclusions.append((a, b))

    def add_spinner(self, sp: SceneSpinner) -> None:
        self.spinners.append(sp)

    # -- C descriptor ------------------------------------------------------
    def to_desc(self, max_pairs_per_body: int = 16,
                truncation: int = abi.TRUNCATION_AUTOMATIC,
                tet_inversion_prevention: bool = False, device: int = -1):
        """Flatten into an `avbd_scene_desc`. Returns (desc, keepalive).

        Records are packed through numpy structured arrays whose dtype is the
        ctypes record layout, so large scenes convert at C speed."""
        keep = []

        def pack(ctype, rows):
            dt = np.dtype(ctype)
            a = np.array(rows, dtype=dt) if rows else np.zeros(1, dtype=dt)
            a = np.ascontiguousarray(a)
            keep.append(a)
            return len(rows), a.ctypes.data_as(C.POINTER(ctype))

        def dyn(fr, dfr):
            return fr if dfr is None else dfr

        bodies = [(b.size, b.density, b.friction, dyn(b.friction, b.dynamic_friction),
                   b.position, b.rotation, b.velocity, b.shape, 1 if b.is_particle else 0,
                   0 if b.mass is None else 1, 0.0 if b.mass is None else b.mass,
                   (0.0, 0.0, 0.0) if b.diagonal_inertia is None else tuple(b.diagonal_inertia),
                   b.gravity_scale) for b in self.bodies]
        hull_rows = []
        colliders = []
        for c in self.colliders:
            first, count = 0, 0
            if c.hull_vertices:
                first, count = len(hull_rows), len(c.hull_vertices)
                hull_rows.extend(c.hull_vertices)
            colliders.append((c.body, c.size, c.friction, dyn(c.friction, c.dynamic_friction),
                              c.local_position, c.local_rotation, c.shape, c.collision_group,
                              1 if c.collides_with_shared else 0, 1 if c.collision_enabled else 0,
                              1 if c.world_round_anchor else 0, first, count))
        joints = [(j.body_a, j.body_b, _vec(j.r_a), _vec(j.r_b), j.stiffness_lin,
                   j.stiffness_ang, j.fracture, 1 if j.fracture_linear else 0,
                   0 if j.hinge_axis is None else 1,
                   (0.0, 0.0, 0.0) if j.hinge_axis is None else tuple(j.hinge_axis),
                   j.motor_target, j.motor_torque, j.motor_rate, j.motor_stiffness,
                   j.motor_damping, j.motor_mode, j.armature, j.limit_lo, j.limit_hi)
                  for j in self.joints]
        springs = [(s.body_a, s.body_b, _vec(s.r_a), _vec(s.r_b), s.stiffness, s.rest,
                    1 if s.hard else 0) for s in self.springs]
        tets = [(t.ids, t.mu, t.lam, 1 if t.self_collision else 0) for t in self.tets]
        tris = [(t.ids, t.mu, t.lam, t.bend) for t in self.tris]
        excl = [tuple(e) for e in self.exclusions]
        spin = [(s.body, _vec(s.axis), s.omega) for s in self.spinners]

        desc = abi.SceneDesc()
        desc.abi_version = abi.ABI_VERSION
        desc.num_bodies, desc.bodies = pack(abi.BodyDesc, bodies)
        desc.num_colliders, desc.colliders = pack(abi.ColliderDesc, colliders)
        hv = np.ascontiguousarray(np.asarray(hull_rows if hull_rows else [(0.0, 0.0, 0.0)],
                                             dtype=np.float32).reshape(-1))
        keep.append(hv)
        desc.num_hull_vertices = len(hull_rows)
        desc.hull_vertices = hv.ctypes.data_as(C.POINTER(C.c_float))
        desc.num_joints, desc.joints = pack(abi.JointDesc, joints)
        desc.num_springs, desc.springs = pack(abi.SpringDesc, springs)
        desc.num_tets, desc.tets = pack(abi.TetDesc, tets)
        desc.num_tris, desc.tris = pack(abi.TriDesc, tris)
        desc.num_exclusions, desc.exclusions = pack(abi.ExclusionDesc, excl)
        desc.num_spinners, desc.spinners = pack(abi.SpinnerDesc, spin)
        desc.settings = self.settings.to_c()
        desc.max_pairs_per_body = max_pairs_per_body
        desc.truncation_selection = truncation
        desc.tet_inversion_prevention = 1 if tet_inversion_prevention else 0
        desc.device = device
        return desc, keep
