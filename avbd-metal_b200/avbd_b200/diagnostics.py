"""Host-side diagnostics over solver state (GPUSolver.debugClothMetrics,
GPUSolver.swift:2687-2770, and the particle kinetic energy the reference's
cloth tests sum, ClothTests.swift)."""
from __future__ import annotations

import numpy as np

from .scene import PhysicsScene


def _closest_points(p, a, b, c):
    """Closest point on triangles (a, b, c) to points p, row-wise (Ericson)."""
    ab, ac, ap = b - a, c - a, p - a
    d1 = np.einsum("ij,ij->i", ab, ap)
    d2 = np.einsum("ij,ij->i", ac, ap)
    bp = p - b
    d3 = np.einsum("ij,ij->i", ab, bp)
    d4 = np.einsum("ij,ij->i", ac, bp)
    cp = p - c
    d5 = np.einsum("ij,ij->i", ab, cp)
    d6 = np.einsum("ij,ij->i", ac, cp)
    vc = d1 * d4 - d3 * d2
    vb = d5 * d2 - d1 * d6
    va = d3 * d6 - d5 * d4
    denom = va + vb + vc
    with np.errstate(divide="ignore", invalid="ignore"):
        v = np.where(np.abs(denom) < 1e-20, 0.0, vb / denom)
        w = np.where(np.abs(denom) < 1e-20, 0.0, vc / denom)
        q = a + ab * v[:, None] + ac * w[:, None]
        e1 = (d4 - d3) / np.maximum((d4 - d3) + (d5 - d6), 1e-12)
        q = np.where(((va <= 0) & ((d4 - d3) >= 0) & ((d5 - d6) >= 0))[:, None], b + (c - b) * e1[:, None], q)
        e2 = d2 / np.maximum(d2 - d6, 1e-12)
        q = np.where(((vb <= 0) & (d2 >= 0) & (d6 <= 0))[:, None], a + ac * e2[:, None], q)
        q = np.where(((d6 >= 0) & (d5 <= d6))[:, None], c, q)
        e3 = d1 / np.maximum(d1 - d3, 1e-12)
        q = np.where(((vc <= 0) & (d1 >= 0) & (d3 <= 0))[:, None], a + ab * e3[:, None], q)
        q = np.where(((d3 >= 0) & (d4 <= d3))[:, None], b, q)
        q = np.where(((d1 <= 0) & (d2 <= 0))[:, None], a, q)
    return q


def cloth_metrics(scene: PhysicsScene, positions: np.ndarray):
    """(minGap, maxStretch) of debugClothMetrics: the smallest skin-corrected
    distance from a surface particle to a triangle outside its one-ring, and
    the largest relative stretch of the stiff springs and hard rods."""
    pos = np.asarray(positions, dtype=np.float64)[:, :3]
    radius = np.array([b.size[0] * 0.5 for b in scene.bodies])
    tris = np.array([t.ids for t in scene.tris], dtype=np.int64).reshape(-1, 3)
    ring = {}
    for a, b, c in tris:
        for u, v in ((a, b), (b, c), (a, c)):
            ring.setdefault(u, set()).add(v)
            ring.setdefault(v, set()).add(u)
    verts = sorted(set(tris.ravel().tolist())) if len(tris) else []
    min_gap = np.inf
    for v in verts:
        nb = ring.get(v, set())
        mask = np.array([(v not in t) and not (t[0] in nb or t[1] in nb or t[2] in nb) for t in tris])
        if not mask.any():
            continue
        t = tris[mask]
        p = np.repeat(pos[v][None, :], len(t), axis=0)
        q = _closest_points(p, pos[t[:, 0]], pos[t[:, 1]], pos[t[:, 2]])
        rt = np.maximum(radius[t[:, 0]], np.maximum(radius[t[:, 1]], radius[t[:, 2]]))
        gaps = np.linalg.norm(p - q, axis=1) - (radius[v] + rt)
        min_gap = min(min_gap, float(gaps.min()))
    max_stretch = 0.0
    for s in scene.springs:
        if not (s.stiffness >= 1000 or s.hard):
            continue
        rest = s.rest
        if rest < 0:
            rest = float(np.linalg.norm(np.array(scene.bodies[s.body_a].position) -
                                        np.array(scene.bodies[s.body_b].position)))
        if rest > 1e-6:
            st = float(np.linalg.norm(pos[s.body_a] - pos[s.body_b])) / rest - 1.0
            max_stretch = max(max_stretch, st)
    return (0.0 if min_gap == np.inf else min_gap), max_stretch


def particle_kinetic_energy(scene: PhysicsScene, velocities: np.ndarray, masses: np.ndarray) -> float:
    """Sum of 1/2 m |v|^2 over the scene's particles."""
    v = np.asarray(velocities, dtype=np.float64)[:, :3]
    idx = [i for i, b in enumerate(scene.bodies) if b.is_particle]
    return float(0.5 * np.sum(masses[idx] * np.sum(v[idx] ** 2, axis=1)))
