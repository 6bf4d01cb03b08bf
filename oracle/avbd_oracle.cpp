// avbd_oracle.cpp — CPU oracle of the AVBD solver step ("Oracle A").
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE.  This file is a serial C++
// restatement of the reference's GPU solver path (LuckyIYI/avbd-metal,
// Sources/PhysicsAVBD/GPU/GPUSolver.swift + Shaders/*.metal) written for one
// purpose: to check the CUDA implementation.  Only tests/, the smoke() entry
// point and the cpu_baseline leg of bench.py may load it; the product library
// never links it.
//
// Semantics: the reference's stage order (GPUSolver.swift:3138-4375) with
// colors solved serially, bodies of one color in colorList order, and the
// 8-lane primal reduction order of primal_particles_split
// (40_solver.metal:1544-1684) reproduced exactly, so that — with IEEE float32
// arithmetic and no FMA contraction — the oracle is a bit-level reference for
// the GPU path.  Parity is "unpinned" against the reference itself (Swift and
// Metal cannot run here); it is pinned by the analytic gates of the
// reference's own tests (see tests/test_oracle_gates.py).
//
// Optional OpenMP: bodies of one color are independent, so the per-color loop
// may run in parallel without changing any result (used for the CPU baseline).
#include "oracle_solver.h"

namespace oracle {


// ==========================================================================
// Upload (GPUSolver.swift:338-638, :901-2081)
// ==========================================================================
static bool is_dynamic_desc(const avbd_body_desc& b) {
    if (b.has_explicit_mass) return b.mass > 0.0f;
    return b.density > 0.0f;
}

static std::vector<std::array<int, 3>> tet_boundary_faces(const avbd_scene_desc* s);

int Solver::create(const avbd_scene_desc* s) {
    if (!s || s->abi_version != AVBD_ABI_VERSION) { error = "bad scene descriptor"; return AVBD_ERR_INVALID_ARGUMENT; }
    settings = s->settings;
    nb = s->num_bodies;
    nc = s->num_colliders;
    for (uint32_t i = 0; i < nc; i++) {
        const avbd_collider_desc& c = s->colliders[i];
        if (c.body < 0 || (uint32_t)c.body >= nb) { error = "collider owner out of range"; return AVBD_ERR_INVALID_ARGUMENT; }
        if (c.shape > AVBD_SHAPE_CAPSULE) { error = "unknown collider shape"; return AVBD_ERR_INVALID_ARGUMENT; }
        if (c.hull_count > 0) {
            if (c.hull_count < 4 || c.hull_count > 64) { error = "a convex collider needs 4...64 hull vertices"; return AVBD_ERR_INVALID_ARGUMENT; }
            if (!s->hull_vertices || (uint64_t)c.hull_offset + c.hull_count > s->num_hull_vertices) { error = "hull vertex range out of range"; return AVBD_ERR_INVALID_ARGUMENT; }
            for (uint32_t k = 0; k < 3 * c.hull_count; k++)
                if (!std::isfinite(s->hull_vertices[3 * (size_t)c.hull_offset + k])) { error = "convex collider vertices must be finite"; return AVBD_ERR_INVALID_ARGUMENT; }
        }
    }
    for (uint32_t i = 0; i < nb; i++)
        if (s->bodies[i].shape > AVBD_SHAPE_CAPSULE) { error = "unknown body shape"; return AVBD_ERR_INVALID_ARGUMENT; }

    uint32_t enabled = 0;
    for (uint32_t i = 0; i < nc; i++) enabled += s->colliders[i].collision_enabled ? 1u : 0u;
    uint32_t mppb = s->max_pairs_per_body ? s->max_pairs_per_body : 16u;
    maxPairs = std::max<uint32_t>(4096u, enabled * mppb);
    mapCapacity = next_pow2(2 * maxPairs);
    gridHashSize = next_pow2(std::max<uint32_t>(64u, 2u * std::max<uint32_t>(1u, enabled)));

    std::vector<std::array<int, 3>> boundary = tet_boundary_faces(s);
    numTris = (uint32_t)boundary.size() + s->num_tris;

    posLin.assign(nb, F4{}); posAng.assign(nb, F4{}); initLin.assign(nb, F4{});
    initAng.assign(nb, F4{}); inertLin.assign(nb, F4{}); inertAng.assign(nb, F4{});
    velLin.assign(nb, F4{}); velAng.assign(nb, F4{}); prevVelLin.assign(nb, F4{});
    props.assign(nb, F4{}); shape.assign(nb, F4{}); spinVel.assign(nb, F4{});
    ogcPrev.assign(nb, F4{});
    gravityScale.assign(nb, 1.0f); shapeType.assign(nb, 0); boundsBits.assign(nb, 0x7F7F7F7Fu);
    clothGroup.assign(nb, 0); clothVert.assign(nb, 0);
    isDynamic.assign(nb, 0); isParticle.assign(nb, 0);
    colorsA.assign(nb, 0); colorsB.assign(nb, 0);

    const float PI = 3.14159265358979323846f;
    for (uint32_t i = 0; i < nb; i++) {
        const avbd_body_desc& b = s->bodies[i];
        float mass = 0.0f, radius = 0.0f;
        F3 moment = f3s(0);
        F3 size = f3(b.size[0], b.size[1], b.size[2]);
        if (b.shape == AVBD_SHAPE_BOX) {
            mass = b.density > 0.0f ? size.x * size.y * size.z * b.density : 0.0f;
            moment = F3{(size.y * size.y + size.z * size.z) / 12.0f * mass,
                        (size.x * size.x + size.z * size.z) / 12.0f * mass,
                        (size.x * size.x + size.y * size.y) / 12.0f * mass};
            radius = length(size * 0.5f);
        } else if (b.shape == AVBD_SHAPE_SPHERE) {
            float r = size.x / 2.0f;
            mass = b.density > 0.0f ? 4.0f / 3.0f * PI * r * r * r * b.density : 0.0f;
            moment = f3s(0.4f * mass * r * r);
            radius = r;
        } else if (b.shape == AVBD_SHAPE_TORUS) {
            float R = size.x, r = size.y;
            mass = b.density > 0.0f ? 2.0f * PI * PI * R * r * r * b.density : 0.0f;
            float iDia = mass * (R * R / 2.0f + 5.0f * r * r / 8.0f);
            float iAxis = mass * (R * R + 3.0f * r * r / 4.0f);
            moment = f3(iDia, iDia, iAxis);
            radius = R + r;
        } else {
            float L = size.x, r = size.y;
            mass = b.density > 0.0f ? PI * r * r * (L + 4.0f * r / 3.0f) * b.density : 0.0f;
            float iAxis = 0.5f * mass * r * r;
            float iPerp = mass * (L * L / 12.0f + r * r / 4.0f);
            moment = f3(iPerp, iPerp, iAxis);
            radius = L / 2.0f + r;
        }
        if (b.has_explicit_mass) {
            mass = b.mass;
            moment = f3(b.diagonal_inertia[0], b.diagonal_inertia[1], b.diagonal_inertia[2]);
        }
        posLin[i] = f4(b.position[0], b.position[1], b.position[2], mass);
        posAng[i] = f4(b.rotation[0], b.rotation[1], b.rotation[2], b.rotation[3]);
        velLin[i] = f4(b.velocity[0], b.velocity[1], b.velocity[2], 0.0f);
        prevVelLin[i] = velLin[i];
        props[i] = f4(moment, b.friction);
        shape[i] = f4(size, b.is_particle ? -radius : radius);
        gravityScale[i] = b.gravity_scale;
        shapeType[i] = b.shape;
        colorsA[i] = colorsB[i] = i % MAX_COLORS;
        isDynamic[i] = is_dynamic_desc(b) ? 1 : 0;
        isParticle[i] = b.is_particle ? 1 : 0;
    }
    scenePos = posLin;

    // colliders
    colOwner.assign(nc, 0); colShapeType.assign(nc, 0); colGroup.assign(nc, 0); colShared.assign(nc, 0);
    colShape.assign(nc, F4{}); colLocalPos.assign(nc, F4{}); colLocalRot.assign(nc, F4{});
    colFrictionS.assign(nc, 0); colFrictionD.assign(nc, 0);
    colHullFirst.assign(nc, 0); colHullCount.assign(nc, 0); hullVerts.clear();
    // bounding radius about the collider origin; the farthest hull vertex
    // for a convex hull (GPUSolver.swift:993-1002)
    auto collider_radius = [s](const avbd_collider_desc& c) -> float {
        if (c.hull_count > 0) {
            float r = 0.0f;
            for (uint32_t k = 0; k < c.hull_count; k++) {
                const float* v = s->hull_vertices + 3 * (size_t)(c.hull_offset + k);
                r = std::max(r, length(f3(v[0], v[1], v[2])));
            }
            return r;
        }
        F3 sz = f3(c.size[0], c.size[1], c.size[2]);
        if (c.shape == AVBD_SHAPE_SPHERE) return sz.x / 2.0f;
        if (c.shape == AVBD_SHAPE_TORUS) return sz.x + sz.y;
        if (c.shape == AVBD_SHAPE_CAPSULE) return sz.x / 2.0f + sz.y;
        return length(sz * 0.5f);
    };
    std::vector<float> radii;
    for (uint32_t i = 0; i < nc; i++) {
        const avbd_collider_desc& c = s->colliders[i];
        float r = collider_radius(c);
        bool particle = s->bodies[c.body].is_particle != 0;
        colOwner[i] = (uint32_t)c.body;
        colGroup[i] = c.collision_group;
        colShared[i] = c.collides_with_shared ? 1u : 0u;
        colShape[i] = f4(c.size[0], c.size[1], c.size[2], particle ? -r : r);
        colLocalPos[i] = f4(c.local_position[0], c.local_position[1], c.local_position[2], c.friction);
        colLocalRot[i] = f4(c.local_rotation[0], c.local_rotation[1], c.local_rotation[2], c.local_rotation[3]);
        colFrictionS[i] = c.friction;
        colFrictionD[i] = c.dynamic_friction;
        uint32_t flags = c.shape;
        if (c.hull_count > 0) {
            colHullFirst[i] = (uint32_t)hullVerts.size();
            colHullCount[i] = c.hull_count;
            for (uint32_t k = 0; k < c.hull_count; k++) {
                const float* v = s->hull_vertices + 3 * (size_t)(c.hull_offset + k);
                hullVerts.push_back(f3(v[0], v[1], v[2]));
            }
            flags = 4u;
        }
        if (particle) flags |= 0x10u;
        if (c.world_round_anchor) flags |= 0x20u;
        colShapeType[i] = flags;
        if (c.collision_enabled && isDynamic[c.body]) radii.push_back(r);
    }
    std::vector<float> sorted = radii;
    std::sort(sorted.begin(), sorted.end());
    float median = sorted.empty() ? 0.5f : sorted[sorted.size() / 2];
    float threshold = median * 4.0f;
    bool isolated = false;
    for (uint32_t i = 0; i < nc; i++)
        if (s->colliders[i].collision_enabled && s->colliders[i].collision_group != 0) isolated = true;
    hashedIdx.clear(); globalIdx.clear(); hashedRigidIdx.clear();
    for (uint32_t i = 0; i < nc; i++) {
        const avbd_collider_desc& c = s->colliders[i];
        if (!c.collision_enabled) continue;
        if (collider_radius(c) > threshold || (isolated && c.collision_group == 0)) globalIdx.push_back(i);
        else hashedIdx.push_back(i);
    }
    float maxHashedRadius = 0.05f;
    for (uint32_t i : hashedIdx) maxHashedRadius = fmax_(maxHashedRadius, std::fabs(colShape[i].w));
    for (uint32_t i : hashedIdx)
        if (!s->bodies[s->colliders[i].body].is_particle) hashedRigidIdx.push_back(i);

    // joints (GPUSolver.swift:1092-1195)
    uint32_t nj = s->num_joints;
    joints.assign(nj, JointGPU{});
    const float dt = settings.dt;
    for (uint32_t i = 0; i < nj; i++) {
        const avbd_joint_desc& j = s->joints[i];
        JointGPU g{};
        uint32_t aIdx = j.body_a >= 0 ? (uint32_t)j.body_a : WORLD_BODY;
        uint32_t flags = 0;
        if (std::isinf(j.stiffness_lin)) flags |= 1;
        if (std::isinf(j.stiffness_ang)) flags |= 2;
        if (std::isfinite(j.fracture)) flags |= 4;
        if (j.fracture_linear) flags |= 8;
        g.header = U4{aIdx, (uint32_t)j.body_b, 0, flags};
        const float bigK = 3.0e10f;
        g.rA = f4(j.r_a[0], j.r_a[1], j.r_a[2], fmin_(j.stiffness_lin, bigK));
        g.rB = f4(j.r_b[0], j.r_b[1], j.r_b[2], fmin_(j.stiffness_ang, bigK));
        F3 sizeA = j.body_a >= 0 ? f3(s->bodies[j.body_a].size[0], s->bodies[j.body_a].size[1],
                                      s->bodies[j.body_a].size[2]) : f3s(0);
        F3 sizeB = f3(s->bodies[j.body_b].size[0], s->bodies[j.body_b].size[1], s->bodies[j.body_b].size[2]);
        F3 ss = sizeA + sizeB;
        float torqueArm = dot(ss, ss);
        g.C0Lin = f4(0, 0, 0, torqueArm);
        g.C0Ang = f4(0, 0, 0, fmin_(j.fracture, 3.0e18f));
        F4 qA0 = j.body_a >= 0 ? posAng[j.body_a] : f4(0, 0, 0, 1);
        F4 rel = q_mul(q_inv(qA0), posAng[j.body_b]);
        rel = rel / std::sqrt(dot4(rel, rel));
        g.restRel = rel;
        if (j.has_hinge) {
            g.hingeAxis = f4(j.hinge_axis[0], j.hinge_axis[1], j.hinge_axis[2], 1.0f);
            g.dynamics.x = j.armature;
            if (j.motor_torque > 0.0f) {
                g.motor = f4(j.motor_target, j.motor_torque, 0.0f, j.motor_stiffness);
                g.limits = f4(j.limit_lo, j.limit_hi, j.motor_damping, 0.0f);
                if (j.motor_mode == AVBD_MOTOR_IMPLICIT_POSITION_PD) g.header.w |= MOTOR_IMPLICIT;
                else if (j.motor_mode == AVBD_MOTOR_EXPLICIT_TORQUE_PD) g.header.w |= MOTOR_EXPLICIT;
                else g.header.w |= MOTOR_VELOCITY;
                if (j.motor_rate != 0.0f) rateMotors.push_back(RateMotor{i, j.motor_rate});
            }
            if (j.limit_lo < j.limit_hi && j.motor_torque == 0.0f)
                g.limits = f4(j.limit_lo, j.limit_hi, 0.0f, 0.0f);
        }
        float massA = j.body_a >= 0 ? posLin[j.body_a].w : 0.0f;
        float massB = posLin[j.body_b].w;
        float eff = 0.0f;
        bool have = false;
        for (float m : {massA, massB}) if (m > 0.0f) { eff = have ? fmin_(eff, m) : m; have = true; }
        float floorK = fmin_(1.0e9f, fmax_(1.0f, eff / fmax_(dt * dt, 1.0e-12f)));
        if (std::isinf(j.stiffness_lin)) g.penaltyLin = f4(floorK, floorK, floorK, floorK);
        if (std::isinf(j.stiffness_ang)) g.penaltyAng = f4(floorK, floorK, floorK, floorK);
        if (j.stiffness_lin > 0.0f && std::isfinite(j.stiffness_lin)) {
            float k = fmin_(j.stiffness_lin, 1e9f); g.penaltyLin = f4(k, k, k, k);
        }
        if (j.stiffness_ang > 0.0f && std::isfinite(j.stiffness_ang)) {
            float k = fmin_(j.stiffness_ang, 1e9f); g.penaltyAng = f4(k, k, k, k);
        }
        joints[i] = g;
    }
    initPenLin.resize(nj); initPenAng.resize(nj);
    for (uint32_t i = 0; i < nj; i++) { initPenLin[i] = joints[i].penaltyLin; initPenAng[i] = joints[i].penaltyAng; }

    // springs (GPUSolver.swift:1197-1212)
    springs.assign(s->num_springs, SpringGPU{});
    for (uint32_t i = 0; i < s->num_springs; i++) {
        const avbd_spring_desc& sp = s->springs[i];
        SpringGPU g{};
        g.header = U4{(uint32_t)sp.body_a, (uint32_t)sp.body_b, sp.hard ? 1u : 0u, 0};
        float rest = sp.rest;
        if (rest < 0.0f) {
            F3 pA = xform(xyz(posLin[sp.body_a]), posAng[sp.body_a], f3(sp.r_a[0], sp.r_a[1], sp.r_a[2]));
            F3 pB = xform(xyz(posLin[sp.body_b]), posAng[sp.body_b], f3(sp.r_b[0], sp.r_b[1], sp.r_b[2]));
            rest = length(pA - pB);
        }
        g.rA = f4(sp.r_a[0], sp.r_a[1], sp.r_a[2], sp.stiffness);
        g.rB = f4(sp.r_b[0], sp.r_b[1], sp.r_b[2], rest);
        springs[i] = g;
    }

    // tets (GPUSolver.swift:1214-1235): DmInv rows via the adjugate.
    tets.assign(s->num_tets, TetGPU{});
    for (uint32_t i = 0; i < s->num_tets; i++) {
        const avbd_tet_desc& t = s->tets[i];
        F3 x0 = xyz(posLin[t.ids[0]]);
        F3 d0 = xyz(posLin[t.ids[1]]) - x0;
        F3 d1 = xyz(posLin[t.ids[2]]) - x0;
        F3 d2 = xyz(posLin[t.ids[3]]) - x0;
        float six = dot(d0, cross(d1, d2));
        float vol = std::fabs(six) / 6.0f;
        // Dm has columns d0, d1, d2; inverse rows are (d1 x d2, d2 x d0, d0 x d1) / det.
        F3 r0 = cross(d1, d2) / six;
        F3 r1 = cross(d2, d0) / six;
        F3 r2 = cross(d0, d1) / six;
        TetGPU g{};
        g.ids = U4{(uint32_t)t.ids[0], (uint32_t)t.ids[1], (uint32_t)t.ids[2], (uint32_t)t.ids[3]};
        g.r0 = f4(r0, six);
        g.r1 = f4(r1, t.mu * vol);
        g.r2 = f4(r2, t.lambda * vol);
        tets[i] = g;
    }

    // exclusions (GPUSolver.swift:1265-1287)
    std::vector<uint64_t> excl;
    for (uint32_t i = 0; i < nj; i++)
        if (s->joints[i].body_a >= 0) {
            uint64_t lo = (uint64_t)std::min(s->joints[i].body_a, s->joints[i].body_b);
            uint64_t hi = (uint64_t)std::max(s->joints[i].body_a, s->joints[i].body_b);
            excl.push_back(lo << 32 | hi);
        }
    for (uint32_t i = 0; i < s->num_springs; i++) {
        uint64_t lo = (uint64_t)std::min(s->springs[i].body_a, s->springs[i].body_b);
        uint64_t hi = (uint64_t)std::max(s->springs[i].body_a, s->springs[i].body_b);
        excl.push_back(lo << 32 | hi);
    }
    for (uint32_t i = 0; i < s->num_exclusions; i++) {
        uint64_t lo = (uint64_t)std::min(s->exclusions[i].body_a, s->exclusions[i].body_b);
        uint64_t hi = (uint64_t)std::max(s->exclusions[i].body_a, s->exclusions[i].body_b);
        excl.push_back(lo << 32 | hi);
    }
    std::sort(excl.begin(), excl.end());
    excl.erase(std::unique(excl.begin(), excl.end()), excl.end());
    exclusions.clear();
    for (uint64_t k : excl) { exclusions.push_back((uint32_t)(k >> 32)); exclusions.push_back((uint32_t)(k & 0xFFFFFFFFu)); }

    bool ogcCandidate = false;
    if (numTris > 0) {
        int rc = cloth_upload(s, boundary);
        if (rc != AVBD_OK) return rc;
        // element contacts can arise unless the scene is one closed soft
        // surface without authored triangles or self-collision whose only
        // rigid colliders are far-reaching static ground slabs (then the
        // isotropic stages produce nothing and are skipped)
        std::set<uint32_t> groups;
        bool self = false;
        for (uint32_t v : particleIdx) { groups.insert(clothGroup[v]); self = self || selfCollision[v] != 0; }
        bool rigidReach = false;
        for (uint32_t i = 0; i < nc; i++) {
            const avbd_collider_desc& c = s->colliders[i];
            if (!c.collision_enabled || isParticle[c.body]) continue;
            bool slab = !isDynamic[c.body] && c.shape == AVBD_SHAPE_BOX && c.hull_count == 0 && c.size[0] >= 20.0f && c.size[1] >= 20.0f;
            rigidReach = rigidReach || !slab;
        }
        ogcCandidate = cloth || groups.size() > 1 || self || rigidReach;
    }

    // static coloring (GPUSolver.swift:1956-2049)
    dynamicColoring = (numTris == 0 && s->num_tets == 0);
    colorStart.assign(MAX_COLORS + 2, 0);
    if (!dynamicColoring) {
        std::vector<std::set<uint32_t>> adj(nb);
        auto link2 = [&](int a, int b) {
            if (a < 0 || b < 0) return;
            if (!(isDynamic[a] || isDynamic[b])) return;
            if (isDynamic[a] && isDynamic[b]) { adj[a].insert((uint32_t)b); adj[b].insert((uint32_t)a); }
        };
        for (uint32_t i = 0; i < nj; i++) {
            const avbd_joint_desc& j = s->joints[i];
            if (j.stiffness_lin != 0.0f || j.stiffness_ang != 0.0f || j.motor_torque != 0.0f) link2(j.body_a, j.body_b);
        }
        for (uint32_t i = 0; i < s->num_springs; i++) link2(s->springs[i].body_a, s->springs[i].body_b);
        for (uint32_t i = 0; i < s->num_tets; i++)
            for (int a = 0; a < 4; a++) for (int b = a + 1; b < 4; b++) link2(s->tets[i].ids[a], s->tets[i].ids[b]);
        std::vector<uint32_t> colors(nb, 0);
        uint32_t maxColor = 0;
        for (uint32_t v = 0; v < nb; v++) {
            if (!isDynamic[v]) continue;
            uint64_t used = 0;
            for (uint32_t n : adj[v]) if (n < v && colors[n] < 64) used |= (1ull << colors[n]);
            if (used == ~0ull) { error = "static coloring needs more than 64 colors"; failure = AVBD_FAIL_STATIC_COLOR_CAPACITY; return AVBD_ERR_RUNTIME_FAILURE; }
            uint32_t c = 0;
            while (used & (1ull << c)) c++;
            colors[v] = c;
            maxColor = std::max(maxColor, c);
        }
        staticUsedColors = maxColor + 1;
        std::vector<std::vector<uint32_t>> buckets(MAX_COLORS);
        for (uint32_t v = 0; v < nb; v++) if (isDynamic[v]) buckets[colors[v]].push_back(v);
        colorList.clear();
        for (int c = 0; c < MAX_COLORS; c++) {
            colorStart[c] = (uint32_t)colorList.size();
            colorCounts[c] = (uint32_t)buckets[c].size();
            colorList.insert(colorList.end(), buckets[c].begin(), buckets[c].end());
        }
        colorStart[MAX_COLORS] = (uint32_t)colorList.size();
        colorStart[MAX_COLORS + 1] = staticUsedColors;
        for (uint32_t v = 0; v < nb; v++) colorsA[v] = colors[v];
    }

    // per-frame buffers
    manifolds.assign(maxPairs, ManifoldGPU{});
    prevManifolds.assign(maxPairs, ManifoldGPU{});
    mapKeyA.assign(mapCapacity, 0); mapKeyB.assign(mapCapacity, 0); mapVal.assign(mapCapacity, 0);
    cellCount.assign(gridHashSize, 0); cellStart.assign(gridHashSize, 0); cellRigid.assign(gridHashSize, 0);
    cellBodies.assign(std::max<size_t>(1, hashedIdx.size()), 0);
    pairs.assign(2 * maxPairs, 0);

    // params
    P.numBodies = nb; P.numJoints = nj; P.numSprings = (uint32_t)springs.size();
    P.numTets = (uint32_t)tets.size(); P.mapCapacity = mapCapacity; P.maxPairs = maxPairs;
    P.cellSize = maxHashedRadius * 2.0f; P.gridHashSize = gridHashSize;
    P.numHashed = (uint32_t)hashedIdx.size(); P.numGlobals = (uint32_t)globalIdx.size();
    P.numHashedRigid = (uint32_t)hashedRigidIdx.size();
    P.numTris = numTris; P.numParticles = numTris == 0 ? 0 : numParticles;
    clothViscosity = settings.cloth_viscosity;
    P.maxSpeed = fmax_(30.0f, 1.5f * P.cellSize / settings.dt * 0.5f);

    spinners.assign(s->spinners, s->spinners + s->num_spinners);
    for (auto& sp : spinners)
        spinVel[sp.body] = f4(sp.axis[0] * sp.omega, sp.axis[1] * sp.omega, sp.axis[2] * sp.omega, 1.0f);
    // effectiveSurfaceTruncationMode (GPUSolver.swift:93-101)
    P.surfaceTruncationMode = 0;
    if (P.numParticles > 0) {
        uint32_t sel = s->truncation_selection;
        bool volumetricSelf = false;
        for (uint32_t i = 0; i < s->num_tets; i++) volumetricSelf = volumetricSelf || s->tets[i].self_collision;
        uint32_t automatic = (volumetricSelf || (s->num_tris > 0 && s->num_tets == 0)) ? 2u : 1u;
        P.surfaceTruncationMode = sel == AVBD_TRUNCATION_AUTOMATIC ? automatic : sel;
    }
    P.tetInversionPreventionEnabled = (P.surfaceTruncationMode == 2u && s->tet_inversion_prevention) ? 1u : 0u;
    P.planarDATRelaxation = 0.85f;
    if (P.surfaceTruncationMode == 2u && s->num_tets > 0) {
        error = "Planar-DAT truncation of tet surfaces is not restated";
        return AVBD_ERR_UNSUPPORTED;
    }
    ogc = ogcCandidate && P.surfaceTruncationMode == 1u;
    colorJacobi = (cloth && P.surfaceTruncationMode == 2u) || ogc;
    if (ogc) {
        maxSoft = maxSoftIso;
        softMapCapacity = softMapCapacityIso;
        soft.assign(maxSoft, SoftContactGPU{});
        prevSoft.assign(maxSoft, SoftContactGPU{});
        softKeyA.assign(softMapCapacity, 0); softKeyB.assign(softMapCapacity, 0); softVal.assign(softMapCapacity, 0);
    }
    return AVBD_OK;
}

// Boundary faces of a tet mesh: faces owned by exactly one tet, wound
// outward against the opposite vertex, sorted (GPUSolver.swift:875-897).
static std::vector<std::array<int, 3>> tet_boundary_faces(const avbd_scene_desc* s) {
    std::vector<std::array<int, 3>> out;
    if (s->num_tets == 0) return out;
    struct Face { std::array<int, 3> tri; int opp; int count; };
    std::map<std::array<int, 3>, Face> faces;
    static const int idx[4][4] = {{0, 1, 2, 3}, {0, 1, 3, 2}, {0, 2, 3, 1}, {1, 2, 3, 0}};
    for (uint32_t t = 0; t < s->num_tets; t++) {
        const int* ids = s->tets[t].ids;
        for (auto& f : idx) {
            std::array<int, 3> tri = {ids[f[0]], ids[f[1]], ids[f[2]]};
            std::array<int, 3> key = tri;
            std::sort(key.begin(), key.end());
            auto it = faces.find(key);
            if (it != faces.end()) it->second.count++;
            else faces[key] = Face{tri, ids[f[3]], 1};
        }
    }
    for (auto& kv : faces) {
        if (kv.second.count != 1) continue;
        int a = kv.second.tri[0], b = kv.second.tri[1], c = kv.second.tri[2];
        const float* pa = s->bodies[a].position;
        F3 A = f3(pa[0], pa[1], pa[2]);
        F3 B = f3(s->bodies[b].position[0], s->bodies[b].position[1], s->bodies[b].position[2]);
        F3 C = f3(s->bodies[c].position[0], s->bodies[c].position[1], s->bodies[c].position[2]);
        const float* po = s->bodies[kv.second.opp].position;
        F3 n = cross(B - A, C - A);
        if (dot(n, f3(po[0], po[1], po[2]) - A) > 0.0f) std::swap(b, c);
        out.push_back({a, b, c});
    }
    std::sort(out.begin(), out.end());
    return out;
}

void Solver::sync_params() {
    P.dt = settings.dt; P.gravity = settings.gravity; P.alpha = settings.alpha;
    P.betaLin = settings.beta_lin; P.betaAng = settings.beta_ang; P.gamma = settings.gamma;
    P.lambdaMax = settings.lambda_max; P.iterations = (uint32_t)settings.iterations;
    P.rodDecayPow = settings.rod_decay_pow; P.particleDamping = settings.particle_damping;
    P.frame = (uint32_t)frameIndex; P.frictionCombineMode = settings.friction_combine_mode;
    P.collisionMargin = fmax_(settings.collision_margin, 0.0f);
    P.rigidLinearDamping = fmax_(settings.rigid_linear_damping, 0.0f);
    P.rigidAngularDamping = fmax_(settings.rigid_angular_damping, 0.0f);
    clothViscosity = settings.cloth_viscosity;
}

// ==========================================================================
// Broadphase (20_broadphase.metal:69-131, :287-512)
// ==========================================================================
static inline F3 collider_center(const Solver& S, uint32_t c) {
    uint32_t b = S.colOwner[c];
    return xyz(S.posLin[b]) + q_rotate(S.posAng[b], xyz(S.colLocalPos[c]));
}

static bool pair_excluded(const std::vector<uint32_t>& ex, uint32_t a, uint32_t b) {
    uint32_t lo = 0, hi = (uint32_t)(ex.size() / 2);
    uint32_t count = hi;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t ex_ = ex[2 * mid], ey = ex[2 * mid + 1];
        if (ex_ < a || (ex_ == a && ey < b)) lo = mid + 1; else hi = mid;
    }
    if (lo >= count) return false;
    return ex[2 * lo] == a && ex[2 * lo + 1] == b;
}

uint32_t Solver::process_producer(uint32_t producer, bool emit, uint32_t base) {
    uint32_t count = 0;
    // Filters shared by the cell scan and the globals scan; every filter is a
    // pure predicate, so their order does not change the emitted set.
    auto test = [&](uint32_t a, uint32_t b, F3 pa, float ra, uint32_t ownerA, bool aDyn,
                    uint32_t outA, uint32_t outB) {
        (void)a;
        uint32_t ownerB = colOwner[b];
        if (ownerA == ownerB) return;
        if (!aDyn && posLin[ownerB].w <= 0.0f) return;
        float rb = std::fabs(colShape[b].w);
        F3 pb = collider_center(*this, b);
        F3 dp = pa - pb;
        float r = ra + rb;
        if (dot(dp, dp) > r * r) return;
        uint32_t lo = std::min(ownerA, ownerB), hi = std::max(ownerA, ownerB);
        if (pair_excluded(exclusions, lo, hi)) return;
        uint32_t slot = base + count;
        if (emit && slot < P.maxPairs) { pairs[2 * slot] = outA; pairs[2 * slot + 1] = outB; }
        count++;
    };
    if (producer < P.numHashed) {
        uint32_t a = hashedIdx[producer];
        uint32_t ownerA = colOwner[a];
        uint32_t groupA = colGroup[a];
        F3 pa = collider_center(*this, a);
        float ra = std::fabs(colShape[a].w);
        bool aDyn = posLin[ownerA].w > 0.0f;
        uint32_t ga = clothGroup[ownerA];
        bool scanCells = !(ga != 0 && P.numHashedRigid == 0);
        int cx, cy, cz;
        cell_coord(pa, P.cellSize, cx, cy, cz);
        if (scanCells) {
            uint32_t visited[27];
            uint32_t nv = 0;
            for (int dz = -1; dz <= 1; dz++)
                for (int dy = -1; dy <= 1; dy++)
                    for (int dx = -1; dx <= 1; dx++) {
                        uint32_t h = cell_hash(cx + dx, cy + dy, cz + dz, groupA, P.gridHashSize);
                        bool dup = false;
                        for (uint32_t v = 0; v < nv; v++) if (visited[v] == h) { dup = true; break; }
                        if (dup) continue;
                        visited[nv++] = h;
                        if (ga != 0 && cellRigid[h] == 0) continue;
                        uint32_t s0 = cellStart[h], e0 = s0 + cellCount[h];
                        for (uint32_t k = s0; k < e0; k++) {
                            uint32_t b = cellBodies[k];
                            if (b <= a) continue;
                            if (!domains_compatible(groupA, colGroup[b], colShared[a], colShared[b])) continue;
                            // soft surface vs soft surface: element contacts own it
                            if (ga != 0 && clothGroup[colOwner[b]] != 0) continue;
                            test(a, b, pa, ra, ownerA, aDyn, a, b);
                        }
                    }
        }
        for (uint32_t g = 0; g < P.numGlobals; g++) {
            uint32_t b = globalIdx[g];
            if (!domains_compatible(groupA, colGroup[b], colShared[a], colShared[b])) continue;
            if (ga != 0 && clothGroup[colOwner[b]] == ga) continue;
            test(a, b, pa, ra, ownerA, aDyn, std::min(a, b), std::max(a, b));
        }
    } else {
        uint32_t gp = producer - P.numHashed;
        if (gp >= P.numGlobals) return 0;
        uint32_t a = globalIdx[gp];
        uint32_t ownerA = colOwner[a];
        uint32_t groupA = colGroup[a];
        F3 pa = collider_center(*this, a);
        float ra = std::fabs(colShape[a].w);
        bool aDyn = posLin[ownerA].w > 0.0f;
        uint32_t ga = clothGroup[ownerA];
        for (uint32_t g = gp + 1; g < P.numGlobals; g++) {
            uint32_t b = globalIdx[g];
            if (!domains_compatible(groupA, colGroup[b], colShared[a], colShared[b])) continue;
            if (ga != 0 && clothGroup[colOwner[b]] == ga) continue;
            test(a, b, pa, ra, ownerA, aDyn, std::min(a, b), std::max(a, b));
        }
    }
    return count;
}

void Solver::broadphase() {
    std::fill(cellCount.begin(), cellCount.end(), 0u);
    std::fill(cellRigid.begin(), cellRigid.end(), 0u);
    std::vector<uint32_t> cellOf(P.numHashed);
    for (uint32_t i = 0; i < P.numHashed; i++) {
        uint32_t b = hashedIdx[i];
        F3 c = collider_center(*this, b);
        int x, y, z;
        cell_coord(c, P.cellSize, x, y, z);
        uint32_t h = cell_hash(x, y, z, colGroup[b], P.gridHashSize);
        cellOf[i] = h;
        cellCount[h]++;
        if (colShape[b].w >= 0.0f) cellRigid[h] = 1u;
    }
    uint32_t run = 0;
    for (uint32_t h = 0; h < P.gridHashSize; h++) { cellStart[h] = run; run += cellCount[h]; }
    std::vector<uint32_t> cursor(cellStart);
    for (uint32_t i = 0; i < P.numHashed; i++) cellBodies[cursor[cellOf[i]]++] = hashedIdx[i];
    for (uint32_t h = 0; h < P.gridHashSize; h++)
        std::sort(cellBodies.begin() + cellStart[h], cellBodies.begin() + cellStart[h] + cellCount[h]);

    uint32_t producers = P.numHashed + P.numGlobals;
    pairCount.assign(producers, 0);
    pairStart.assign(producers, 0);
    for (uint32_t p = 0; p < producers; p++) pairCount[p] = process_producer(p, false, 0);
    run = 0;
    for (uint32_t p = 0; p < producers; p++) { pairStart[p] = run; run += pairCount[p]; }
    for (uint32_t p = 0; p < producers; p++) process_producer(p, true, pairStart[p]);
    pairCandidates = run;
    numPairs = std::min(run, P.maxPairs);
}

// ==========================================================================
// Narrowphase: sphere/sphere, sphere/box, box/box (30_narrowphase.metal)
// ==========================================================================
struct Box { F3 center, half; F3 ax[3]; };
struct AxisBest { int type, ia, ib; float sep; F3 n; bool valid; };
static const float SAT_EPS = 1.0e-6f, PLANE_EPS = 1.0e-5f, MERGE_DIST_SQ = 1.0e-6f;
static const int NP_MAX_POLY = 16;

static inline float box_half(const Box& b, int i) { return comp(b.half, i); }

static float spec_cap(float ra, float rb, float margin) {
    float r = fmin_(std::fabs(ra), std::fabs(rb));
    return fmin_(0.25f, fmax_(4.0f * margin, 3.0f * r));
}
static float detect_margin(F3 n, F3 relVel, const Params& P, float ra, float rb) {
    float approach = fmax_(0.0f, -dot(relVel, n));
    float allowed = fmin_(approach * P.dt, spec_cap(ra, rb, P.collisionMargin));
    return P.collisionMargin + allowed;
}
static bool test_axis(const Box& A, const Box& B, F3 delta, F3 axis, int type, int ia, int ib,
                      F3 relVel, float cap, const Params& P, AxisBest& best) {
    float lenSq = dot(axis, axis);
    if (lenSq < SAT_EPS) return true;
    F3 n = axis * rsqrt_(lenSq);
    if (dot(n, delta) < 0.0f) n = -n;
    float dist = std::fabs(dot(delta, n));
    float rA = A.half.x * std::fabs(dot(n, A.ax[0])) + A.half.y * std::fabs(dot(n, A.ax[1]))
             + A.half.z * std::fabs(dot(n, A.ax[2]));
    float rB = B.half.x * std::fabs(dot(n, B.ax[0])) + B.half.y * std::fabs(dot(n, B.ax[1]))
             + B.half.z * std::fabs(dot(n, B.ax[2]));
    float sep = dist - (rA + rB);
    float approach = fmax_(0.0f, -dot(relVel, n));
    float allowed = fmin_(approach * P.dt, cap);
    if (sep > allowed) return false;
    if (!best.valid || sep > best.sep) { best.valid = true; best.type = type; best.ia = ia; best.ib = ib; best.sep = sep; best.n = n; }
    return true;
}
static F3 support(const Box& b, F3 dir) {
    float sx = dot(dir, b.ax[0]) >= 0.0f ? 1.0f : -1.0f;
    float sy = dot(dir, b.ax[1]) >= 0.0f ? 1.0f : -1.0f;
    float sz = dot(dir, b.ax[2]) >= 0.0f ? 1.0f : -1.0f;
    return b.center + b.ax[0] * (b.half.x * sx) + b.ax[1] * (b.half.y * sy) + b.ax[2] * (b.half.z * sz);
}
static void face_axes(const Box& b, int i, F3& u, F3& v, float& eu, float& ev) {
    if (i == 0) { u = b.ax[1]; v = b.ax[2]; eu = b.half.y; ev = b.half.z; }
    else if (i == 1) { u = b.ax[0]; v = b.ax[2]; eu = b.half.x; ev = b.half.z; }
    else { u = b.ax[0]; v = b.ax[1]; eu = b.half.x; ev = b.half.y; }
}
static int clip_poly(const F3* in, int n, F3 nrm, float off, F3* out) {
    if (n <= 0) return 0;
    int m = 0;
    F3 a = in[n - 1];
    float da = dot(nrm, a) - off;
    for (int i = 0; i < n; i++) {
        F3 b = in[i];
        float db = dot(nrm, b) - off;
        bool aIn = da <= PLANE_EPS, bIn = db <= PLANE_EPS;
        if (aIn != bIn) {
            float t = 0.0f, den = da - db;
            if (std::fabs(den) > SAT_EPS) t = clampf_(da / den, 0.0f, 1.0f);
            if (m < NP_MAX_POLY) out[m++] = a + (b - a) * t;
        }
        if (bIn && m < NP_MAX_POLY) out[m++] = b;
        a = b; da = db;
    }
    return m;
}
static void support_edge(const Box& b, int axis, F3 dir, F3& eA, F3& eB) {
    int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
    float s1 = dot(dir, b.ax[a1]) >= 0.0f ? 1.0f : -1.0f;
    float s2 = dot(dir, b.ax[a2]) >= 0.0f ? 1.0f : -1.0f;
    F3 c = b.center + b.ax[a1] * (box_half(b, a1) * s1) + b.ax[a2] * (box_half(b, a2) * s2);
    eA = c - b.ax[axis] * box_half(b, axis);
    eB = c + b.ax[axis] * box_half(b, axis);
}
static void closest_seg_seg(F3 p0, F3 p1, F3 q0, F3 q1, F3& c0, F3& c1) {
    F3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
    float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    float s = 0.0f, t = 0.0f;
    if (a <= SAT_EPS && e <= SAT_EPS) { c0 = p0; c1 = q0; return; }
    if (a <= SAT_EPS) {
        t = clampf_(f / e, 0.0f, 1.0f);
    } else {
        float c = dot(d1, r);
        if (e <= SAT_EPS) {
            s = clampf_(-c / a, 0.0f, 1.0f);
        } else {
            float b = dot(d1, d2);
            float den = a * e - b * b;
            if (std::fabs(den) > SAT_EPS) s = clampf_((b * f - c * e) / den, 0.0f, 1.0f);
            t = (b * s + f) / e;
            if (t < 0.0f) { t = 0.0f; s = clampf_(-c / a, 0.0f, 1.0f); }
            else if (t > 1.0f) { t = 1.0f; s = clampf_((b - c) / a, 0.0f, 1.0f); }
        }
    }
    c0 = p0 + d1 * s;
    c1 = q0 + d2 * t;
}
struct NPContact { F3 xA, xB; uint32_t feature; };
static bool add_contact(NPContact* cs, int& count, F3* mids, F3 xA, F3 xB, uint32_t feature) {
    F3 mid = (xA + xB) * 0.5f;
    for (int i = 0; i < count; i++) if (distance2(mid, mids[i]) < MERGE_DIST_SQ) return false;
    if (count >= MAX_CONTACTS) return false;
    cs[count] = NPContact{xA, xB, feature};
    mids[count] = mid;
    count++;
    return true;
}
// Tangential target shift of a kinematic spinner surface (30_narrowphase.metal:274-284).
static void spin_shift(F4 wA, F4 wB, F3 rAoff, F3 rBoff, F3 t1, F3 t2, float dt, float alpha,
                       float& sx, float& sy) {
    F3 sA = wA.w != 0.0f ? cross(xyz(wA), rAoff) * dt : f3s(0);
    F3 sB = wB.w != 0.0f ? cross(xyz(wB), rBoff) * dt : f3s(0);
    F3 rel = sB - sA;
    float k = 1.0f / fmax_(1.0f - alpha, 0.01f);
    sx = dot(t1, rel) * k;
    sy = dot(t2, rel) * k;
}
static F3 penalty_floor(const Solver& S, uint32_t ia, uint32_t ib) {
    float mA = S.posLin[ia].w, mB = S.posLin[ib].w;
    float minMass = fmin_(mA > 0.0f ? mA : FLT_MAX, mB > 0.0f ? mB : FLT_MAX);
    if (minMass == FLT_MAX) return f3s(PENALTY_MIN);
    float k = fmin_(PENALTY_MAX, fmax_(PENALTY_MIN, minMass / fmax_(S.P.dt * S.P.dt, 1e-12f)));
    return f3(k, fmin_(k, PENALTY_MAX_T), fmin_(k, PENALTY_MAX_T));
}

int Solver::map_find(uint32_t a, uint32_t b) const {
    uint32_t h = pair_map_hash(a, b, P.mapCapacity);
    for (uint32_t probe = 0; probe < P.mapCapacity; probe++) {
        uint32_t ka = mapKeyA[h];
        if (ka == 0) return -1;
        if (ka == a + 1 && mapKeyB[h] == b) return (int)mapVal[h];
        h = (h + 1) & (P.mapCapacity - 1u);
    }
    return -1;
}

// --------------------------------------------------------------------------
// Convex hull vs box, capsule and torus pairs (30_narrowphase.metal:189-340,
// :430-975).  Same contact rules as the sphere and box paths: feature-keyed
// warm start for hulls, proximity-matched for the round shapes.
// --------------------------------------------------------------------------
struct NPair {
    uint32_t ia, ib, ba, bb;
    F4 bodyPA, bodyPB, qBodyA, qBodyB, qA, qB;
    F3 vA, vB;
    Box A, B;
};

static void emit_feature_manifold(const Solver& S, const NPair& p, ManifoldGPU& outM,
                                  const NPContact* contacts, int count, F3 nrm) {
    const Params& P = S.P;
    F3 t1, t2;
    orthonormal(nrm, t1, t2);
    float sf = combine_friction(S.colFrictionS[p.ia], S.colFrictionS[p.ib], P.frictionCombineMode);
    float df = combine_friction(S.colFrictionD[p.ia], S.colFrictionD[p.ib], P.frictionCombineMode);
    int prev = S.map_find(p.ia, p.ib);
    outM.header = U4{p.ba, p.bb, (uint32_t)count, 1u};
    outM.basisN = f4(nrm, df);
    outM.basisT1 = f4(t1, sf);
    float warm = P.alpha * P.gamma;
    F4 qAc = q_conj(p.qBodyA), qBc = q_conj(p.qBodyB);
    for (int i = 0; i < count; i++) {
        F3 rA = q_rotate(qAc, contacts[i].xA - xyz(p.bodyPA));
        F3 rB = q_rotate(qBc, contacts[i].xB - xyz(p.bodyPB));
        F3 lambda = f3s(0), penalty = f3s(0);
        float stick = 0.0f;
        if (prev >= 0) {
            const ManifoldGPU& pm = S.prevManifolds[prev];
            for (uint32_t j = 0; j < pm.header.z; j++) {
                if (fbits(pm.contacts[j].rA.w) == contacts[i].feature) {
                    lambda = xyz(pm.contacts[j].lambda);
                    penalty = xyz(pm.contacts[j].penalty);
                    stick = pm.contacts[j].rB.w;
                    if (stick != 0.0f) { rA = xyz(pm.contacts[j].rA); rB = xyz(pm.contacts[j].rB); }
                    break;
                }
            }
        }
        F3 xAw = xform(xyz(p.bodyPA), p.qBodyA, rA);
        F3 xBw = xform(xyz(p.bodyPB), p.qBodyB, rB);
        F3 d = xAw - xBw;
        F3 C0 = f3(dot(nrm, d) + P.collisionMargin, dot(t1, d), dot(t2, d));
        float sx, sy;
        spin_shift(S.spinVel[p.ba], S.spinVel[p.bb], xAw - xyz(p.bodyPA), xBw - xyz(p.bodyPB), t1, t2, P.dt, P.alpha, sx, sy);
        C0.y -= sx; C0.z -= sy;
        lambda *= warm;
        penalty = clamp3(penalty * P.gamma, penalty_floor(S, p.ba, p.bb), f3(PENALTY_MAX, PENALTY_MAX_T, PENALTY_MAX_T));
        outM.contacts[i].rA = f4(rA, bitsf(contacts[i].feature));
        outM.contacts[i].rB = f4(rB, stick);
        outM.contacts[i].C0 = f4(C0, 0);
        outM.contacts[i].lambda = f4(lambda, 0);
        outM.contacts[i].penalty = f4(penalty, 0);
    }
}

// keepAnchors: capsules keep sticking anchors only between two
// material-anchored colliders (:711-724); tori never (:944-962).
static void emit_round_manifold(const Solver& S, const NPair& p, ManifoldGPU& outM, const NPContact* contacts,
                                int count, F3 nrm, float matchDist, bool capsuleRule) {
    const Params& P = S.P;
    F3 t1, t2;
    orthonormal(nrm, t1, t2);
    float sf = combine_friction(S.colFrictionS[p.ia], S.colFrictionS[p.ib], P.frictionCombineMode);
    float df = combine_friction(S.colFrictionD[p.ia], S.colFrictionD[p.ib], P.frictionCombineMode);
    int prev = S.map_find(p.ia, p.ib);
    bool roundA = (S.colShapeType[p.ia] & 0x20u) != 0, roundB = (S.colShapeType[p.ib] & 0x20u) != 0;
    outM.header = U4{p.ba, p.bb, (uint32_t)count, 1u | (roundA ? 2u : 0u) | (roundB ? 4u : 0u)};
    outM.basisN = f4(nrm, df);
    outM.basisT1 = f4(t1, sf);
    float warm = P.alpha * P.gamma;
    bool keepAnchors = capsuleRule && !roundA && !roundB;
    F4 qAc = q_conj(p.qBodyA), qBc = q_conj(p.qBodyB);
    for (int i = 0; i < count; i++) {
        F3 rA_ = roundA ? contacts[i].xA - xyz(p.bodyPA) : q_rotate(qAc, contacts[i].xA - xyz(p.bodyPA));
        F3 rB_ = roundB ? contacts[i].xB - xyz(p.bodyPB) : q_rotate(qBc, contacts[i].xB - xyz(p.bodyPB));
        F3 lambda = f3s(0), penalty = f3s(0);
        float stick = 0.0f;
        if (prev >= 0) {
            const ManifoldGPU& pm = S.prevManifolds[prev];
            float bestD = matchDist;
            int bestJ = -1;
            for (uint32_t j = 0; j < pm.header.z; j++) {
                float dj = distance(xyz(pm.contacts[j].rA), rA_);
                if (dj < bestD) { bestD = dj; bestJ = (int)j; }
            }
            if (bestJ >= 0) {
                lambda = xyz(pm.contacts[bestJ].lambda);
                penalty = xyz(pm.contacts[bestJ].penalty);
                F3 t1o = xyz(pm.basisT1);
                F3 t2o = cross(xyz(pm.basisN), t1o);
                F3 lt = t1o * lambda.y + t2o * lambda.z;
                lambda.y = dot(t1, lt);
                lambda.z = dot(t2, lt);
                if (keepAnchors) {
                    stick = pm.contacts[bestJ].rB.w;
                    if (stick != 0.0f) { rA_ = xyz(pm.contacts[bestJ].rA); rB_ = xyz(pm.contacts[bestJ].rB); }
                }
            }
        }
        // tori measure the gap between the hit points themselves
        // (30_narrowphase.metal:925-958); capsules between the points their
        // stored anchors give back (:727-731)
        F3 xAw = !capsuleRule ? contacts[i].xA
                              : (roundA ? xyz(p.bodyPA) + rA_ : xform(xyz(p.bodyPA), p.qBodyA, rA_));
        F3 xBw = !capsuleRule ? contacts[i].xB
                              : (roundB ? xyz(p.bodyPB) + rB_ : xform(xyz(p.bodyPB), p.qBodyB, rB_));
        F3 d = xAw - xBw;
        F3 C0 = f3(dot(nrm, d) + P.collisionMargin, dot(t1, d), dot(t2, d));
        float sx, sy;
        spin_shift(S.spinVel[p.ba], S.spinVel[p.bb], xAw - xyz(p.bodyPA), xBw - xyz(p.bodyPB), t1, t2, P.dt, P.alpha, sx, sy);
        C0.y -= sx; C0.z -= sy;
        lambda *= warm;
        penalty = clamp3(penalty * P.gamma, penalty_floor(S, p.ba, p.bb), f3(PENALTY_MAX, PENALTY_MAX_T, PENALTY_MAX_T));
        outM.contacts[i].rA = f4(rA_, bitsf(contacts[i].feature));
        outM.contacts[i].rB = f4(rB_, stick);
        outM.contacts[i].C0 = f4(C0, 0);
        outM.contacts[i].lambda = f4(lambda, 0);
        outM.contacts[i].penalty = f4(penalty, 0);
    }
}

static int min_axis(F3 v) {
    int a = 0;
    if (v.y < comp(v, a)) a = 1;
    if (v.z < comp(v, a)) a = 2;
    return a;
}

// 30_narrowphase.metal:286-290
static F3 closest_on_segment(F3 p, F3 a, F3 b) {
    F3 ab = b - a;
    float t = clampf_(dot(p - a, ab) / fmax_(dot(ab, ab), 1e-12f), 0.0f, 1.0f);
    return a + ab * t;
}

struct HullCand { F3 xHull, xBox, boxToHull; float sep; uint32_t feature; };

// 30_narrowphase.metal:203-246
static bool hull_vertex_box(F3 vw, uint32_t vid, const Box& box, F4 qBox, F3 rel, float hullR, float boxR,
                            const Params& P, HullCand& out) {
    F3 local = q_rotate(q_conj(qBox), vw - box.center);
    F3 h = box.half;
    F3 cl = clamp3(local, -h, h);
    F3 nL, bL;
    float sep;
    bool inside = local.x >= -h.x && local.y >= -h.y && local.z >= -h.z &&
                  local.x <= h.x && local.y <= h.y && local.z <= h.z;
    if (inside) {
        F3 clr = h - abs3(local);
        int axis = min_axis(clr);
        nL = f3s(0);
        setcomp(nL, axis, comp(local, axis) >= 0.0f ? 1.0f : -1.0f);
        bL = local;
        setcomp(bL, axis, comp(nL, axis) * comp(h, axis));
        sep = -comp(clr, axis);
    } else {
        F3 dl = local - cl;
        float dist = length(dl);
        if (dist < 1e-8f) return false;
        nL = dl / dist;
        float det = detect_margin(q_rotate(qBox, nL), rel, P, hullR, boxR);
        if (dist > det) return false;
        bL = cl;
        sep = dist;
    }
    out.xHull = vw;
    out.xBox = q_rotate(qBox, bL) + box.center;
    out.boxToHull = q_rotate(qBox, nL);
    out.sep = sep;
    out.feature = (4u << 24) | (vid & 0x00FFFFFFu);
    return true;
}

// 30_narrowphase.metal:430-545
static void narrow_hull(const Solver& S, const NPair& p, ManifoldGPU& outM, uint32_t stA, uint32_t stB) {
    const Params& P = S.P;
    bool hIsA = stA == 4;
    if ((stA == 4 && stB == 4) || (hIsA ? stB : stA) != 0) { outM.header = U4{p.ba, p.bb, 0, 0}; return; }
    uint32_t ih = hIsA ? p.ia : p.ib;
    F4 qH = hIsA ? p.qA : p.qB;
    F3 pH = hIsA ? p.A.center : p.B.center;
    const Box& box = hIsA ? p.B : p.A;
    F4 qBox = hIsA ? p.qB : p.qA;
    F3 rel = hIsA ? (p.vA - p.vB) : (p.vB - p.vA);
    float hullR = std::fabs(S.colShape[ih].w);
    float boxR = std::fabs(S.colShape[hIsA ? p.ib : p.ia].w);
    uint32_t first = S.colHullFirst[ih], nv = S.colHullCount[ih];
    auto candidate = [&](uint32_t v, HullCand& c) {
        F3 vw = pH + q_rotate(qH, S.hullVerts[first + v]);
        return hull_vertex_box(vw, v, box, qBox, rel, hullR, boxR, P, c);
    };
    HullCand best{};
    bool have = false;
    for (uint32_t v = 0; v < nv; v++) {
        HullCand c;
        if (!candidate(v, c)) continue;
        if (!have || c.sep < best.sep - 1e-8f || (std::fabs(c.sep - best.sep) <= 1e-8f && c.feature < best.feature)) {
            best = c;
            have = true;
        }
    }
    if (!have) { outM.header = U4{p.ba, p.bb, 0, 0}; return; }
    HullCand chosen[MAX_CONTACTS];
    int count = 1;
    chosen[0] = best;
    float band = 0.75f * P.collisionMargin;
    while (count < MAX_CONTACTS) {
        HullCand next{};
        bool haveNext = false;
        float bestSpread = -1.0f;
        for (uint32_t v = 0; v < nv; v++) {
            HullCand c;
            if (!candidate(v, c)) continue;
            if (c.sep > best.sep + band || dot(c.boxToHull, best.boxToHull) < 0.98f) continue;
            bool dup = false;
            float minSpread = FLT_MAX;
            for (int j = 0; j < count; j++) {
                if (c.feature == chosen[j].feature) { dup = true; break; }
                F3 dd = c.xHull - chosen[j].xHull;
                dd = dd - best.boxToHull * dot(best.boxToHull, dd);
                minSpread = fmin_(minSpread, dot(dd, dd));
            }
            if (dup) continue;
            if (!haveNext || minSpread > bestSpread + 1e-10f ||
                (std::fabs(minSpread - bestSpread) <= 1e-10f && c.feature < next.feature)) {
                next = c;
                bestSpread = minSpread;
                haveNext = true;
            }
        }
        if (!haveNext || bestSpread < MERGE_DIST_SQ) break;
        chosen[count++] = next;
    }
    NPContact contacts[MAX_CONTACTS];
    for (int i = 0; i < count; i++)
        contacts[i] = NPContact{hIsA ? chosen[i].xHull : chosen[i].xBox, hIsA ? chosen[i].xBox : chosen[i].xHull,
                                chosen[i].feature};
    emit_feature_manifold(S, p, outM, contacts, count, hIsA ? best.boxToHull : -best.boxToHull);
}

// 30_narrowphase.metal:547-745
static void narrow_capsule(const Solver& S, const NPair& p, ManifoldGPU& outM, uint32_t stA, uint32_t stB) {
    const Params& P = S.P;
    bool cIsA = stA == 3;
    uint32_t ic = cIsA ? p.ia : p.ib, io = cIsA ? p.ib : p.ia;
    F4 qC = cIsA ? p.qA : p.qB, qO = cIsA ? p.qB : p.qA;
    F3 pC = cIsA ? p.A.center : p.B.center, pO = cIsA ? p.B.center : p.A.center;
    F4 shC = S.colShape[ic], shO = S.colShape[io];
    float half_ = shC.x * 0.5f, rc = shC.y;
    F3 axC = q_rotate(qC, f3(0, 0, 1));
    F3 c0 = pC - axC * half_, c1 = pC + axC * half_;
    uint32_t other = cIsA ? stB : stA;
    F3 relCO = cIsA ? (p.vB - p.vA) : (p.vA - p.vB);
    NPContact hits[3];
    int nh = 0;
    F3 nCO = f3(0, 0, 1);
    if (other == 1) {
        float rs = shO.x * 0.5f;
        F3 q = closest_on_segment(pO, c0, c1);
        F3 dd = pO - q;
        float dist = length(dd);
        F3 nT = dist > 1e-6f ? dd / dist : f3(0, 0, 1);
        float dm = detect_margin(nT, relCO, P, shC.w, shO.w);
        if (dist <= rc + rs + dm) {
            nCO = nT;
            hits[0] = NPContact{q + nCO * rc, pO - nCO * rs, 0};
            nh = 1;
        }
    } else if (other == 3) {
        float halfO = shO.x * 0.5f, ro = shO.y;
        F3 axO = q_rotate(qO, f3(0, 0, 1));
        F3 o0 = pO - axO * halfO, o1 = pO + axO * halfO;
        F3 qa, qb;
        closest_seg_seg(c0, c1, o0, o1, qa, qb);
        F3 dd = qb - qa;
        float dist = length(dd);
        F3 nT = dist > 1e-6f ? dd / dist : f3(0, 0, 1);
        float dm = detect_margin(nT, relCO, P, shC.w, shO.w);
        if (dist <= rc + ro + dm) {
            nCO = nT;
            hits[0] = NPContact{qa + nCO * rc, qb - nCO * ro, 0};
            nh = 1;
        }
    } else {
        F4 qOc = q_conj(qO);
        F3 halfO = xyz(shO) * 0.5f;
        F3 nAccum = f3s(0);
        for (int seed = 0; seed < 3 && nh < 3; seed++) {
            float t = (float)seed * 0.5f;
            F3 q = c0 + (c1 - c0) * t;
            F3 bw = q;
            for (int it = 0; it < 5; it++) {
                F3 lb = clamp3(q_rotate(qOc, q - pO), -halfO, halfO);
                bw = q_rotate(qO, lb) + pO;
                q = closest_on_segment(bw, c0, c1);
            }
            F3 dd = bw - q;
            float dist = length(dd);
            F3 n;
            if (dist < 1e-6f) {
                F3 lb = q_rotate(qOc, q - pO);
                F3 pen = halfO - abs3(lb);
                int axis = min_axis(pen);
                F3 nl = f3s(0);
                setcomp(nl, axis, comp(lb, axis) >= 0.0f ? 1.0f : -1.0f);
                n = -q_rotate(qO, nl);
                bw = q - n * comp(pen, axis);
            } else {
                n = dd / dist;
                float dm = detect_margin(n, relCO, P, shC.w, shO.w);
                if (dist - rc > dm) continue;
            }
            bool dup = false;
            for (int h = 0; h < nh; h++)
                if (distance(hits[h].xA, q + n * rc) < 0.4f * rc + 0.05f) { dup = true; break; }
            if (dup) continue;
            hits[nh] = NPContact{q + n * rc, bw, (uint32_t)seed};
            nAccum = nAccum + n;
            nh++;
        }
        if (nh > 0) nCO = normalize(nAccum);
    }
    if (nh == 0) { outM.header = U4{p.ba, p.bb, 0, 0}; return; }
    NPContact contacts[3];
    for (int i = 0; i < nh; i++)
        contacts[i] = NPContact{cIsA ? hits[i].xA : hits[i].xB, cIsA ? hits[i].xB : hits[i].xA, hits[i].feature};
    emit_round_manifold(S, p, outM, contacts, nh, cIsA ? -nCO : nCO, 0.6f * (shC.y + 0.2f), true);
}

struct Torus { F3 center, axis, u, v; float R, r; };

// 30_narrowphase.metal:300-332
static Torus torus_frame(F3 pos, F4 q, float R, float r) {
    Torus t;
    t.center = pos;
    t.axis = q_rotate(q, f3(0, 0, 1));
    t.u = std::fabs(t.axis.x) > std::fabs(t.axis.z) ? f3(-t.axis.y, t.axis.x, 0.0f) : f3(0.0f, -t.axis.z, t.axis.y);
    t.u = normalize(t.u);
    t.v = cross(t.axis, t.u);
    t.R = R;
    t.r = r;
    return t;
}
static F3 torus_spine(const Torus& t, F3 p) {
    F3 d = p - t.center;
    d = d - t.axis * dot(t.axis, d);
    float l = length(d);
    return l < 1e-6f ? t.center + t.u * t.R : t.center + d / l * t.R;
}

// cos and sin of the spine sample angles float(i) / 32 * 2 * pi, correctly
// rounded at those float angles.
static const float kSpineCos[32] = {
    1.0f, 0.980785251f, 0.923879504f, 0.831469595f, 0.707106769f, 0.555570185f, 0.382683426f, 0.195090234f,
    -4.37113883e-08f, -0.195090324f, -0.382683516f, -0.555570364f, -0.707106769f, -0.831469655f, -0.923879623f,
    -0.98078531f, -1.0f, -0.980785251f, -0.923879504f, -0.831469536f, -0.70710665f, -0.555570006f, -0.382683128f,
    -0.195090383f, 1.19248806e-08f, 0.195090413f, 0.382683605f, 0.555570424f, 0.707107008f, 0.831469595f,
    0.923879564f, 0.98078531f};
static const float kSpineSin[32] = {
    0.0f, 0.195090324f, 0.382683456f, 0.555570245f, 0.707106769f, 0.831469655f, 0.923879504f, 0.98078531f,
    1.0f, 0.980785251f, 0.923879504f, 0.831469536f, 0.707106769f, 0.555570185f, 0.382683277f, 0.195090309f,
    -8.74227766e-08f, -0.195090488f, -0.382683426f, -0.555570304f, -0.707106888f, -0.831469774f, -0.923879683f,
    -0.980785251f, -1.0f, -0.980785251f, -0.923879445f, -0.831469476f, -0.707106531f, -0.555570304f,
    -0.382683426f, -0.195090234f};

// 30_narrowphase.metal:747-975
static void narrow_torus(const Solver& S, const NPair& p, ManifoldGPU& outM, uint32_t stA, uint32_t stB) {
    const Params& P = S.P;
    struct TorusHit { F3 xT, xO, n; float sep; uint32_t feature; };
    bool tIsA = stA == 2;
    uint32_t it = tIsA ? p.ia : p.ib, io = tIsA ? p.ib : p.ia;
    F4 qT = tIsA ? p.qA : p.qB, qO = tIsA ? p.qB : p.qA;
    F3 pT = tIsA ? p.A.center : p.B.center, pO = tIsA ? p.B.center : p.A.center;
    F4 shT = S.colShape[it], shO = S.colShape[io];
    Torus T = torus_frame(pT, qT, shT.x, shT.y);
    uint32_t other = tIsA ? stB : stA;
    float detectM = fmax_(P.collisionMargin, 0.8f * T.r);
    TorusHit hits[4];
    int nHits = 0;
    if (other == 1) {
        float rs = shO.x * 0.5f;
        F3 spine = torus_spine(T, pO);
        F3 dd = pO - spine;
        float dist = length(dd);
        if (dist <= T.r + rs + detectM) {
            F3 n = dist > 1e-6f ? dd / dist : f3(0, 0, 1);
            hits[0] = TorusHit{spine + n * T.r, pO - n * rs, -n, dist - T.r - rs, 0};
            nHits = 1;
        }
    } else {
        const int NSAMP = 32;
        bool isBox = other == 0, isCap = other == 3;
        Torus T2{};
        F4 qOc = q_conj(qO);
        F3 halfO = xyz(shO) * 0.5f;
        float otherR = 0.0f;
        F3 cs0 = f3s(0), cs1 = f3s(0);
        if (isCap) {
            float chalf = shO.x * 0.5f;
            F3 axO = q_rotate(qO, f3(0, 0, 1));
            cs0 = pO - axO * chalf;
            cs1 = pO + axO * chalf;
            otherR = shO.y;
        } else if (!isBox) {
            T2 = torus_frame(pO, qO, shO.x, shO.y);
            otherR = T2.r;
        }
        auto closest_other = [&](F3 q) {
            if (isBox) return q_rotate(qO, clamp3(q_rotate(qOc, q - pO), -halfO, halfO)) + pO;
            if (isCap) return closest_on_segment(q, cs0, cs1);
            return torus_spine(T2, q);
        };
        float dists[32];
        F3 closest[32];
        for (int i = 0; i < NSAMP; i++) {
            F3 q = T.center + (T.u * kSpineCos[i] + T.v * kSpineSin[i]) * T.R;
            F3 b = closest_other(q);
            closest[i] = b;
            dists[i] = distance(q, b);
        }
        bool used[32] = {};
        for (int pick = 0; pick < 4; pick++) {
            int best = -1;
            float bd = FLT_MAX;
            for (int i = 0; i < NSAMP; i++) {
                if (used[i]) continue;
                if (dists[i] < bd) { bd = dists[i]; best = i; }
            }
            if (best < 0) break;
            if (bd - T.r - otherR > detectM) break;
            for (int k = -3; k <= 3; k++) used[(best + k + NSAMP) % NSAMP] = true;
            F3 q = T.center + (T.u * kSpineCos[best] + T.v * kSpineSin[best]) * T.R;
            F3 b = closest[best];
            for (int it2 = 0; it2 < 2; it2++) {
                q = torus_spine(T, b);
                b = closest_other(q);
            }
            F3 dd = q - b;
            float dist = length(dd);
            F3 n;
            F3 xO_ = b;
            if (dist < 1e-6f) {
                if (isBox) {
                    F3 lb = q_rotate(qOc, q - pO);
                    F3 pen = halfO - abs3(lb);
                    int axis = min_axis(pen);
                    F3 nl = f3s(0);
                    setcomp(nl, axis, comp(lb, axis) >= 0.0f ? 1.0f : -1.0f);
                    n = q_rotate(qO, nl);
                    xO_ = q + n * comp(pen, axis);
                } else if (isCap) {
                    n = normalize(cross(T.axis, normalize(cs1 - cs0)) + f3(1e-4f, 0, 0));
                } else {
                    n = normalize(cross(T.axis, T2.axis) + f3(1e-4f, 0, 0));
                }
            } else {
                if (dist - T.r - otherR > detectM) continue;
                n = dd / dist;
            }
            hits[nHits] = TorusHit{q - n * T.r, xO_ + (isBox ? f3s(0) : n * otherR), n, dist - T.r - otherR,
                                   (uint32_t)best};
            nHits++;
        }
    }
    if (nHits == 0) { outM.header = U4{p.ba, p.bb, 0, 0}; return; }
    int deep = 0;
    float minSep = FLT_MAX;
    for (int h = 0; h < nHits; h++)
        if (hits[h].sep < minSep) { minSep = hits[h].sep; deep = h; }
    F3 nT = hits[deep].n;
    NPContact contacts[4];
    for (int i = 0; i < nHits; i++)
        contacts[i] = NPContact{tIsA ? hits[i].xT : hits[i].xO, tIsA ? hits[i].xO : hits[i].xT, hits[i].feature};
    emit_round_manifold(S, p, outM, contacts, nHits, tIsA ? nT : -nT, 1.1f * shT.x, false);
}

void Solver::narrow_one(uint32_t gid) {
    uint32_t ia = pairs[2 * gid], ib = pairs[2 * gid + 1];
    uint32_t ba = colOwner[ia], bb = colOwner[ib];
    F4 bodyPA = posLin[ba], bodyPB = posLin[bb];
    F4 qBodyA = posAng[ba], qBodyB = posAng[bb];
    F3 centerA = xyz(bodyPA) + q_rotate(qBodyA, xyz(colLocalPos[ia]));
    F3 centerB = xyz(bodyPB) + q_rotate(qBodyB, xyz(colLocalPos[ib]));
    F4 qA = q_mul(qBodyA, colLocalRot[ia]);
    F4 qB = q_mul(qBodyB, colLocalRot[ib]);
    F3 vA = xyz(velLin[ba]) + cross(xyz(velAng[ba]), centerA - xyz(bodyPA));
    F3 vB = xyz(velLin[bb]) + cross(xyz(velAng[bb]), centerB - xyz(bodyPB));
    F3 relVel = vB - vA;
    Box A, B;
    A.center = centerA; A.half = xyz(colShape[ia]) * 0.5f;
    A.ax[0] = q_rotate(qA, f3(1, 0, 0)); A.ax[1] = q_rotate(qA, f3(0, 1, 0)); A.ax[2] = q_rotate(qA, f3(0, 0, 1));
    B.center = centerB; B.half = xyz(colShape[ib]) * 0.5f;
    B.ax[0] = q_rotate(qB, f3(1, 0, 0)); B.ax[1] = q_rotate(qB, f3(0, 1, 0)); B.ax[2] = q_rotate(qB, f3(0, 0, 1));
    F3 delta = B.center - A.center;
    ManifoldGPU& outM = manifolds[gid];
    outM.colliderPair = U4{ia, ib, 0, 0};
    uint32_t stA = colShapeType[ia] & 0xFu, stB = colShapeType[ib] & 0xFu;
    bool sphA = stA == 1, sphB = stB == 1;
    if (stA >= 2 || stB >= 2) {
        NPair p{ia, ib, ba, bb, bodyPA, bodyPB, qBodyA, qBodyB, qA, qB, vA, vB, A, B};
        if (stA == 4 || stB == 4) narrow_hull(*this, p, outM, stA, stB);
        else if ((stA == 3 || stB == 3) && stA != 2 && stB != 2) narrow_capsule(*this, p, outM, stA, stB);
        else narrow_torus(*this, p, outM, stA, stB);
        return;
    }

    NPContact contacts[MAX_CONTACTS];
    int count = 0;
    F3 nrm;
    const float warm = P.alpha * P.gamma;
    if (sphA || sphB) {
        float rA = colShape[ia].x * 0.5f, rB = colShape[ib].x * 0.5f;
        if (sphA && sphB) {
            F3 d = A.center - B.center;
            float dist = length(d);
            F3 nT = dist > 1e-9f ? d / dist : f3(0, 0, 1);
            float dm = detect_margin(nT, vA - vB, P, rA, rB);
            if (dist > rA + rB + dm) { outM.header = U4{ba, bb, 0, 0}; return; }
            nrm = nT;
            contacts[0] = NPContact{A.center - nrm * rA, B.center + nrm * rB, 0};
            count = 1;
        } else {
            bool sIsA = sphA;
            float r = sIsA ? rA : rB;
            const Box& box = sIsA ? B : A;
            F4 qBox = sIsA ? qB : qA;
            F3 sc = sIsA ? A.center : B.center;
            F3 local = q_rotate(q_conj(qBox), sc - box.center);
            F3 h = box.half;
            F3 cl = clamp3(local, -h, h);
            F3 nLocal, qLocal;
            if (cl.x == local.x && cl.y == local.y && cl.z == local.z) {
                F3 pen = h - abs3(local);
                int axis = 0;
                if (pen.y < comp(pen, axis)) axis = 1;
                if (pen.z < comp(pen, axis)) axis = 2;
                F3 n = f3s(0);
                setcomp(n, axis, comp(local, axis) >= 0.0f ? 1.0f : -1.0f);
                nLocal = n;
                qLocal = local;
                setcomp(qLocal, axis, comp(n, axis) * comp(h, axis));
            } else {
                F3 d = local - cl;
                float dist = length(d);
                F3 nLT = d / fmax_(dist, 1e-9f);
                F3 nWT = q_rotate(qBox, nLT);
                F3 vS = sIsA ? vA : vB, vBx = sIsA ? vB : vA;
                float dm = detect_margin(nWT, vS - vBx, P, r, sIsA ? colShape[ib].w : colShape[ia].w);
                if (dist > r + dm) { outM.header = U4{ba, bb, 0, 0}; return; }
                nLocal = nLT;
                qLocal = cl;
            }
            F3 nW = q_rotate(qBox, nLocal);
            F3 qW = q_rotate(qBox, qLocal) + box.center;
            F3 xS = sc - nW * r;
            nrm = sIsA ? nW : -nW;
            contacts[0] = NPContact{sIsA ? xS : qW, sIsA ? qW : xS, 0};
            count = 1;
        }
        F3 t1, t2;
        orthonormal(nrm, t1, t2);
        float sf = combine_friction(colFrictionS[ia], colFrictionS[ib], P.frictionCombineMode);
        float df = combine_friction(colFrictionD[ia], colFrictionD[ib], P.frictionCombineMode);
        int prev = map_find(ia, ib);
        bool roundA = (colShapeType[ia] & 0x20u) != 0, roundB = (colShapeType[ib] & 0x20u) != 0;
        uint32_t flags = 1u | (roundA ? 2u : 0u) | (roundB ? 4u : 0u);
        outM.header = U4{ba, bb, (uint32_t)count, flags};
        outM.basisN = f4(nrm, df);
        outM.basisT1 = f4(t1, sf);
        F4 qAc = q_conj(qBodyA), qBc = q_conj(qBodyB);
        for (int i = 0; i < count; i++) {
            F3 rA_ = roundA ? contacts[i].xA - xyz(bodyPA) : q_rotate(qAc, contacts[i].xA - xyz(bodyPA));
            F3 rB_ = roundB ? contacts[i].xB - xyz(bodyPB) : q_rotate(qBc, contacts[i].xB - xyz(bodyPB));
            F3 lambda = f3s(0), penalty = f3s(0);
            float stick = 0.0f;
            if (prev >= 0) {
                const ManifoldGPU& pm = prevManifolds[prev];
                uint32_t pn = pm.header.z;
                float bestD = 0.5f * fmax_(rA, rB);
                int bestJ = -1;
                for (uint32_t j = 0; j < pn; j++) {
                    float dj = distance(xyz(pm.contacts[j].rA), rA_);
                    if (dj < bestD) { bestD = dj; bestJ = (int)j; }
                }
                if (bestJ >= 0) {
                    lambda = xyz(pm.contacts[bestJ].lambda);
                    penalty = xyz(pm.contacts[bestJ].penalty);
                    F3 t1o = xyz(pm.basisT1);
                    F3 t2o = cross(xyz(pm.basisN), t1o);
                    F3 lt = t1o * lambda.y + t2o * lambda.z;
                    lambda.y = dot(t1, lt);
                    lambda.z = dot(t2, lt);
                    bool partA = colShape[ia].w < 0.0f, partB = colShape[ib].w < 0.0f;
                    if ((partA || !roundA) && (partB || !roundB)) {
                        stick = pm.contacts[bestJ].rB.w;
                        if (stick != 0.0f) { rA_ = xyz(pm.contacts[bestJ].rA); rB_ = xyz(pm.contacts[bestJ].rB); }
                    }
                }
            }
            F3 xAw = roundA ? xyz(bodyPA) + rA_ : xform(xyz(bodyPA), qBodyA, rA_);
            F3 xBw = roundB ? xyz(bodyPB) + rB_ : xform(xyz(bodyPB), qBodyB, rB_);
            F3 d = xAw - xBw;
            F3 C0 = f3(dot(nrm, d) + P.collisionMargin, dot(t1, d), dot(t2, d));
            float sx, sy;
            spin_shift(spinVel[ba], spinVel[bb], xAw - xyz(bodyPA), xBw - xyz(bodyPB), t1, t2, P.dt, P.alpha, sx, sy);
            C0.y -= sx; C0.z -= sy;
            lambda *= warm;
            F3 lo = penalty_floor(*this, ba, bb);
            F3 hi = f3(PENALTY_MAX, PENALTY_MAX_T, PENALTY_MAX_T);
            penalty = clamp3(penalty * P.gamma, lo, hi);
            outM.contacts[i].rA = f4(rA_, bitsf(contacts[i].feature));
            outM.contacts[i].rB = f4(rB_, stick);
            outM.contacts[i].C0 = f4(C0, 0);
            outM.contacts[i].lambda = f4(lambda, 0);
            outM.contacts[i].penalty = f4(penalty, 0);
        }
        return;
    }

    // box - box SAT (30_narrowphase.metal:1138-1321)
    AxisBest bestFace{0, 0, 0, -FLT_MAX, f3s(0), false};
    AxisBest bestEdge{0, 0, 0, -FLT_MAX, f3s(0), false};
    float cap = spec_cap(colShape[ia].w, colShape[ib].w, P.collisionMargin);
    bool separated = false;
    for (int i = 0; i < 3 && !separated; i++)
        if (!test_axis(A, B, delta, A.ax[i], 0, i, -1, relVel, cap, P, bestFace)) separated = true;
    for (int i = 0; i < 3 && !separated; i++)
        if (!test_axis(A, B, delta, B.ax[i], 1, -1, i, relVel, cap, P, bestFace)) separated = true;
    for (int i = 0; i < 3 && !separated; i++)
        for (int j = 0; j < 3 && !separated; j++)
            if (!test_axis(A, B, delta, cross(A.ax[i], B.ax[j]), 2, i, j, relVel, cap, P, bestEdge)) separated = true;
    if (separated || !bestFace.valid) { outM.header = U4{ba, bb, 0, 0}; return; }
    AxisBest best = bestFace;
    if (bestEdge.valid && 0.95f * bestEdge.sep > bestFace.sep + 0.01f) best = bestEdge;
    F3 mids[MAX_CONTACTS];
    if (best.type == 2) {
        F3 a0, a1, b0, b1, xA, xB;
        support_edge(A, best.ia, best.n, a0, a1);
        support_edge(B, best.ib, -best.n, b0, b1);
        closest_seg_seg(a0, a1, b0, b1, xA, xB);
        uint32_t feature = (2u << 24) | ((uint32_t)(best.ia & 0xFF) << 8) | (uint32_t)(best.ib & 0xFF);
        add_contact(contacts, count, mids, xA, xB, feature);
        if (count == 0) add_contact(contacts, count, mids, support(A, best.n), support(B, -best.n), feature);
    } else {
        bool refIsA = best.type == 0;
        int refAxis = refIsA ? best.ia : best.ib;
        const Box& ref = refIsA ? A : B;
        const Box& inc = refIsA ? B : A;
        F3 refOut = refIsA ? best.n : -best.n;
        float signR = dot(refOut, ref.ax[refAxis]) >= 0.0f ? 1.0f : -1.0f;
        F3 refN = ref.ax[refAxis] * signR;
        F3 refC = ref.center + refN * box_half(ref, refAxis);
        F3 refU, refV; float refEU, refEV;
        face_axes(ref, refAxis, refU, refV, refEU, refEV);
        int incAxis = 0;
        float bestD = -FLT_MAX;
        for (int i = 0; i < 3; i++) {
            float d = std::fabs(dot(inc.ax[i], refN));
            if (d > bestD) { bestD = d; incAxis = i; }
        }
        float signI = dot(inc.ax[incAxis], refN) > 0.0f ? -1.0f : 1.0f;
        F3 incN = inc.ax[incAxis] * signI;
        F3 incC = inc.center + incN * box_half(inc, incAxis);
        F3 incU, incV; float incEU, incEV;
        face_axes(inc, incAxis, incU, incV, incEU, incEV);
        F3 p0[NP_MAX_POLY], p1[NP_MAX_POLY];
        p0[0] = incC + incU * incEU + incV * incEV;
        p0[1] = incC - incU * incEU + incV * incEV;
        p0[2] = incC - incU * incEU - incV * incEV;
        p0[3] = incC + incU * incEU - incV * incEV;
        int n = 4;
        n = clip_poly(p0, n, refU, dot(refU, refC) + refEU, p1);
        n = clip_poly(p1, n, -refU, dot(-refU, refC) + refEU, p0);
        n = clip_poly(p0, n, refV, dot(refV, refC) + refEV, p1);
        n = clip_poly(p1, n, -refV, dot(-refV, refC) + refEV, p0);
        uint32_t prefix = (refIsA ? 0u : 1u) << 24;
        prefix |= (uint32_t)(refAxis & 0xFF) << 16;
        prefix |= (uint32_t)(incAxis & 0xFF) << 8;
        float slop = PLANE_EPS + fmax_(0.0f, best.sep);
        for (int i = 0; i < n && count < MAX_CONTACTS; i++) {
            F3 pInc = p0[i];
            float d = dot(pInc - refC, refN);
            if (d > slop) continue;
            F3 pRef = pInc - refN * d;
            add_contact(contacts, count, mids, refIsA ? pRef : pInc, refIsA ? pInc : pRef, prefix | (uint32_t)(i & 0xFF));
        }
        if (count == 0) add_contact(contacts, count, mids, support(A, best.n), support(B, -best.n), prefix);
    }
    nrm = -best.n;
    F3 t1, t2;
    orthonormal(nrm, t1, t2);
    float sf = combine_friction(colFrictionS[ia], colFrictionS[ib], P.frictionCombineMode);
    float df = combine_friction(colFrictionD[ia], colFrictionD[ib], P.frictionCombineMode);
    int prev = map_find(ia, ib);
    outM.header = U4{ba, bb, (uint32_t)count, 1u};
    outM.basisN = f4(nrm, df);
    outM.basisT1 = f4(t1, sf);
    F4 qAc = q_conj(qBodyA), qBc = q_conj(qBodyB);
    for (int i = 0; i < count; i++) {
        F3 rA = q_rotate(qAc, contacts[i].xA - xyz(bodyPA));
        F3 rB = q_rotate(qBc, contacts[i].xB - xyz(bodyPB));
        F3 lambda = f3s(0), penalty = f3s(0);
        float stick = 0.0f;
        if (prev >= 0) {
            const ManifoldGPU& pm = prevManifolds[prev];
            for (uint32_t j = 0; j < pm.header.z; j++) {
                if (fbits(pm.contacts[j].rA.w) == contacts[i].feature) {
                    lambda = xyz(pm.contacts[j].lambda);
                    penalty = xyz(pm.contacts[j].penalty);
                    stick = pm.contacts[j].rB.w;
                    if (stick != 0.0f) { rA = xyz(pm.contacts[j].rA); rB = xyz(pm.contacts[j].rB); }
                    break;
                }
            }
        }
        F3 xAw = xform(xyz(bodyPA), qBodyA, rA);
        F3 xBw = xform(xyz(bodyPB), qBodyB, rB);
        F3 d = xAw - xBw;
        F3 C0 = f3(dot(nrm, d) + P.collisionMargin, dot(t1, d), dot(t2, d));
        float sx, sy;
        spin_shift(spinVel[ba], spinVel[bb], xAw - xyz(bodyPA), xBw - xyz(bodyPB), t1, t2, P.dt, P.alpha, sx, sy);
        C0.y -= sx; C0.z -= sy;
        lambda *= warm;
        penalty = clamp3(penalty * P.gamma, penalty_floor(*this, ba, bb), f3(PENALTY_MAX, PENALTY_MAX_T, PENALTY_MAX_T));
        outM.contacts[i].rA = f4(rA, bitsf(contacts[i].feature));
        outM.contacts[i].rB = f4(rB, stick);
        outM.contacts[i].C0 = f4(C0, 0);
        outM.contacts[i].lambda = f4(lambda, 0);
        outM.contacts[i].penalty = f4(penalty, 0);
    }
}

void Solver::narrowphase() {
    for (uint32_t g = 0; g < numPairs; g++) narrow_one(g);
}

// Persistence map rebuilt from this frame's manifolds, queried next frame
// (20_broadphase.metal:555-593).  Serial insertion in manifold order.
void Solver::map_rebuild() {
    std::fill(mapKeyA.begin(), mapKeyA.end(), 0u);
    for (uint32_t g = 0; g < numPairs; g++) {
        const ManifoldGPU& m = manifolds[g];
        if (m.header.z == 0) continue;
        uint32_t a = m.colliderPair.x, b = m.colliderPair.y;
        uint32_t h = pair_map_hash(a, b, P.mapCapacity);
        for (uint32_t probe = 0; probe < P.mapCapacity; probe++) {
            if (mapKeyA[h] == 0) { mapKeyA[h] = a + 1; mapKeyB[h] = b; mapVal[h] = g; break; }
            h = (h + 1) & (P.mapCapacity - 1u);
        }
    }
}

// ==========================================================================
// Warm start (40_solver.metal:546-722)
// ==========================================================================
static float twist_angle(F4 qAr, F4 qB, F3 axis) {
    F4 r = q_mul(q_inv(qAr), qB);
    if (r.w < 0.0f) r = -r;
    return 2.0f * atan2_series(dot(xyz(r), axis), r.w);
}

void Solver::warmstart_joints() {
    for (uint32_t si = 0; si < springs.size(); si++) {
        SpringGPU& sp = springs[si];
        if (sp.header.z == 0) continue;
        uint32_t a = sp.header.x, b = sp.header.y;
        F3 pA = xform(xyz(posLin[a]), posAng[a], xyz(sp.rA));
        F3 pB = xform(xyz(posLin[b]), posAng[b], xyz(sp.rB));
        sp.dual.z = 0.5f * fmax_(length(pA - pB) - sp.rB.w, 0.0f);
        float warm = P.alpha * P.gamma;
        if (P.rodDecayPow > 0.0f) {
            F3 d = pA - pB;
            F3 dPrev = d - (xyz(velLin[a]) - xyz(velLin[b])) * P.dt;
            float dl = length(d), dpl = length(dPrev);
            if (dl > 1e-7f && dpl > 1e-7f) {
                float ct = clampf_(dot(d / dl, dPrev / dpl), 0.0f, 1.0f);
                warm *= std::pow(ct, P.rodDecayPow);
            }
        }
        sp.dual.x *= warm;
        sp.dual.y = fmin_(clampf_(sp.dual.y * P.gamma, PENALTY_MIN, PENALTY_MAX), sp.rA.w);
    }
    for (uint32_t gid = 0; gid < joints.size(); gid++) {
        JointGPU& j = joints[gid];
        if (j.header.z != 0) continue;
        uint32_t a = j.header.x, b = j.header.y;
        F3 pA = a == WORLD_BODY ? xyz(j.rA) : xform(xyz(posLin[a]), posAng[a], xyz(j.rA));
        F3 pB = xform(xyz(posLin[b]), posAng[b], xyz(j.rB));
        F4 qA = a == WORLD_BODY ? f4(0, 0, 0, 1) : posAng[a];
        float torqueArm = j.C0Lin.w;
        j.C0Lin = f4(pA - pB, torqueArm);
        F3 c0a;
        F3 axis = xyz(j.hingeAxis);
        if (j.hingeAxis.w != 0.0f) {
            F3 aB = q_rotate(posAng[b], axis);
            F3 aA = q_rotate(q_mul(qA, j.restRel), axis);
            c0a = cross(aA, aB) * torqueArm;
            if (j.dynamics.x > 0.0f) {
                float twist = twist_angle(q_mul(qA, j.restRel), posAng[b], axis);
                F3 omegaA = a == WORLD_BODY ? f3s(0) : xyz(velAng[a]);
                float twistRate = dot(xyz(velAng[b]) - omegaA, aB);
                j.dynamics.y = twist + P.dt * twistRate;
            }
        } else {
            c0a = q_sub(q_mul(qA, j.restRel), posAng[b]) * torqueArm;
        }
        j.C0Ang = f4(c0a, j.C0Ang.w);
        if (j.motor.y > 0.0f) {
            j.motor.z = 0.0f;
            j.dynamics.z = 0.0f;
            uint32_t mode = j.header.w & MOTOR_MODE_MASK;
            if (mode == MOTOR_EXPLICIT || mode == MOTOR_VELOCITY) {
                F4 qAr = a == WORLD_BODY ? j.restRel : q_mul(posAng[a], j.restRel);
                float twist = twist_angle(qAr, posAng[b], axis);
                F3 axisW = q_rotate(posAng[b], axis);
                F3 omegaA = a == WORLD_BODY ? f3s(0) : xyz(velAng[a]);
                float twistRate = dot(xyz(velAng[b]) - omegaA, axisW);
                if (mode == MOTOR_VELOCITY)
                    j.dynamics.z = clampf_(j.limits.z * (j.motor.x - twistRate), -j.motor.y, j.motor.y);
                else
                    j.dynamics.z = clampf_(j.motor.w * (j.motor.x - twist) - j.limits.z * twistRate,
                                           -j.motor.y, j.motor.y);
            }
        }
        float warm = P.alpha * P.gamma;
        float stiffLin = j.rA.w, stiffAng = j.rB.w;
        j.lambdaLin.x *= warm; j.lambdaLin.y *= warm; j.lambdaLin.z *= warm;
        j.lambdaAng.x *= warm; j.lambdaAng.y *= warm; j.lambdaAng.z *= warm;
        F3 pl = clamp3(xyz(j.penaltyLin) * P.gamma, f3s(PENALTY_MIN), f3s(PENALTY_MAX));
        F3 pa = clamp3(xyz(j.penaltyAng) * P.gamma, f3s(PENALTY_MIN), f3s(PENALTY_MAX));
        pl = fmin3(pl, f3s(stiffLin));
        pa = fmin3(pa, f3s(stiffAng));
        j.penaltyLin = f4(pl, j.penaltyLin.w);
        j.penaltyAng = f4(pa, j.penaltyAng.w);
    }
}

void Solver::warmstart_bodies() {
    const float dt = P.dt;
    for (uint32_t gid = 0; gid < nb; gid++) {
        F4 pl = posLin[gid], pa = posAng[gid];
        float mass = pl.w;
        F3 vl = xyz(velLin[gid]), va = xyz(velAng[gid]);
        F3 inertial = xyz(pl) + vl * dt;
        float bodyGravity = P.gravity * gravityScale[gid];
        if (mass > 0.0f) inertial += f3(0, 0, bodyGravity) * (dt * dt);
        inertLin[gid] = f4(inertial, 0);
        inertAng[gid] = q_addw(pa, va * dt);
        F3 accel = (vl - xyz(prevVelLin[gid])) / dt;
        float gsign = P.gravity < 0.0f ? -1.0f : (P.gravity > 0.0f ? 1.0f : 0.0f);
        float w = clampf_(accel.z * gsign / std::fabs(P.gravity), 0.0f, 1.0f);
        if (!std::isfinite(w)) w = 0.0f;
        initLin[gid] = f4(xyz(pl), 0);
        initAng[gid] = pa;
        if (P.surfaceTruncationMode != 0u && shape[gid].w < 0.0f) ogcPrev[gid] = f4(xyz(pl), 0);
        if (mass > 0.0f) {
            F3 guess = xyz(pl) + vl * dt + f3(0, 0, bodyGravity) * (w * dt * dt);
            if (P.surfaceTruncationMode == 1u && shape[gid].w < 0.0f) {
                float d2 = bitsf(boundsBits[gid]);
                if (d2 < 1e37f) {
                    float bv = fmax_(0.45f * std::sqrt(d2), -0.2f * shape[gid].w);
                    F3 tot = guess - xyz(pl);
                    float t2 = dot(tot, tot);
                    if (t2 > bv * bv) guess = xyz(pl) + tot * (bv * rsqrt_(t2));
                }
            }
            posLin[gid] = f4(guess, mass);
            posAng[gid] = q_addw(pa, va * dt);
        }
    }
}

// ==========================================================================
// Adjacency (40_solver.metal:27-243): per body, sorted (kind<<28 | index).
// ==========================================================================
void Solver::adjacency() {
    std::vector<std::vector<uint32_t>> lists(nb);
    auto add = [&](uint32_t b, uint32_t entry) { if (body_dynamic(b)) lists[b].push_back(entry); };
    for (uint32_t g = 0; g < joints.size(); g++) {
        const JointGPU& j = joints[g];
        if (j.header.z != 0) continue;
        if (j.rA.w == 0.0f && j.rB.w == 0.0f && j.motor.y == 0.0f) continue;
        uint32_t e = (FK_JOINT << ADJ_KIND_SHIFT) | g;
        add(j.header.x, e); add(j.header.y, e);
    }
    for (uint32_t s = 0; s < springs.size(); s++) {
        uint32_t e = (FK_SPRING << ADJ_KIND_SHIFT) | s;
        add(springs[s].header.x, e); add(springs[s].header.y, e);
    }
    for (uint32_t m = 0; m < numPairs; m++) {
        if (manifolds[m].header.z == 0) continue;
        uint32_t e = (FK_MANIFOLD << ADJ_KIND_SHIFT) | m;
        add(manifolds[m].header.x, e); add(manifolds[m].header.y, e);
    }
    for (uint32_t t = 0; t < tets.size(); t++) {
        uint32_t e = (FK_TET << ADJ_KIND_SHIFT) | t;
        add(tets[t].ids.x, e); add(tets[t].ids.y, e); add(tets[t].ids.z, e); add(tets[t].ids.w, e);
    }
    for (uint32_t i = 0; i < numSoft; i++) {
        uint32_t e = (FK_SOFT << ADJ_KIND_SHIFT) | i;
        const uint32_t ids[4] = {soft[i].ids.x, soft[i].ids.y, soft[i].ids.z, soft[i].ids.w};
        for (uint32_t b : ids) add(b, e);
    }
    for (uint32_t i = 0; i < membranes.size(); i++) {
        uint32_t e = (FK_MEMBRANE << ADJ_KIND_SHIFT) | i;
        add(membranes[i].ids.x, e); add(membranes[i].ids.y, e); add(membranes[i].ids.z, e);
    }
    for (uint32_t i = 0; i < bends.size(); i++) {
        uint32_t e = (FK_BEND << ADJ_KIND_SHIFT) | i;
        add(bends[i].ids.x, e); add(bends[i].ids.y, e); add(bends[i].ids.z, e); add(bends[i].ids.w, e);
    }
    adjStart.assign(nb, 0); adjCount.assign(nb, 0); adjList.clear();
    for (uint32_t b = 0; b < nb; b++) {
        std::sort(lists[b].begin(), lists[b].end());
        adjStart[b] = (uint32_t)adjList.size();
        adjCount[b] = (uint32_t)lists[b].size();
        adjList.insert(adjList.end(), lists[b].begin(), lists[b].end());
    }
}

// ==========================================================================
// Dynamic coloring (40_solver.metal:250-540), rigid-only scenes.
// ==========================================================================
void Solver::neighbor_colors(uint32_t entry, uint32_t self, uint32_t myColor,
                             const std::vector<uint32_t>& colorsIn, uint32_t& maskLo,
                             uint32_t& maskHi, uint32_t& allLo, uint32_t& allHi,
                             bool& conflict) const {
    uint32_t kind = entry >> ADJ_KIND_SHIFT, idx = entry & ADJ_INDEX_MASK;
    uint32_t nbs[3];
    uint32_t n = 0;
    if (kind == FK_TET) {
        const U4& ids = tets[idx].ids;
        for (uint32_t v : {ids.x, ids.y, ids.z, ids.w}) if (v != self && n < 3) nbs[n++] = v;
    } else {
        uint32_t a, b;
        if (kind == FK_JOINT) { a = joints[idx].header.x; b = joints[idx].header.y; }
        else if (kind == FK_SPRING) { a = springs[idx].header.x; b = springs[idx].header.y; }
        else { a = manifolds[idx].header.x; b = manifolds[idx].header.y; }
        nbs[0] = a == self ? b : a;
        n = 1;
    }
    for (uint32_t k = 0; k < n; k++) {
        uint32_t nbb = nbs[k];
        if (nbb == WORLD_BODY || posLin[nbb].w <= 0.0f) continue;
        uint32_t nc_ = colorsIn[nbb];
        uint32_t lo = nc_ < 32 ? (1u << nc_) : 0u;
        uint32_t hi = (nc_ >= 32 && nc_ < 64) ? (1u << (nc_ - 32)) : 0u;
        allLo |= lo; allHi |= hi;
        if (nbb < self) { maskLo |= lo; maskHi |= hi; if (nc_ == myColor) conflict = true; }
    }
}

static inline uint32_t ctz32(uint32_t x) { return (uint32_t)__builtin_ctz(x); }

void Solver::dynamic_coloring() {
    const int passes = 20;
    uint32_t changed[passes] = {};
    std::vector<uint32_t>* src = &colorsA;
    std::vector<uint32_t>* dst = &colorsB;
    for (int pass = 0; pass < passes; pass++) {
        if (!(pass > 0 && changed[pass - 1] == 0u)) {
            for (uint32_t gid = 0; gid < nb; gid++) {
                if (posLin[gid].w <= 0.0f) { (*dst)[gid] = 0; continue; }
                uint32_t my = (*src)[gid];
                uint32_t mLo = 0, mHi = 0, aLo = 0, aHi = 0;
                bool conflict = false;
                for (uint32_t k = adjStart[gid]; k < adjStart[gid] + adjCount[gid]; k++)
                    neighbor_colors(adjList[k], gid, my, *src, mLo, mHi, aLo, aHi, conflict);
                if (conflict) {
                    uint32_t freeLo = ~mLo, nc_;
                    if (freeLo != 0) nc_ = ctz32(freeLo);
                    else { uint32_t freeHi = ~mHi; nc_ = freeHi != 0 ? 32 + ctz32(freeHi) : (MAX_COLORS - 1); }
                    (*dst)[gid] = std::min<uint32_t>(nc_, MAX_COLORS - 1);
                    changed[pass] |= 1u;
                } else {
                    uint32_t freeLo = ~aLo;
                    uint32_t best = freeLo != 0 ? ctz32(freeLo) : (~aHi != 0 ? 32 + ctz32(~aHi) : my);
                    (*dst)[gid] = best < my ? best : my;
                    if (best < my) changed[pass] |= 1u;
                }
            }
        }
        std::swap(src, dst);
    }
    std::vector<uint32_t>& fin = *src;
    if (changed[passes - 1] != 0u) {
        for (uint32_t self = 0; self < nb; self++) {
            if (posLin[self].w <= 0.0f) { fin[self] = 0; continue; }
            uint32_t mLo = 0, mHi = 0, aLo = 0, aHi = 0;
            bool conflict = false;
            for (uint32_t k = adjStart[self]; k < adjStart[self] + adjCount[self]; k++)
                neighbor_colors(adjList[k], self, fin[self], fin, mLo, mHi, aLo, aHi, conflict);
            uint32_t freeLo = ~mLo;
            if (freeLo != 0) fin[self] = ctz32(freeLo);
            else { uint32_t freeHi = ~mHi; fin[self] = freeHi != 0 ? 32 + ctz32(freeHi) : (MAX_COLORS - 1); }
        }
    }
    colorConflicts = 0;
    for (uint32_t gid = 0; gid < nb; gid++) {
        if (posLin[gid].w <= 0.0f) continue;
        uint32_t mLo = 0, mHi = 0, aLo = 0, aHi = 0;
        bool conflict = false;
        for (uint32_t k = adjStart[gid]; k < adjStart[gid] + adjCount[gid]; k++)
            neighbor_colors(adjList[k], gid, fin[gid], fin, mLo, mHi, aLo, aHi, conflict);
        if (conflict) colorConflicts++;
    }
    for (int c = 0; c < MAX_COLORS; c++) colorCounts[c] = 0;
    for (uint32_t gid = 0; gid < nb; gid++) if (posLin[gid].w > 0.0f) colorCounts[fin[gid]]++;
    uint32_t run = 0, used = 0;
    for (int c = 0; c < MAX_COLORS; c++) { colorStart[c] = run; run += colorCounts[c]; if (colorCounts[c]) used = c + 1; }
    colorStart[MAX_COLORS] = run;
    colorStart[MAX_COLORS + 1] = used;
    colorList.assign(run, 0);
    std::vector<uint32_t> cur(colorStart.begin(), colorStart.begin() + MAX_COLORS);
    for (uint32_t gid = 0; gid < nb; gid++) if (posLin[gid].w > 0.0f) colorList[cur[fin[gid]]++] = gid;
    if (src != &colorsA) colorsA = fin;
}

// ==========================================================================
// Primal (40_solver.metal:741-1684): force stamps + 8-lane split reduction.
// ==========================================================================
static M3 geom_stiff_ball_socket(int k, F3 v) {
    M3 m = m3_diag(f3s(-comp(v, k)));
    if (k == 0) { m.r0.x += v.x; m.r1.x += v.y; m.r2.x += v.z; }
    else if (k == 1) { m.r0.y += v.x; m.r1.y += v.y; m.r2.y += v.z; }
    else { m.r0.z += v.x; m.r1.z += v.y; m.r2.z += v.z; }
    return m;
}
static inline float wrap_pi(float x) {
    return x - 6.2831853f * std::floor((x + 3.14159265f) / 6.2831853f);
}

void Solver::stamp_joint(const JointGPU& j, uint32_t self, Accum& acc) const {
    uint32_t a = j.header.x, b = j.header.y;
    bool isA = self == a;
    float torqueArm = j.C0Lin.w;
    F3 penLin = xyz(j.penaltyLin);
    if (dot(penLin, penLin) > 0.0f) {
        F3 pA = a == WORLD_BODY ? xyz(j.rA) : xform(xyz(posLin[a]), posAng[a], xyz(j.rA));
        F3 pB = xform(xyz(posLin[b]), posAng[b], xyz(j.rB));
        F3 C = pA - pB;
        if (j.header.w & 1) C -= xyz(j.C0Lin) * P.alpha;
        F3 F = penLin * C + xyz(j.lambdaLin);
        float jsign = isA ? 1.0f : -1.0f;
        F3 rW = isA ? q_rotate(posAng[a], xyz(j.rA)) : q_rotate(posAng[b], xyz(j.rB));
        M3 jAng = m3_skew(-jsign * rW);
        M3 jAngT = m3_transpose(jAng);
        M3 K = m3_diag(penLin);
        M3 jAngTk = m3_mulm(jAngT, K);
        acc.lhsLin = m3_add(acc.lhsLin, K);
        acc.lhsAng = m3_add(acc.lhsAng, m3_mulm(jAngTk, jAng));
        acc.lhsCross = m3_add(acc.lhsCross, m3_scale(jAngTk, jsign));
        F3 r = jsign * rW;
        M3 H = m3_add(m3_add(m3_scale(geom_stiff_ball_socket(0, r), F.x),
                             m3_scale(geom_stiff_ball_socket(1, r), F.y)),
                      m3_scale(geom_stiff_ball_socket(2, r), F.z));
        acc.lhsAng = m3_add(acc.lhsAng, m3_diagonalize(H));
        acc.rhsLin += jsign * F;
        acc.rhsAng += m3_mul(jAngT, F);
    }
    F3 penAng = xyz(j.penaltyAng);
    if (dot(penAng, penAng) > 0.0f) {
        F4 qA = a == WORLD_BODY ? f4(0, 0, 0, 1) : posAng[a];
        F3 C = q_sub(q_mul(qA, j.restRel), posAng[b]) * torqueArm;
        float s = (isA ? 1.0f : -1.0f) * torqueArm;
        if (j.hingeAxis.w != 0.0f) {
            F3 axis = xyz(j.hingeAxis);
            F3 aB = q_rotate(posAng[b], axis);
            F3 aA = q_rotate(q_mul(qA, j.restRel), axis);
            C = cross(aA, aB) * torqueArm;
            if (j.header.w & 2) C -= xyz(j.C0Ang) * P.alpha;
            F3 F = penAng * C + xyz(j.lambdaAng);
            float alignment = dot(aA, aB);
            M3 J = isA ? m3_add(m3_outer(aA, aB), m3_scale(m3_identity(), -alignment))
                       : m3_add(m3_scale(m3_identity(), alignment), m3_scale(m3_outer(aB, aA), -1.0f));
            J = m3_scale(J, torqueArm);
            M3 JT = m3_transpose(J);
            M3 K = m3_diag(penAng);
            acc.lhsAng = m3_add(acc.lhsAng, m3_mulm(m3_mulm(JT, K), J));
            acc.rhsAng += m3_mul(JT, F);
            if (j.motor.y > 0.0f || j.limits.x < j.limits.y) {
                float twist = twist_angle(q_mul(qA, j.restRel), posAng[b], axis);
                if (j.dynamics.x > 0.0f) {
                    float Ca = wrap_pi(twist - j.dynamics.y);
                    float ka = j.dynamics.x / fmax_(P.dt * P.dt, 1e-12f);
                    float sm = (self == a) ? -1.0f : 1.0f;
                    acc.lhsAng = m3_add(acc.lhsAng, m3_scale(m3_outer(aB, aB), ka));
                    acc.rhsAng += aB * (ka * Ca * sm);
                }
                if (j.limits.x < j.limits.y) {
                    float over = fmax_(twist - j.limits.y, 0.0f) + fmin_(twist - j.limits.x, 0.0f);
                    if (over != 0.0f) {
                        float kL = 4.0e4f;
                        float FL = clampf_(kL * over, -3000.0f, 3000.0f);
                        float sm = (self == a) ? -1.0f : 1.0f;
                        acc.lhsAng = m3_add(acc.lhsAng, m3_scale(m3_outer(aB, aB), kL));
                        acc.rhsAng += aB * (FL * sm);
                    }
                }
                if (j.motor.y > 0.0f) {
                    float sm = (self == a) ? -1.0f : 1.0f;
                    F3 axW = aB;
                    uint32_t mode = j.header.w & MOTOR_MODE_MASK;
                    if (mode == MOTOR_EXPLICIT || mode == MOTOR_VELOCITY) {
                        acc.rhsAng += axW * (-j.dynamics.z * sm);
                    } else {
                        float Cm = wrap_pi(twist - j.motor.x);
                        F4 qA0 = a == WORLD_BODY ? f4(0, 0, 0, 1) : initAng[a];
                        float twist0 = twist_angle(q_mul(qA0, j.restRel), initAng[b], axis);
                        float dTwist = wrap_pi(twist - twist0);
                        float cD = j.limits.z / fmax_(P.dt, 1e-6f);
                        float raw = j.motor.w * Cm + cD * dTwist;
                        float effort = clampf_(raw, -j.motor.y, j.motor.y);
                        if (std::fabs(raw) < j.motor.y)
                            acc.lhsAng = m3_add(acc.lhsAng, m3_scale(m3_outer(axW, axW), j.motor.w + cD));
                        acc.rhsAng += axW * (effort * sm);
                    }
                }
            }
        } else {
            if (j.header.w & 2) C -= xyz(j.C0Ang) * P.alpha;
            F3 F = penAng * C + xyz(j.lambdaAng);
            acc.lhsAng = m3_add(acc.lhsAng, m3_diag(penAng * (s * s)));
            acc.rhsAng += F * s;
        }
    }
}

void Solver::stamp_spring(const SpringGPU& sp, uint32_t self, Accum& acc) const {
    uint32_t a = sp.header.x, b = sp.header.y;
    float stiffness = sp.rA.w, rest = sp.rB.w;
    F3 pA = xform(xyz(posLin[a]), posAng[a], xyz(sp.rA));
    F3 pB = xform(xyz(posLin[b]), posAng[b], xyz(sp.rB));
    F3 d = pA - pB;
    float dLen = length(d);
    if (dLen <= 1.0e-6f) return;
    F3 n = d / dLen;
    float f;
    if (sp.header.z != 0) {
        float C = dLen - rest - sp.dual.z * P.alpha;
        stiffness = sp.dual.y;
        f = stiffness * C + sp.dual.x;
        if (f <= 0.0f) return;
    } else {
        f = stiffness * (dLen - rest);
    }
    bool isA = self == a;
    F3 rW = isA ? q_rotate(posAng[a], xyz(sp.rA)) : q_rotate(posAng[b], xyz(sp.rB));
    F3 jLin = isA ? n : -n;
    F3 jAng = isA ? cross(rW, n) : -cross(rW, n);
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(jLin, jLin), stiffness));
    acc.lhsAng = m3_add(acc.lhsAng, m3_scale(m3_outer(jAng, jAng), stiffness));
    acc.lhsCross = m3_add(acc.lhsCross, m3_scale(m3_outer(jAng, jLin), stiffness));
    acc.rhsLin += jLin * f;
    acc.rhsAng += jAng * f;
    float ft = fmax_(f, 0.0f) / dLen;
    if (ft > 0.0f)
        acc.lhsLin = m3_add(acc.lhsLin, m3_add(m3_diag(f3s(ft)), m3_scale(m3_outer(n, n), -ft)));
}

void Solver::stamp_tet(const TetGPU& t, uint32_t self, Accum& acc) const {
    F3 x0 = xyz(posLin[t.ids.x]), x1 = xyz(posLin[t.ids.y]), x2 = xyz(posLin[t.ids.z]), x3 = xyz(posLin[t.ids.w]);
    float muV = t.r1.w, lamV = t.r2.w;
    float alphaT = 1.0f + muV / fmax_(lamV, 1e-9f);
    F3 d0 = x1 - x0, d1 = x2 - x0, d2 = x3 - x0;
    F3 m0 = xyz(t.r0), m1 = xyz(t.r1), m2 = xyz(t.r2);
    F3 f0 = d0 * m0.x + d1 * m1.x + d2 * m2.x;
    F3 f1 = d0 * m0.y + d1 * m1.y + d2 * m2.y;
    F3 f2 = d0 * m0.z + d1 * m1.z + d2 * m2.z;
    float J = dot(f0, cross(f1, f2));
    F3 j0 = cross(f1, f2), j1 = cross(f2, f0), j2 = cross(f0, f1);
    float s2 = lamV * (J - alphaT);
    F3 p0 = muV * f0 + s2 * j0;
    F3 p1 = muV * f1 + s2 * j1;
    F3 p2 = muV * f2 + s2 * j2;
    F3 w;
    if (self == t.ids.y) w = m0;
    else if (self == t.ids.z) w = m1;
    else if (self == t.ids.w) w = m2;
    else w = -f3(m0.x + m1.x + m2.x, m0.y + m1.y + m2.y, m0.z + m1.z + m2.z);
    F3 grad = p0 * w.x + p1 * w.y + p2 * w.z;
    F3 g = j0 * w.x + j1 * w.y + j2 * w.z;
    acc.rhsLin += grad;
    acc.lhsLin = m3_add(acc.lhsLin, m3_diag(f3s(muV * dot(w, w))));
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(g, g), lamV));
}

void Solver::stamp_manifold(const ManifoldGPU& m, uint32_t self, Accum& acc) const {
    uint32_t a = m.header.x, b = m.header.y, n = m.header.z;
    bool isA = self == a;
    bool sphA = (m.header.w & 2u) != 0, sphB = (m.header.w & 4u) != 0;
    F3 dqALin = xyz(posLin[a]) - xyz(initLin[a]);
    F3 dqAAng = q_sub(posAng[a], initAng[a]);
    F3 dqBLin = xyz(posLin[b]) - xyz(initLin[b]);
    F3 dqBAng = q_sub(posAng[b], initAng[b]);
    F3 nrm = xyz(m.basisN), t1 = xyz(m.basisT1), t2 = cross(nrm, t1);
    float dynF = m.basisN.w, statF = m.basisT1.w;
    for (uint32_t i = 0; i < n; i++) {
        const ContactGPU& c = m.contacts[i];
        F3 rAW = sphA ? xyz(c.rA) : q_rotate(posAng[a], xyz(c.rA));
        F3 rBW = sphB ? xyz(c.rB) : q_rotate(posAng[b], xyz(c.rB));
        F3 C = xyz(c.C0) * (1.0f - P.alpha);
        C += f3(dot(nrm, dqALin), dot(t1, dqALin), dot(t2, dqALin));
        C -= f3(dot(nrm, dqBLin), dot(t1, dqBLin), dot(t2, dqBLin));
        C += f3(dot(cross(rAW, nrm), dqAAng), dot(cross(rAW, t1), dqAAng), dot(cross(rAW, t2), dqAAng));
        C -= f3(dot(cross(rBW, nrm), dqBAng), dot(cross(rBW, t1), dqBAng), dot(cross(rBW, t2), dqBAng));
        F3 F = xyz(c.penalty) * C + xyz(c.lambda);
        F.x = fmin_(F.x, 0.0f);
        float bounds = std::fabs(F.x) * statF;
        float fs = std::sqrt(F.y * F.y + F.z * F.z);
        if (fs > bounds && fs > 0.0f) {
            float db = std::fabs(F.x) * dynF;
            float sc = db / fs;
            F.y *= sc; F.z *= sc;
        }
        float s = isA ? 1.0f : -1.0f;
        M3 jLin = M3{nrm * s, t1 * s, t2 * s};
        F3 rW = isA ? rAW : rBW;
        M3 jAng = M3{cross(rW, jLin.r0), cross(rW, jLin.r1), cross(rW, jLin.r2)};
        M3 K = m3_diag(xyz(c.penalty));
        M3 jLinT = m3_transpose(jLin), jAngT = m3_transpose(jAng);
        M3 jAngTk = m3_mulm(jAngT, K);
        acc.lhsLin = m3_add(acc.lhsLin, m3_mulm(m3_mulm(jLinT, K), jLin));
        acc.lhsAng = m3_add(acc.lhsAng, m3_mulm(jAngTk, jAng));
        acc.lhsCross = m3_add(acc.lhsCross, m3_mulm(jAngTk, jLin));
        acc.rhsLin += m3_mul(jLinT, F);
        acc.rhsAng += m3_mul(jAngT, F);
    }
}

void Solver::stamp_entry(uint32_t entry, uint32_t body, Accum& acc) const {
    uint32_t kind = entry >> ADJ_KIND_SHIFT, idx = entry & ADJ_INDEX_MASK;
    if (kind == FK_JOINT) stamp_joint(joints[idx], body, acc);
    else if (kind == FK_SPRING) stamp_spring(springs[idx], body, acc);
    else if (kind == FK_TET) stamp_tet(tets[idx], body, acc);
    else if (kind == FK_MANIFOLD) stamp_manifold(manifolds[idx], body, acc);
    else if (kind == FK_SOFT) stamp_soft(soft[idx], body, acc);
    else if (kind == FK_MEMBRANE) stamp_membrane(membranes[idx], body, acc);
    else if (kind == FK_BEND) stamp_bend(bends[idx], body, acc);
}

void Solver::primal_body(uint32_t body) {
    bool rigid = shape[body].w >= 0.0f;
    Accum lane[8];
    for (int l = 0; l < 8; l++) lane[l] = accum_zero();
    uint32_t as = adjStart[body], cnt = adjCount[body];
    for (uint32_t k = 0; k < cnt; k++) stamp_entry(adjList[as + k], body, lane[k & 7u]);
    // xor-butterfly over the 8 lanes: offsets 4, 2, 1 (40_solver.metal:1616-1630)
    for (int d = 4; d >= 1; d >>= 1) {
        Accum nx[8];
        for (int l = 0; l < 8; l++) {
            nx[l] = lane[l];
            nx[l].lhsLin = m3_add(lane[l].lhsLin, lane[l ^ d].lhsLin);
            nx[l].rhsLin = lane[l].rhsLin + lane[l ^ d].rhsLin;
            if (rigid) {
                nx[l].lhsAng = m3_add(lane[l].lhsAng, lane[l ^ d].lhsAng);
                nx[l].lhsCross = m3_add(lane[l].lhsCross, lane[l ^ d].lhsCross);
                nx[l].rhsAng = lane[l].rhsAng + lane[l ^ d].rhsAng;
            }
        }
        for (int l = 0; l < 8; l++) lane[l] = nx[l];
    }
    Accum acc = lane[0];
    F4 pl = posLin[body];
    float mass = pl.w;
    float dt2 = P.dt * P.dt;
    acc.lhsLin = m3_add(acc.lhsLin, m3_diag(f3s(mass / dt2)));
    acc.rhsLin += (xyz(pl) - xyz(inertLin[body])) * (mass / dt2);
    F3 dxLin = f3s(0), dxAng = f3s(0);
    if (rigid) {
        M3 inertia = m3_scale(world_inertia(posAng[body], xyz(props[body])), 1.0f / dt2);
        acc.lhsAng = m3_add(acc.lhsAng, inertia);
        acc.rhsAng += m3_mul(inertia, q_sub(posAng[body], inertAng[body]));
        solve6x6(acc.lhsLin, acc.lhsAng, acc.lhsCross, -acc.rhsLin, -acc.rhsAng, dxLin, dxAng);
        if (!finite3(dxLin) || !finite3(dxAng)) return;
        float ang2 = dot(dxAng, dxAng);
        const float maxAng = 0.5f;
        if (ang2 > maxAng * maxAng) dxAng *= maxAng * rsqrt_(ang2);
    } else {
        solve6x6(acc.lhsLin, m3_identity(), m3_zero(), -acc.rhsLin, f3s(0), dxLin, dxAng);
        if (!finite3(dxLin)) return;
    }
    float maxLin = 0.35f * std::fabs(shape[body].w);
    float lin2 = dot(dxLin, dxLin);
    if (lin2 > maxLin * maxLin) dxLin *= maxLin * rsqrt_(lin2);
    if (!rigid && P.numTris > 0u && P.surfaceTruncationMode == 1u) {
        // isotropic OGC bound (40_solver.metal:1361-1382)
        float d2 = bitsf(boundsBits[body]);
        if (d2 < 1e37f) {
            float bv = fmax_(0.45f * std::sqrt(d2), 0.2f * -shape[body].w);
            F3 x0 = xyz(ogcPrev[body]);
            F3 tot = (xyz(pl) + dxLin) - x0;
            float t2 = dot(tot, tot);
            if (t2 > bv * bv) {
                tot *= bv * rsqrt_(t2);
                dxLin = (x0 + tot) - xyz(pl);
#ifdef _OPENMP
#pragma omp atomic
#endif
                ogcPass++;
            }
        }
    }
    if (colorJacobi) {
        posNext[body] = f4(xyz(pl) + dxLin, mass);
        if (rigid) angNext[body] = q_addw(posAng[body], dxAng);
        return;
    }
    posLin[body] = f4(xyz(pl) + dxLin, mass);
    if (rigid) posAng[body] = q_addw(posAng[body], dxAng);
}

void Solver::primal_color(uint32_t c) {
    uint32_t s0 = colorStart[c], e0 = colorStart[c + 1];
    int n = (int)(e0 - s0);
    if (colorJacobi)
        for (uint32_t i = s0; i < e0; i++) { posNext[colorList[i]] = posLin[colorList[i]]; angNext[colorList[i]] = posAng[colorList[i]]; }
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1 && n > 256)
#endif
    for (int i = 0; i < n; i++) primal_body(colorList[s0 + (uint32_t)i]);
}

// ==========================================================================
// Dual (40_solver.metal:1729-1906)
// ==========================================================================
void Solver::dual_joint(uint32_t gid) {
    JointGPU& j = joints[gid];
    if (j.header.z != 0) return;
    uint32_t a = j.header.x, b = j.header.y;
    float torqueArm = j.C0Lin.w, stiffLin = j.rA.w, stiffAng = j.rB.w;
    F3 penLin = xyz(j.penaltyLin);
    if (dot(penLin, penLin) > 0.0f) {
        F3 pA = a == WORLD_BODY ? xyz(j.rA) : xform(xyz(posLin[a]), posAng[a], xyz(j.rA));
        F3 pB = xform(xyz(posLin[b]), posAng[b], xyz(j.rB));
        F3 C = pA - pB;
        if (j.header.w & 1) {
            C -= xyz(j.C0Lin) * P.alpha;
            F3 l = clamp3(penLin * C + xyz(j.lambdaLin), f3s(-P.lambdaMax), f3s(P.lambdaMax));
            j.lambdaLin = f4(l, j.lambdaLin.w);
        }
        float cap = fmin_(stiffLin, PENALTY_MAX);
        F3 p = fmin3(penLin + abs3(C) * P.betaLin, f3s(cap));
        j.penaltyLin = f4(p, j.penaltyLin.w);
    }
    F3 penAng = xyz(j.penaltyAng);
    if (dot(penAng, penAng) > 0.0f) {
        F4 qA = a == WORLD_BODY ? f4(0, 0, 0, 1) : posAng[a];
        F3 C;
        if (j.hingeAxis.w != 0.0f) {
            F3 axis = xyz(j.hingeAxis);
            F3 aB = q_rotate(posAng[b], axis);
            F3 aA = q_rotate(q_mul(qA, j.restRel), axis);
            C = cross(aA, aB) * torqueArm;
        } else {
            C = q_sub(q_mul(qA, j.restRel), posAng[b]) * torqueArm;
        }
        if (j.header.w & 2) {
            C -= xyz(j.C0Ang) * P.alpha;
            F3 l = clamp3(penAng * C + xyz(j.lambdaAng), f3s(-P.lambdaMax), f3s(P.lambdaMax));
            j.lambdaAng = f4(l, j.lambdaAng.w);
        }
        float cap = fmin_(stiffAng, PENALTY_MAX);
        F3 p = fmin3(penAng + abs3(C) * P.betaAng, f3s(cap));
        j.penaltyAng = f4(p, j.penaltyAng.w);
    }
    float fracture = j.C0Ang.w;
    F3 la = xyz(j.lambdaAng);
    float lin2 = (j.header.w & 8) ? dot(xyz(j.lambdaLin), xyz(j.lambdaLin)) : 0.0f;
    if ((j.header.w & 4) && dot(la, la) + lin2 > fracture * fracture) {
        j.penaltyLin = F4{}; j.penaltyAng = F4{}; j.lambdaLin = F4{}; j.lambdaAng = F4{};
        j.header.z = 1;
    }
}

void Solver::dual_spring(uint32_t si) {
    SpringGPU& sp = springs[si];
    if (sp.header.z == 0) return;
    uint32_t a = sp.header.x, b = sp.header.y;
    F3 pA = xform(xyz(posLin[a]), posAng[a], xyz(sp.rA));
    F3 pB = xform(xyz(posLin[b]), posAng[b], xyz(sp.rB));
    float C = length(pA - pB) - sp.rB.w - sp.dual.z * P.alpha;
    float mA = posLin[a].w, mB = posLin[b].w;
    float mMin = fmin_(mA > 0.0f ? mA : FLT_MAX, mB > 0.0f ? mB : FLT_MAX);
    float cap = fmin_(P.lambdaMax, fmax_(2.0f, 5.0e3f * mMin));
    sp.dual.x = clampf_(0.98f * sp.dual.x + sp.dual.y * C, 0.0f, cap);
    if (C > 0.0f) sp.dual.y = fmin_(sp.dual.y + C * P.betaLin, fmin_(sp.rA.w, PENALTY_MAX));
}

void Solver::dual_manifold(uint32_t gid) {
    ManifoldGPU& m = manifolds[gid];
    uint32_t n = m.header.z;
    if (n == 0) return;
    uint32_t a = m.header.x, b = m.header.y;
    bool sphA = (m.header.w & 2u) != 0, sphB = (m.header.w & 4u) != 0;
    F3 dqALin = xyz(posLin[a]) - xyz(initLin[a]);
    F3 dqAAng = q_sub(posAng[a], initAng[a]);
    F3 dqBLin = xyz(posLin[b]) - xyz(initLin[b]);
    F3 dqBAng = q_sub(posAng[b], initAng[b]);
    float mA = posLin[a].w, mB = posLin[b].w;
    float minMass = fmin_(mA > 0.0f ? mA : FLT_MAX, mB > 0.0f ? mB : FLT_MAX);
    float lamCap = fmin_(P.lambdaMax, fmax_(10.0f, 1.0e5f * minMass));
    F3 nrm = xyz(m.basisN), t1 = xyz(m.basisT1), t2 = cross(nrm, t1);
    float dynF = m.basisN.w, statF = m.basisT1.w;
    for (uint32_t i = 0; i < n; i++) {
        ContactGPU& c = m.contacts[i];
        F3 rAW = sphA ? xyz(c.rA) : q_rotate(posAng[a], xyz(c.rA));
        F3 rBW = sphB ? xyz(c.rB) : q_rotate(posAng[b], xyz(c.rB));
        F3 C = xyz(c.C0) * (1.0f - P.alpha);
        C += f3(dot(nrm, dqALin), dot(t1, dqALin), dot(t2, dqALin));
        C -= f3(dot(nrm, dqBLin), dot(t1, dqBLin), dot(t2, dqBLin));
        C += f3(dot(cross(rAW, nrm), dqAAng), dot(cross(rAW, t1), dqAAng), dot(cross(rAW, t2), dqAAng));
        C -= f3(dot(cross(rBW, nrm), dqBAng), dot(cross(rBW, t1), dqBAng), dot(cross(rBW, t2), dqBAng));
        F3 F = xyz(c.penalty) * C + xyz(c.lambda);
        F.x = fmin_(F.x, 0.0f);
        float bounds = std::fabs(F.x) * statF;
        float fs = std::sqrt(F.y * F.y + F.z * F.z);
        if (fs > bounds && fs > 0.0f) {
            float db = std::fabs(F.x) * dynF;
            float sc = db / fs;
            F.y *= sc; F.z *= sc;
        }
        F.x = fmax_(F.x, -lamCap);
        c.lambda = f4(F, 0);
        F3 pen = xyz(c.penalty);
        if (F.x < 0.0f) pen.x = fmin_(pen.x + P.betaLin * std::fabs(C.x), PENALTY_MAX);
        if (fs <= bounds) {
            pen.y = fmin_(pen.y + P.betaLin * std::fabs(C.y), PENALTY_MAX_T);
            pen.z = fmin_(pen.z + P.betaLin * std::fabs(C.z), PENALTY_MAX_T);
            c.rB.w = std::sqrt(C.y * C.y + C.z * C.z) < STICK_THRESH ? 1.0f : 0.0f;
        }
        c.penalty = f4(pen, 0);
    }
}

void Solver::dual_all() {
    for (uint32_t g = 0; g < joints.size(); g++) dual_joint(g);
    for (uint32_t s = 0; s < springs.size(); s++) dual_spring(s);
    for (uint32_t m = 0; m < numPairs; m++) if (manifolds[m].header.z != 0) dual_manifold(m);
    for (uint32_t i = 0; i < numSoft; i++) dual_soft(i);
}

// ==========================================================================
// Finalize (40_solver.metal:2108-2147)
// ==========================================================================
void Solver::finalize() {
    for (uint32_t gid = 0; gid < nb; gid++) {
        prevVelLin[gid] = velLin[gid];
        if (posLin[gid].w <= 0.0f) continue;
        F3 oldV = xyz(velLin[gid]);
        F3 v = (xyz(posLin[gid]) - xyz(initLin[gid])) / P.dt;
        float s2 = dot(v, v);
        if (s2 > P.maxSpeed * P.maxSpeed) v *= P.maxSpeed * rsqrt_(s2);
        if (shape[gid].w < 0.0f && P.particleDamping > 0.0f) {
            F3 ballistic = oldV + f3(0, 0, P.gravity * gravityScale[gid]) * P.dt;
            v = ballistic + (v - ballistic) / (1.0f + P.particleDamping * P.dt);
        }
        if (shape[gid].w >= 0.0f && P.rigidLinearDamping > 0.0f) v *= std::exp(-P.rigidLinearDamping * P.dt);
        F3 omega = q_sub(posAng[gid], initAng[gid]) / P.dt;
        if (shape[gid].w >= 0.0f && P.rigidAngularDamping > 0.0f) omega *= std::exp(-P.rigidAngularDamping * P.dt);
        velLin[gid] = f4(v, 0);
        velAng[gid] = f4(omega, 0);
    }
}

void Solver::advance_spinners() {
    const float TWO_PI = 6.28318530717958647692f;
    for (auto& rm : rateMotors) {
        float target = joints[rm.joint].motor.x + rm.rate * settings.dt;
        target -= TWO_PI * std::round(target / TWO_PI);
        joints[rm.joint].motor.x = target;
    }
    for (auto& sp : spinners) {
        F4 q = posAng[sp.body];
        float half = 0.5f * sp.omega * settings.dt;
        float sn = std::sin(half);
        F4 dq = f4(sp.axis[0] * sn, sp.axis[1] * sn, sp.axis[2] * sn, std::cos(half));
        F4 nq = q_mul(dq, q);
        posAng[sp.body] = nq / std::sqrt(dot4(nq, nq));
    }
}

float Solver::max_constraint_error() const {
    float err = 0.0f;
    for (const JointGPU& j : joints) {
        if (!(j.header.z == 0 && (j.rA.w > 0.0f || j.rB.w > 0.0f))) continue;
        uint32_t a = j.header.x, b = j.header.y;
        F3 pA = a == WORLD_BODY ? xyz(j.rA) : xform(xyz(posLin[a]), posAng[a], xyz(j.rA));
        F3 pB = xform(xyz(posLin[b]), posAng[b], xyz(j.rB));
        err = fmax_(err, length(pA - pB));
    }
    // the frame's manifolds were swapped into prevManifolds at the end of the
    // step; diagnostics read them there (GPUSolver.swift:4846-4853)
    for (uint32_t g = 0; g < numPairs; g++) {
        const ManifoldGPU& m = prevManifolds[g];
        uint32_t a = m.header.x, b = m.header.y;
        bool sphA = (m.header.w & 2u) != 0, sphB = (m.header.w & 4u) != 0;
        for (uint32_t i = 0; i < m.header.z; i++) {
            F3 xA = sphA ? xyz(posLin[a]) + xyz(m.contacts[i].rA) : xform(xyz(posLin[a]), posAng[a], xyz(m.contacts[i].rA));
            F3 xB = sphB ? xyz(posLin[b]) + xyz(m.contacts[i].rB) : xform(xyz(posLin[b]), posAng[b], xyz(m.contacts[i].rB));
            float pen = dot(xyz(m.basisN), xA - xB) + P.collisionMargin;
            err = fmax_(err, fmax_(0.0f, -pen));
        }
    }
    return err;
}

// ==========================================================================
// AL residual r = ||grad of the AL objective||_2 over every dynamic DOF.  The
// reference defines only diag_error (40_solver.metal:2189-2229); the residual
// is the right-hand side that primal_body assembles (the stamps of
// 40_solver.metal:741-1359 plus the inertial term M/dt^2 (x - x~)), for
// particles over 3 DOFs and for rigid bodies over 6 (angular part with the
// world inertia / dt^2 times q_sub(q, q~)).  Per body the squared norm is a
// float, the total a double sum.
// ==========================================================================
float Solver::body_residual_sq(uint32_t body) const {
    bool rigid = shape[body].w >= 0.0f;
    Accum lane[8];
    for (int l = 0; l < 8; l++) lane[l] = accum_zero();
    uint32_t as = adjStart[body], cnt = adjCount[body];
    for (uint32_t k = 0; k < cnt; k++) stamp_entry(adjList[as + k], body, lane[k & 7u]);
    for (int d = 4; d >= 1; d >>= 1) {
        F3 nl[8], na[8];
        for (int l = 0; l < 8; l++) {
            nl[l] = lane[l].rhsLin + lane[l ^ d].rhsLin;
            na[l] = lane[l].rhsAng + lane[l ^ d].rhsAng;
        }
        for (int l = 0; l < 8; l++) { lane[l].rhsLin = nl[l]; lane[l].rhsAng = na[l]; }
    }
    F4 pl = posLin[body];
    float dt2 = P.dt * P.dt;
    F3 rl = lane[0].rhsLin + (xyz(pl) - xyz(inertLin[body])) * (pl.w / dt2);
    if (!rigid) return dot(rl, rl);
    F4 q = posAng[body];
    M3 inertia = m3_scale(world_inertia(q, xyz(props[body])), 1.0f / dt2);
    F3 ra = lane[0].rhsAng + m3_mul(inertia, q_sub(q, inertAng[body]));
    return dot(rl, rl) + dot(ra, ra);
}

double Solver::residual() const {
    uint32_t colorBound = dynamicColoring ? (uint32_t)MAX_COLORS : staticUsedColors;
    uint32_t n = colorStart[colorBound];
    std::vector<float> per(n);
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1 && n > 256)
#endif
    for (int i = 0; i < (int)n; i++) per[i] = body_residual_sq(colorList[i]);
    double s = 0.0;
    for (uint32_t i = 0; i < n; i++) s += (double)per[i];
    return std::sqrt(s);
}

// ==========================================================================
// One frame (GPUSolver.swift:3138-4375)
// ==========================================================================
void Solver::step() {
    sync_params();
    std::fill(boundsBits.begin(), boundsBits.end(), 0x7F7F7F7Fu);
    ogcExceeded = 0;
    ogcPass = 0;
    colorConflicts = 0;
    const bool planar = P.surfaceTruncationMode == 2u && numTris > 0;
    dat = DatCounters{};
    softRaw = 0;
    numSoft = 0;
    hook(ST_BROADPHASE, 0, 0);
    broadphase();
    hook(ST_BROADPHASE, 0, 1);
    hook(ST_NARROWPHASE, 0, 0);
    narrowphase();
    hook(ST_NARROWPHASE, 0, 1);
    hook(ST_MAP, 0, 0);
    map_rebuild();
    hook(ST_MAP, 0, 1);
    if (planar) {
        elem_grid();
        dat_build_pairs();                     // step-start pose
        rt_emit();
    } else if (ogc) {
        ogc_detect();
    }
    hook(ST_WARM_JOINTS, 0, 0);
    warmstart_joints();
    hook(ST_WARM_JOINTS, 0, 1);
    hook(ST_WARM_BODIES, 0, 0);
    warmstart_bodies();
    hook(ST_WARM_BODIES, 0, 1);
    if (planar) {
        dat_reduce(0xFFFFFFFFu);               // predictor pass
        dat_apply_particles();
        elem_grid();                           // accepted predictor pose
        dat_build_pairs();
        dat_emit_contacts();
        soft_map_rebuild();
        for (uint32_t v : particleIdx) ogcPrev[v] = f4(xyz(posLin[v]), 0.0f);
    }
    hook(ST_ADJACENCY, 0, 0);
    adjacency();
    hook(ST_ADJACENCY, 0, 1);
    if (dynamicColoring) {
        hook(ST_COLORING, 0, 0);
        dynamic_coloring();
        hook(ST_COLORING, 0, 1);
    }
    uint32_t colorBound = dynamicColoring ? (uint32_t)MAX_COLORS : staticUsedColors;
    if (traceEnabled) {
        trace.assign(2 + P.iterations, 0.0);
        trace[0] = trace[1] = residual();
    }
    for (uint32_t it = 0; it < P.iterations; it++) {
        ogcPass = 0;
        for (uint32_t c = 0; c < colorBound; c++) {
            hook(ST_PRIMAL, (int)c, 0);
            primal_color(c);
            hook(ST_PRIMAL, (int)c, 1);
            if (planar) {
                dat_reduce(c);
                dat_apply_color(c);
            } else if (ogc) {
                publish_color(c);
            }
        }
        hook(ST_DUAL, (int)it, 0);
        dual_all();
        hook(ST_DUAL, (int)it, 1);
        // mid-solve bound refresh when more than 1% of the surface vertices
        // were bound-limited (ogc_refresh_args, 25_cloth.metal:857-870)
        if (ogc && it + 1 < P.iterations && ogcPass * 100u > P.numParticles) ogc_refresh();
        ogcExceeded = ogcPass;
        if (traceEnabled) trace[2 + it] = residual();
    }
    if (planar) dat_restore_failed_surface();
    hook(ST_FINALIZE, 0, 0);
    finalize();
    hook(ST_FINALIZE, 0, 1);
    if (numTris > 0 && clothViscosity > 0.0f) smooth_particle_velocities();
    advance_spinners();
    frameIndex++;
    // the manifolds written this frame become next frame's warm-start source
    std::swap(manifolds, prevManifolds);
    if (cloth || ogc) std::swap(soft, prevSoft);
    if (ogc) { std::swap(vtTrack, vtTrackPrev); std::swap(eeTrack, eeTrackPrev); }
    if (pairCandidates > maxPairs && failure == AVBD_FAIL_NONE) {
        failure = AVBD_FAIL_RIGID_PAIR_CAPACITY;
        error = "rigid pair capacity exceeded";
    }
    if (ogc && failure == AVBD_FAIL_NONE && dat.softCandidates > maxSoft) {
        failure = AVBD_FAIL_SOFT_CONTACT_CAPACITY;
        error = "soft contact capacity exceeded";
    }
    if (planar && failure == AVBD_FAIL_NONE) {
        if (dat.softCandidates > maxSoft) { failure = AVBD_FAIL_SOFT_CONTACT_CAPACITY; error = "soft contact capacity exceeded"; }
        else if (dat.pairsPeak > maxDatPairs) { failure = AVBD_FAIL_PLANAR_DAT_PAIR_CAPACITY; error = "Planar-DAT pair capacity exceeded"; }
        else if (dat.gridOverflow > 0) { failure = AVBD_FAIL_PLANAR_DAT_GRID_SPAN; error = "Planar-DAT element grid span exceeded"; }
        else if (dat.invalidAnchor > 0) { failure = AVBD_FAIL_PLANAR_DAT_INVALID_ANCHOR; error = "Planar-DAT invalid anchor"; }
    }
    if (colorConflicts > 0 && failure == AVBD_FAIL_NONE) {
        failure = AVBD_FAIL_UNRESOLVED_COLORING;
        error = "unresolved dynamic coloring";
    }
}

}  // namespace oracle

// ==========================================================================
// C entry points used by the tests (ctypes) and bench.py's cpu_baseline.
// ==========================================================================
using oracle::Solver;
extern "C" {

int oracle_create(const avbd_scene_desc* scene, void** out) {
    if (!out) return AVBD_ERR_INVALID_ARGUMENT;
    Solver* s = new Solver();
    int rc = s->create(scene);
    if (rc != AVBD_OK) {
        std::fprintf(stderr, "oracle_create: %s\n", s->error.c_str());
        delete s;
        *out = nullptr;
        return rc;
    }
    *out = s;
    return AVBD_OK;
}
void oracle_destroy(void* h) { delete static_cast<Solver*>(h); }
int oracle_set_threads(void* h, int n) { static_cast<Solver*>(h)->threads = n < 1 ? 1 : n; return AVBD_OK; }
int oracle_set_settings(void* h, const avbd_settings* st) { static_cast<Solver*>(h)->settings = *st; return AVBD_OK; }
int oracle_set_capacity_for_testing(void* h, int which, uint32_t value) {
    Solver* s = static_cast<Solver*>(h);
    if (which == AVBD_CAPACITY_SOFT_CONTACTS) s->maxSoft = std::min<uint32_t>(value, (uint32_t)s->soft.size());
    else if (which == AVBD_CAPACITY_PLANAR_DAT_PAIRS) s->maxDatPairs = std::min(value, s->maxDatPairs);
    else return AVBD_ERR_INVALID_ARGUMENT;
    return AVBD_OK;
}
int oracle_step(void* h, uint32_t frames) {
    Solver* s = static_cast<Solver*>(h);
    for (uint32_t f = 0; f < frames; f++) {
        if (s->failure != AVBD_FAIL_NONE) return AVBD_ERR_RUNTIME_FAILURE;
        s->step();
    }
    return s->failure != AVBD_FAIL_NONE ? AVBD_ERR_RUNTIME_FAILURE : AVBD_OK;
}
int oracle_runtime_failure(void* h, int* kind) { *kind = static_cast<Solver*>(h)->failure; return AVBD_OK; }
int oracle_get_positions(void* h, uint32_t n, float* pos, float* rot) {
    Solver* s = static_cast<Solver*>(h);
    if (n > s->nb) return AVBD_ERR_INVALID_ARGUMENT;
    if (pos) std::memcpy(pos, s->posLin.data(), n * 16);
    if (rot) std::memcpy(rot, s->posAng.data(), n * 16);
    return AVBD_OK;
}
int oracle_get_body_states(void* h, uint32_t n, avbd_body_state* out) {
    Solver* s = static_cast<Solver*>(h);
    if (n > s->nb) return AVBD_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < n; i++) {
        avbd_body_state& o = out[i];
        o.position[0] = s->posLin[i].x; o.position[1] = s->posLin[i].y; o.position[2] = s->posLin[i].z;
        o.rotation[0] = s->posAng[i].x; o.rotation[1] = s->posAng[i].y; o.rotation[2] = s->posAng[i].z; o.rotation[3] = s->posAng[i].w;
        o.velocity[0] = s->velLin[i].x; o.velocity[1] = s->velLin[i].y; o.velocity[2] = s->velLin[i].z;
        o.angular_velocity[0] = s->velAng[i].x; o.angular_velocity[1] = s->velAng[i].y; o.angular_velocity[2] = s->velAng[i].z;
    }
    return AVBD_OK;
}
int oracle_set_motor_targets(void* h, const uint32_t* ids, uint32_t n, const float* targets) {
    Solver* s = static_cast<Solver*>(h);
    for (uint32_t i = 0; i < n; i++) {
        if (ids[i] >= s->joints.size()) return AVBD_ERR_INVALID_ARGUMENT;
        oracle::JointGPU& j = s->joints[ids[i]];
        if ((j.header.w & oracle::MOTOR_MODE_MASK) == 0) continue;
        j.motor.x = targets[i];
    }
    return AVBD_OK;
}
// GPUSolver.swift:2481-2494, :2534-2551, :2564-2578
int oracle_set_joint_world_anchors(void* h, const uint32_t* ids, uint32_t n, const float* xyz) {
    Solver* s = static_cast<Solver*>(h);
    for (uint32_t i = 0; i < n; i++) {
        if (ids[i] >= s->joints.size()) return AVBD_ERR_INVALID_ARGUMENT;
        oracle::JointGPU& j = s->joints[ids[i]];
        j.rA.x = xyz[3 * i]; j.rA.y = xyz[3 * i + 1]; j.rA.z = xyz[3 * i + 2];
    }
    return AVBD_OK;
}
int oracle_set_motor_velocities(void* h, const uint32_t* ids, uint32_t n, const float* v) {
    Solver* s = static_cast<Solver*>(h);
    for (uint32_t i = 0; i < n; i++) {
        if (ids[i] >= s->joints.size()) return AVBD_ERR_INVALID_ARGUMENT;
        s->joints[ids[i]].motor.x = v[i];
    }
    return AVBD_OK;
}
int oracle_set_motor_torques(void* h, const uint32_t* ids, uint32_t n, const float* t) {
    Solver* s = static_cast<Solver*>(h);
    for (uint32_t i = 0; i < n; i++) {
        if (ids[i] >= s->joints.size()) return AVBD_ERR_INVALID_ARGUMENT;
        s->joints[ids[i]].motor.y = t[i];
    }
    return AVBD_OK;
}
// GPUSolver.swift:2606-2637
int oracle_get_motor_states(void* h, const uint32_t* ids, uint32_t n, float* angles, float* velocities) {
    using namespace oracle;
    Solver* s = static_cast<Solver*>(h);
    for (uint32_t i = 0; i < n; i++) {
        if (ids[i] >= s->joints.size()) return AVBD_ERR_INVALID_ARGUMENT;
        const JointGPU& j = s->joints[ids[i]];
        uint32_t a = j.header.x, b = j.header.y;
        F4 qB = s->posAng[b];
        F4 qA = a == 0xFFFFFFFFu ? F4{0, 0, 0, 1} : s->posAng[a];
        F4 r = q_mul(q_inv(q_mul(qA, j.restRel)), qB);
        if (r.w < 0.0f) r = F4{-r.x, -r.y, -r.z, -r.w};
        F3 axis = xyz(j.hingeAxis);
        angles[i] = 2.0f * atan2_series(dot(xyz(r), axis), r.w);
        F3 wB = xyz(s->velAng[b]);
        F3 wA = a == 0xFFFFFFFFu ? f3s(0) : xyz(s->velAng[a]);
        velocities[i] = dot(wB - wA, q_rotate(qB, axis));
    }
    return AVBD_OK;
}
float oracle_atan2(float y, float x) { return oracle::atan2_series(y, x); }
int oracle_set_residual_trace(void* h, int enabled) { static_cast<Solver*>(h)->traceEnabled = enabled != 0; return AVBD_OK; }
int oracle_get_residual_trace(void* h, double* out, uint32_t n) {
    Solver* s = static_cast<Solver*>(h);
    for (uint32_t i = 0; i < n; i++) out[i] = i < s->trace.size() ? s->trace[i] : 0.0;
    return AVBD_OK;
}
int oracle_residual(void* h, double* out) { *out = static_cast<Solver*>(h)->residual(); return AVBD_OK; }
int oracle_max_constraint_error(void* h, float* out) { *out = static_cast<Solver*>(h)->max_constraint_error(); return AVBD_OK; }
int oracle_get_counters(void* h, avbd_counters* out) {
    Solver* s = static_cast<Solver*>(h);
    std::memset(out, 0, sizeof(*out));
    out->frame = s->frameIndex;
    out->num_pairs = s->numPairs;
    out->pair_candidates = s->pairCandidates;
    out->color_conflicts = s->colorConflicts;
    out->ogc_exceeded = s->ogcExceeded;
    out->used_colors = s->dynamicColoring ? s->colorStart[64 + 1] : s->staticUsedColors;
    for (int c = 0; c < 64; c++) out->color_counts[c] = s->colorCounts[c];
    out->num_soft = s->numSoft;
    out->soft_candidates = s->dat.softCandidates;
    out->dat_pairs = s->dat.pairsPeak;
    out->dat_vt_pairs = s->dat.vtPeak;
    out->dat_ee_pairs = s->dat.eePeak;
    out->dat_grid_overflows = s->dat.gridOverflow;
    out->dat_invalid_anchors = s->dat.invalidAnchor;
    out->dat_truncations = s->dat.truncations;
    out->dat_vt_degenerate = s->dat.vtDegenerate;
    out->dat_ee_degenerate = s->dat.eeDegenerate;
    out->dat_nonfinite = s->dat.nonfinite;
    out->dat_tet_degenerate = s->dat.tetDegenerate;
    if (s->ogc) {
        out->soft_rt = s->numSoftRT;
        out->soft_vt = s->numSoftVT;
        out->soft_ee = s->numSoftEE;
    }
    return AVBD_OK;
}
static const void* oracle_buffer(Solver* s, int which, size_t& bytes) {
    switch (which) {
    case AVBD_BUF_POS_LIN: bytes = s->posLin.size() * 16; return s->posLin.data();
    case AVBD_BUF_POS_ANG: bytes = s->posAng.size() * 16; return s->posAng.data();
    case AVBD_BUF_VEL_LIN: bytes = s->velLin.size() * 16; return s->velLin.data();
    case AVBD_BUF_VEL_ANG: bytes = s->velAng.size() * 16; return s->velAng.data();
    case AVBD_BUF_PAIRS: bytes = (size_t)s->numPairs * 8; return s->pairs.data();
    // manifolds were swapped at the end of the frame: the last frame's are in prevManifolds
    case AVBD_BUF_MANIFOLDS: bytes = (size_t)s->numPairs * sizeof(oracle::ManifoldGPU); return s->prevManifolds.data();
    case AVBD_BUF_ADJ_START: bytes = s->adjStart.size() * 4; return s->adjStart.data();
    case AVBD_BUF_ADJ_COUNT: bytes = s->adjCount.size() * 4; return s->adjCount.data();
    case AVBD_BUF_ADJ_LIST: bytes = s->adjList.size() * 4; return s->adjList.data();
    case AVBD_BUF_COLORS: bytes = s->colorsA.size() * 4; return s->colorsA.data();
    case AVBD_BUF_COLOR_START: bytes = s->colorStart.size() * 4; return s->colorStart.data();
    case AVBD_BUF_COLOR_LIST: bytes = s->colorList.size() * 4; return s->colorList.data();
    case AVBD_BUF_CELL_START: bytes = s->cellStart.size() * 4; return s->cellStart.data();
    case AVBD_BUF_CELL_COUNT: bytes = s->cellCount.size() * 4; return s->cellCount.data();
    case AVBD_BUF_CELL_BODIES: bytes = (size_t)s->P.numHashed * 4; return s->cellBodies.data();
    case AVBD_BUF_MAP_KEY_A: bytes = s->mapKeyA.size() * 4; return s->mapKeyA.data();
    case AVBD_BUF_MAP_KEY_B: bytes = s->mapKeyB.size() * 4; return s->mapKeyB.data();
    case AVBD_BUF_MAP_VAL: bytes = s->mapVal.size() * 4; return s->mapVal.data();
    case AVBD_BUF_JOINTS: bytes = s->joints.size() * sizeof(oracle::JointGPU); return s->joints.data();
    case AVBD_BUF_SPRINGS: bytes = s->springs.size() * sizeof(oracle::SpringGPU); return s->springs.data();
    case AVBD_BUF_TETS: bytes = s->tets.size() * sizeof(oracle::TetGPU); return s->tets.data();
    case AVBD_BUF_INIT_LIN: bytes = s->initLin.size() * 16; return s->initLin.data();
    case AVBD_BUF_INERT_LIN: bytes = s->inertLin.size() * 16; return s->inertLin.data();
    case AVBD_BUF_EXCLUSIONS: bytes = s->exclusions.size() * 4; return s->exclusions.data();
    case AVBD_BUF_HASHED_IDX: bytes = s->hashedIdx.size() * 4; return s->hashedIdx.data();
    case AVBD_BUF_GLOBAL_IDX: bytes = s->globalIdx.size() * 4; return s->globalIdx.data();
    case AVBD_BUF_TRIS: bytes = s->tris.size() * 16; return s->tris.data();
    case AVBD_BUF_EDGES: bytes = s->edges.size() * 4; return s->edges.data();
    case AVBD_BUF_NBR_START: bytes = s->nbrStart.size() * 4; return s->nbrStart.data();
    case AVBD_BUF_NBR_COUNT: bytes = s->nbrCount.size() * 4; return s->nbrCount.data();
    case AVBD_BUF_NBR_LIST: bytes = s->nbrList.size() * 4; return s->nbrList.data();
    case AVBD_BUF_PARTICLE_IDX: bytes = (size_t)s->numParticles * 4; return s->particleIdx.data();
    case AVBD_BUF_MEMBRANES: bytes = s->membranes.size() * sizeof(oracle::MembraneGPU); return s->membranes.data();
    case AVBD_BUF_BENDS: bytes = s->bends.size() * sizeof(oracle::BendGPU); return s->bends.data();
    // element contacts were swapped at the end of the frame like the manifolds
    case AVBD_BUF_SOFT: bytes = (size_t)s->numSoft * sizeof(oracle::SoftContactGPU); return s->prevSoft.data();
    case AVBD_BUF_DAT_PAIRS: bytes = s->datPairs.size() * 16; return s->datPairs.data();
    case AVBD_BUF_CLOTH_GROUP: bytes = s->clothGroup.size() * 4; return s->clothGroup.data();
    case AVBD_BUF_OGC_PREV: bytes = s->ogcPrev.size() * 16; return s->ogcPrev.data();
    default: bytes = 0; return nullptr;
    }
}
size_t oracle_debug_buffer_size(void* h, int which) {
    size_t bytes = 0;
    oracle_buffer(static_cast<Solver*>(h), which, bytes);
    return bytes;
}
int oracle_debug_read(void* h, int which, void* dst, size_t bytes) {
    size_t have = 0;
    const void* src = oracle_buffer(static_cast<Solver*>(h), which, have);
    if (!src || bytes > have) return AVBD_ERR_INVALID_ARGUMENT;
    std::memcpy(dst, src, bytes);
    return AVBD_OK;
}

}  // extern "C"
