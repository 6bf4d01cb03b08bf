// oracle_render.cpp — CPU restatement of the headless render and
// observation compute (Shaders/50_render.metal:7-212,
// Shaders/60_robotics.metal:8-69).  Test infrastructure: the checker of the
// CUDA kernels in render.cu, never part of the product path.
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle_solver.h"

using namespace oracle;

namespace {

float fract_(float x) { return x - std::floor(x); }

// 50_render.metal:25-32
F3 palette(uint32_t i) {
    float h = fract_((float)i * 0.61803398875f);
    F3 off = f3(5.0f / 6.0f, 3.0f / 6.0f, 1.0f / 6.0f);
    F3 p = f3(std::fabs(fract_(h + off.x) * 6.0f - 3.0f) - 1.0f, std::fabs(fract_(h + off.y) * 6.0f - 3.0f) - 1.0f,
              std::fabs(fract_(h + off.z) * 6.0f - 3.0f) - 1.0f);
    F3 hue = clamp3(p, f3s(0.0f), f3s(1.0f));
    F3 base = f3s(0.92f);
    return (base + (hue - base) * 0.62f) * 0.98f;
}

F3 safe_normalize(F3 v) {
    float l = length(v);
    return l > 1e-12f ? v / l : f3s(0.0f);
}

bool in_box(float px, float py, float cx, float cy, float cs, float sn, float hx, float hy) {
    float dx = px - cx, dy = py - cy;
    float lx = cs * dx + sn * dy;
    float ly = -sn * dx + cs * dy;
    return std::fabs(lx) <= hx && std::fabs(ly) <= hy;
}

uint8_t to_byte(float c) { return (uint8_t)(clampf_(c, 0.0f, 1.0f) * 255.0f); }

// cos and sin of atan2(fwd.y, fwd.x) for the rotated +x axis
void heading(F4 q, float& cs, float& sn) {
    F3 f = q_rotate(q, f3(1, 0, 0));
    float l = std::sqrt(f.x * f.x + f.y * f.y);
    if (l > 0.0f) { cs = f.x / l; sn = f.y / l; }
    else { cs = 1.0f; sn = 0.0f; }
}

}  // namespace

extern "C" {

// 50_render.metal:34-97
int oracle_build_instances(void* h, const uint32_t* ids, uint32_t n, const float* colors, uint32_t mode, float* out) {
    Solver* s = static_cast<Solver*>(h);
    for (uint32_t g = 0; g < n; g++) {
        uint32_t col = ids[g];
        uint32_t body = s->colOwner[col];
        F4 pl = s->posLin[body], qb = s->posAng[body];
        F4 q = q_mul(qb, s->colLocalRot[col]);
        F3 center = xyz(pl) + q_rotate(qb, xyz(s->colLocalPos[col]));
        float x = q.x, y = q.y, z = q.z, w = q.w;
        float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, wx = w * x, wy = w * y, wz = w * z;
        F3 c0 = f3(1.0f - 2.0f * (yy + zz), 2.0f * (xy + wz), 2.0f * (xz - wy));
        F3 c1 = f3(2.0f * (xy - wz), 1.0f - 2.0f * (xx + zz), 2.0f * (yz + wx));
        F3 c2 = f3(2.0f * (xz + wy), 2.0f * (yz - wx), 1.0f - 2.0f * (xx + yy));
        uint32_t st = s->colShapeType[col] & 0xFu;
        F4 sh = s->colShape[col];
        F3 sz = st >= 2 ? f3s(1.0f) : xyz(sh);
        float* o = out + 24 * (size_t)g;
        if (st == 0 && pl.w <= 0.0f && sh.x > 150.0f) { std::memset(o, 0, 24 * sizeof(float)); continue; }
        float rec[24] = {c0.x * sz.x, c0.y * sz.x, c0.z * sz.x, 0.0f, c1.x * sz.y, c1.y * sz.y, c1.z * sz.y, 0.0f,
                         c2.x * sz.z, c2.y * sz.z, c2.z * sz.z, 0.0f, center.x, center.y, center.z, 1.0f};
        F3 c = pl.w > 0.0f ? palette(mode == 1 ? s->colorsA[body] : body) : f3(0.58f, 0.60f, 0.66f);
        if (colors && colors[4 * g + 3] > 0.0f) c = f3(colors[4 * g], colors[4 * g + 1], colors[4 * g + 2]);
        rec[16] = c.x; rec[17] = c.y; rec[18] = c.z; rec[19] = (float)st;
        rec[20] = sh.x; rec[21] = sh.y; rec[22] = sh.w; rec[23] = pl.w > 0.0f ? 1.0f : 0.0f;
        std::memcpy(o, rec, sizeof(rec));
    }
    return 0;
}

// 50_render.metal:104-180: face normals, then the angle x area weighted
// gather over each surface vertex's incident triangles (in surface order)
int oracle_soft_normals(void* h, float clothScale, float* out) {
    Solver* s = static_cast<Solver*>(h);
    uint32_t nt = s->numTris, nb = s->nb;
    if (nt == 0) return 0;
    std::vector<F3> faceN(nt);
    std::vector<std::vector<uint32_t>> inc(nb);
    for (uint32_t t = 0; t < nt; t++) {
        U4 tr = s->tris[t];
        F3 a = xyz(s->posLin[tr.x]), b = xyz(s->posLin[tr.y]), c = xyz(s->posLin[tr.z]);
        faceN[t] = cross(b - a, c - a);
        inc[tr.x].push_back(t); inc[tr.y].push_back(t); inc[tr.z].push_back(t);
    }
    std::vector<uint8_t> cloth(nb, 0);
    for (uint32_t t = 0; t < s->numAuthoredTris; t++) {
        cloth[s->tris[t].x] = 1; cloth[s->tris[t].y] = 1; cloth[s->tris[t].z] = 1;
    }
    for (uint32_t v = 0; v < nb; v++) {
        if (inc[v].empty()) continue;
        F3 p = xyz(s->posLin[v]);
        F3 acc = f3s(0.0f);
        float wsum = 0.0f;
        for (uint32_t t : inc[v]) {
            U4 tr = s->tris[t];
            F3 fn = faceN[t];
            float area = 0.5f * length(fn);
            F3 ea, eb;
            if (tr.x == v) { ea = xyz(s->posLin[tr.y]) - p; eb = xyz(s->posLin[tr.z]) - p; }
            else if (tr.y == v) { ea = xyz(s->posLin[tr.x]) - p; eb = xyz(s->posLin[tr.z]) - p; }
            else { ea = xyz(s->posLin[tr.x]) - p; eb = xyz(s->posLin[tr.y]) - p; }
            float ang = std::acos(clampf_(dot(safe_normalize(ea), safe_normalize(eb)), -1.0f, 1.0f));
            float w = area * ang;
            acc = acc + safe_normalize(fn) * w;
            wsum += w;
        }
        float coherence = wsum > 1e-9f ? length(acc) / wsum : 0.0f;
        if (length(acc) < 1e-6f) acc = faceN[inc[v][0]];
        float sc = cloth[v] ? clothScale : 1.0f;
        float c2 = clampf_(coherence * coherence, 0.0f, 1.0f);
        float thick = std::fabs(s->shape[v].w) * sc * (0.25f + (1.0f - 0.25f) * c2);
        F3 n = safe_normalize(acc);
        out[4 * v] = n.x; out[4 * v + 1] = n.y; out[4 * v + 2] = n.z; out[4 * v + 3] = thick;
    }
    return 0;
}

// GPUSolver.swift:1849-1907: rest normal (unit, +z when zero) and rest
// inverse; a zero inverse becomes the inverse of the scene-pose edge matrix
int oracle_set_skin_bindings(void* h, const avbd_skin_binding* b, uint32_t n) {
    Solver* s = static_cast<Solver*>(h);
    s->skins.assign(n, Solver::Skin{});
    for (uint32_t i = 0; i < n; i++) {
        const avbd_skin_binding& g = b[i];
        for (int k = 0; k < 4; k++)
            if (g.ids[k] >= s->nb) return AVBD_ERR_INVALID_ARGUMENT;
        Solver::Skin& o = s->skins[i];
        o.ids = U4{g.ids[0], g.ids[1], g.ids[2], g.ids[3]};
        o.weights = F4{g.weights[0], g.weights[1], g.weights[2], g.weights[3]};
        const float* rn = g.rest_normal;
        float l2 = rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2];
        if (l2 > 1e-12f) { float l = std::sqrt(l2); o.restNormal = f3(rn[0] / l, rn[1] / l, rn[2] / l); }
        else o.restNormal = f3(0, 0, 1);
        auto sq = [](const float* v) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; };
        if (sq(g.inv0) + sq(g.inv1) + sq(g.inv2) > 1e-16f) {
            o.inv0 = f3(g.inv0[0], g.inv0[1], g.inv0[2]);
            o.inv1 = f3(g.inv1[0], g.inv1[1], g.inv1[2]);
            o.inv2 = f3(g.inv2[0], g.inv2[1], g.inv2[2]);
            continue;
        }
        F3 x0 = xyz(s->scenePos[g.ids[0]]);
        F3 d0 = xyz(s->scenePos[g.ids[1]]) - x0, d1 = xyz(s->scenePos[g.ids[2]]) - x0, d2 = xyz(s->scenePos[g.ids[3]]) - x0;
        F3 r0 = cross(d1, d2), r1 = cross(d2, d0), r2 = cross(d0, d1);
        float det = d0.x * r0.x + d0.y * r0.y + d0.z * r0.z;
        if (std::fabs(det) > 1e-12f) {
            o.inv0 = f3(r0.x / det, r0.y / det, r0.z / det);
            o.inv1 = f3(r1.x / det, r1.y / det, r1.z / det);
            o.inv2 = f3(r2.x / det, r2.y / det, r2.z / det);
        } else {
            o.inv0 = f3(1, 0, 0); o.inv1 = f3(0, 1, 0); o.inv2 = f3(0, 0, 1);
        }
    }
    return 0;
}

// 50_render.metal:182-212
int oracle_skin_deform(void* h, float* out) {
    Solver* s = static_cast<Solver*>(h);
    for (size_t i = 0; i < s->skins.size(); i++) {
        const Solver::Skin& b = s->skins[i];
        F3 q0 = xyz(s->posLin[b.ids.x]), q1 = xyz(s->posLin[b.ids.y]);
        F3 q2 = xyz(s->posLin[b.ids.z]), q3 = xyz(s->posLin[b.ids.w]);
        F3 p = q0 * b.weights.x + q1 * b.weights.y + q2 * b.weights.z + q3 * b.weights.w;
        F3 e0 = q1 - q0, e1 = q2 - q0, e2 = q3 - q0;
        F3 f0 = e0 * b.inv0.x + e1 * b.inv1.x + e2 * b.inv2.x;
        F3 f1 = e0 * b.inv0.y + e1 * b.inv1.y + e2 * b.inv2.y;
        F3 f2 = e0 * b.inv0.z + e1 * b.inv1.z + e2 * b.inv2.z;
        F3 n0 = b.restNormal;
        F3 n = cross(f1, f2) * n0.x + cross(f2, f0) * n0.y + cross(f0, f1) * n0.z;
        if (length(n) < 1e-10f) n = n0;
        F3 nn = safe_normalize(n);
        float rec[8] = {p.x, p.y, p.z, 1.0f, nn.x, nn.y, nn.z, 0.0f};
        std::memcpy(out + 8 * i, rec, sizeof(rec));
    }
    return 0;
}

// 60_robotics.metal:21-69
int oracle_render_pusht_obs(void* h, const avbd_pusht_env* envs, uint32_t numEnvs, uint32_t res, uint8_t* out) {
    Solver* s = static_cast<Solver*>(h);
    const uint8_t pal[4][3] = {{to_byte(0.06f), to_byte(0.06f), to_byte(0.06f)},
                               {to_byte(0.10f), to_byte(0.55f), to_byte(0.12f)},
                               {to_byte(0.85f), to_byte(0.15f), to_byte(0.12f)},
                               {to_byte(0.2f), to_byte(0.4f), to_byte(0.95f)}};
    for (uint32_t e = 0; e < numEnvs; e++) {
        const avbd_pusht_env& env = envs[e];
        float gc = (float)std::cos((double)env.goal[0]), gs = (float)std::sin((double)env.goal[0]);
        float gx = env.frame[2] + env.frame[0], gy = env.frame[3] + env.frame[1];
        float barX = gx + (-gs) * 0.125f, barY = gy + gc * 0.125f;
        float stemX = gx + gs * 0.325f, stemY = gy + (-gc) * 0.325f;
        float c1, s1, c2, s2;
        heading(s->posAng[env.ids[1]], c1, s1);
        heading(s->posAng[env.ids[2]], c2, s2);
        F4 pb = s->posLin[env.ids[1]], ps = s->posLin[env.ids[2]], pt = s->posLin[env.ids[0]];
        float span = 2.0f * env.goal[1], denom = (float)(res - 1u);
        for (uint32_t py = 0; py < res; py++) {
            float wy = env.frame[1] + ((float)py / denom - 0.5f) * span;
            for (uint32_t px = 0; px < res; px++) {
                float wx = env.frame[0] + ((float)px / denom - 0.5f) * span;
                int kind = 0;
                if (in_box(wx, wy, barX, barY, gc, gs, 0.5f, 0.125f) || in_box(wx, wy, stemX, stemY, gc, gs, 0.125f, 0.325f))
                    kind = 1;
                if (in_box(wx, wy, pb.x, pb.y, c1, s1, 0.5f, 0.125f)) kind = 2;
                if (in_box(wx, wy, ps.x, ps.y, c2, s2, 0.125f, 0.325f)) kind = 2;
                float dx = wx - pt.x, dy = wy - pt.y;
                if (std::sqrt(dx * dx + dy * dy) < 0.13f) kind = 3;
                uint8_t* o = out + (((size_t)e * res + py) * res + px) * 3;
                o[0] = pal[kind][0]; o[1] = pal[kind][1]; o[2] = pal[kind][2];
            }
        }
    }
    return 0;
}

}  // extern "C"
