// render.cu — headless render and observation compute: instance transforms
// of rigid colliders, smooth normals of the soft surface, skinned render
// meshes and Push-T pixel observations, written to plain device buffers.
//
// Follows Shaders/50_render.metal:7-212 and Shaders/60_robotics.metal:8-69.
// All of them are one pass over independent records; the Push-T kernel is
// the byte-heavy one (num_envs x res^2 x 3 bytes) and writes 12-byte pixel
// quads per thread so that consecutive threads store consecutive words.
#include "dmath.cuh"
#include "kernels.h"

namespace avbd {

namespace {

__device__ __forceinline__ float fract_(float x) { return x - floorf(x); }

// Golden-ratio hue cycling lifted toward white (50_render.metal:25-32).
__device__ float3 palette(uint32_t i) {
    const float h = fract_((float)i * 0.61803398875f);
    const float3 off = mk3(5.0f / 6.0f, 3.0f / 6.0f, 1.0f / 6.0f);
    float3 p;
    p.x = fabsf(fract_(h + off.x) * 6.0f - 3.0f) - 1.0f;
    p.y = fabsf(fract_(h + off.y) * 6.0f - 3.0f) - 1.0f;
    p.z = fabsf(fract_(h + off.z) * 6.0f - 3.0f) - 1.0f;
    const float3 hue = clamp3(p, s3(0.0f), s3(1.0f));
    const float3 base = s3(0.92f);
    return (base + (hue - base) * 0.62f) * 0.98f;
}

__device__ __forceinline__ float3 safe_normalize(float3 v) {
    const float l = len3(v);
    return l > 1e-12f ? v / l : s3(0.0f);
}

__device__ __forceinline__ void store4(float* o, float a, float b, float c, float w) {
    *reinterpret_cast<float4*>(o) = make_float4(a, b, c, w);
}

}  // namespace

// One record per listed collider (50_render.metal:34-97).
__global__ void k_build_instances(const DevPtrs d, const uint32_t* ids, const float4* colors, uint32_t n,
                                  uint32_t colorMode, float* out) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= n) return;
    const uint32_t col = ids[gid];
    const uint32_t body = d.colOwner[col];
    const float4 pl = d.posLin[body];
    const float4 qb = d.posAng[body];
    const float4 q = q_mul(qb, d.colLocalRot[col]);
    const float3 center = xyz(pl) + q_rotate(qb, xyz(d.colLocalPos[col]));
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    const float xx = x * x, yy = y * y, zz = z * z;
    const float xy = x * y, xz = x * z, yz = y * z;
    const float wx = w * x, wy = w * y, wz = w * z;
    const float3 c0 = mk3(1.0f - 2.0f * (yy + zz), 2.0f * (xy + wz), 2.0f * (xz - wy));
    const float3 c1 = mk3(2.0f * (xy - wz), 1.0f - 2.0f * (xx + zz), 2.0f * (yz + wx));
    const float3 c2 = mk3(2.0f * (xz + wy), 2.0f * (yz - wx), 1.0f - 2.0f * (xx + yy));
    const uint32_t st = d.colShapeType[col] & SHAPE_KIND_MASK;
    const float4 sh = d.colShape[col];
    const float3 sz = st >= 2 ? s3(1.0f) : xyz(sh);
    float* o = out + 24 * (size_t)gid;
    // the static ground slab is not drawn (a floor replaces it)
    if (st == 0 && pl.w <= 0.0f && sh.x > 150.0f) {
        for (int k = 0; k < 24; k += 4) store4(o + k, 0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    store4(o + 0, c0.x * sz.x, c0.y * sz.x, c0.z * sz.x, 0.0f);
    store4(o + 4, c1.x * sz.y, c1.y * sz.y, c1.z * sz.y, 0.0f);
    store4(o + 8, c2.x * sz.z, c2.y * sz.z, c2.z * sz.z, 0.0f);
    store4(o + 12, center.x, center.y, center.z, 1.0f);
    float3 c = pl.w > 0.0f ? palette(colorMode == 1 ? d.colorsA[body] : body) : mk3(0.58f, 0.60f, 0.66f);
    if (colors) {
        const float4 rc = colors[gid];
        if (rc.w > 0.0f) c = xyz(rc);
    }
    store4(o + 16, c.x, c.y, c.z, (float)st);
    store4(o + 20, sh.x, sh.y, sh.w, pl.w > 0.0f ? 1.0f : 0.0f);
}

// Raw face normals (twice the area along the normal), 50_render.metal:104-117.
__global__ void k_face_normals(const DevPtrs d, uint32_t numTris, float4* faceN) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= numTris) return;
    const uint4 tr = d.tris[t];
    const float3 a = xyz(d.posLin[tr.x]), b = xyz(d.posLin[tr.y]), c = xyz(d.posLin[tr.z]);
    faceN[t] = mk4(cross(b - a, c - a), 0.0f);
}

// Angle x area weighted vertex normals with the curvature-thinned render
// thickness (50_render.metal:119-180).
__global__ void k_vertex_normals(const DevPtrs d, const uint32_t* surfVerts, const uint32_t* vtStart,
                                 const uint32_t* vtCount, const uint32_t* vtList, uint32_t numSurf,
                                 const float4* faceN, float clothScale, float4* out) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= numSurf) return;
    const uint32_t v = surfVerts[gid];
    const float3 p = xyz(d.posLin[v]);
    float3 acc = s3(0.0f);
    float wsum = 0.0f;
    const uint32_t s = vtStart[gid], e = s + vtCount[gid];
    for (uint32_t k = s; k < e; k++) {
        const uint32_t t = vtList[k];
        const uint4 tr = d.tris[t];
        const float3 fn = xyz(faceN[t]);
        const float area = 0.5f * len3(fn);
        float3 ea, eb;
        if (tr.x == v) { ea = xyz(d.posLin[tr.y]) - p; eb = xyz(d.posLin[tr.z]) - p; }
        else if (tr.y == v) { ea = xyz(d.posLin[tr.x]) - p; eb = xyz(d.posLin[tr.z]) - p; }
        else { ea = xyz(d.posLin[tr.x]) - p; eb = xyz(d.posLin[tr.y]) - p; }
        const float ang = acosf(clampf(dot(safe_normalize(ea), safe_normalize(eb)), -1.0f, 1.0f));
        const float w = area * ang;
        acc += safe_normalize(fn) * w;
        wsum += w;
    }
    // a fold-over can cancel the weighted sum: fall back to the first face
    const float coherence = wsum > 1e-9f ? len3(acc) / wsum : 0.0f;
    if (len3(acc) < 1e-6f && e > s) acc = xyz(faceN[vtList[s]]);
    const float sc = d.clothVert[v] != 0u ? clothScale : 1.0f;
    const float c2 = clampf(coherence * coherence, 0.0f, 1.0f);
    const float thick = fabsf(d.shape[v].w) * sc * (0.25f + (1.0f - 0.25f) * c2);
    out[v] = mk4(safe_normalize(acc), thick);
}

// Skinned render vertices (50_render.metal:182-212).
__global__ void k_skin_deform(const float4* posLin, const SkinBinding* bind, uint32_t n, float4* out) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= n) return;
    const SkinBinding b = bind[gid];
    const float3 q0 = xyz(posLin[b.ids.x]), q1 = xyz(posLin[b.ids.y]);
    const float3 q2 = xyz(posLin[b.ids.z]), q3 = xyz(posLin[b.ids.w]);
    const float3 p = q0 * b.weights.x + q1 * b.weights.y + q2 * b.weights.z + q3 * b.weights.w;
    // F = Ds Dm^-1 column by column; the normal maps by cof(F)
    const float3 e0 = q1 - q0, e1 = q2 - q0, e2 = q3 - q0;
    const float3 f0 = e0 * b.inv0.x + e1 * b.inv1.x + e2 * b.inv2.x;
    const float3 f1 = e0 * b.inv0.y + e1 * b.inv1.y + e2 * b.inv2.y;
    const float3 f2 = e0 * b.inv0.z + e1 * b.inv1.z + e2 * b.inv2.z;
    const float3 n0 = xyz(b.restNormal);
    float3 nn = cross(f1, f2) * n0.x + cross(f2, f0) * n0.y + cross(f0, f1) * n0.z;
    if (len3(nn) < 1e-10f) nn = n0;
    out[2 * gid] = mk4(p, 1.0f);
    out[2 * gid + 1] = mk4(safe_normalize(nn), 0.0f);
}

namespace {

__device__ __forceinline__ bool in_box(float px, float py, float cx, float cy, float cs, float sn, float hx,
                                       float hy) {
    const float dx = px - cx, dy = py - cy;
    const float lx = cs * dx + sn * dy;
    const float ly = -sn * dx + cs * dy;
    return fabsf(lx) <= hx && fabsf(ly) <= hy;
}

__device__ __forceinline__ uint32_t to_byte(float c) { return (uint32_t)(clampf(c, 0.0f, 1.0f) * 255.0f); }

// Heading of a body in the ground plane as (cos, sin) of atan2(fwd.y, fwd.x)
// for fwd = its rotated +x axis: the normalised (fwd.x, fwd.y), (1, 0) when
// the axis is vertical.
__device__ __forceinline__ void heading(float4 q, float& cs, float& sn) {
    const float3 f = q_rotate(q, mk3(1.0f, 0.0f, 0.0f));
    const float l = sqrtf(f.x * f.x + f.y * f.y);
    if (l > 0.0f) { cs = f.x / l; sn = f.y / l; }
    else { cs = 1.0f; sn = 0.0f; }
}

}  // namespace

// Push-T observations (60_robotics.metal:21-69) in two passes.
// k_pusht_shapes: one thread per environment places its shapes (goal T from
// the table, block T and pusher from the body poses) into 24 floats.
// k_pusht_obs: blockIdx.y walks the environments; every thread reads its
// environment's 24 floats (the same address across the block) and
// classifies pixels.  The pixel-centre offsets (float)j / (res - 1) - 0.5
// are a shared table (the same division as per pixel, done once per block).
// A quad of pixels whose centre is farther from a shape's centre than the
// shape's bounding radius plus two pixel widths cannot touch it, so that
// shape's exact test is skipped (most quads are background).
// QUADS (res a multiple of 4): each thread classifies four consecutive
// pixels of a row into three 32-bit words, the block stages its 3 KB run in
// shared memory and writes it out as 16-byte stores (the run starts on a
// 16-byte boundary: 3 * res^2 and 3072 are multiples of 48).  Otherwise one
// thread per pixel with byte stores.
constexpr uint32_t kObsThreads = 256;

__device__ __forceinline__ bool near_(float x, float y, float cx, float cy, float r2) {
    const float dx = x - cx, dy = y - cy;
    return dx * dx + dy * dy <= r2;
}

__global__ void k_pusht_shapes(const float4* posLin, const float4* posAng, const PushTDev* envs, uint32_t numEnvs,
                               uint32_t res, float4* shapes) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= numEnvs) return;
    const PushTDev env = envs[e];
    float sh[24];
    const float gx = env.frame.z + env.frame.x, gy = env.frame.w + env.frame.y;
    const float gc = env.goalCos, gs = env.goalSin;
    sh[0] = gx + (-gs) * 0.125f; sh[1] = gy + gc * 0.125f;    // goal bar centre
    sh[2] = gx + gs * 0.325f;    sh[3] = gy + (-gc) * 0.325f; // goal stem centre
    sh[4] = gc; sh[5] = gs;
    float cs, sn;
    heading(posAng[env.ids.y], cs, sn);
    sh[6] = posLin[env.ids.y].x; sh[7] = posLin[env.ids.y].y; sh[8] = cs; sh[9] = sn;
    heading(posAng[env.ids.z], cs, sn);
    sh[10] = posLin[env.ids.z].x; sh[11] = posLin[env.ids.z].y; sh[12] = cs; sh[13] = sn;
    sh[14] = posLin[env.ids.x].x; sh[15] = posLin[env.ids.x].y;
    sh[16] = env.frame.x; sh[17] = env.frame.y;
    sh[18] = 2.0f * env.halfWin;
    // squared cull radii: bar (0.5 x 0.125 half extents), stem (0.125 x
    // 0.325), pusher disc (0.13), each plus two pixel widths
    const float pw = fabsf(sh[18]) / (float)(res - 1u);
    const float rb = 0.5154f + 2.0f * pw, rs = 0.3483f + 2.0f * pw, rt = 0.13f + 2.0f * pw;
    sh[19] = rb * rb; sh[20] = rs * rs; sh[21] = rt * rt;
    sh[22] = 0.0f; sh[23] = 0.0f;
    for (int k = 0; k < 6; k++) shapes[6 * e + k] = make_float4(sh[4 * k], sh[4 * k + 1], sh[4 * k + 2], sh[4 * k + 3]);
}

template <bool QUADS>
__global__ void __launch_bounds__(kObsThreads) k_pusht_obs(const float4* shapes, uint32_t numEnvs, uint32_t res,
                                                           uint8_t* out) {
    extern __shared__ float offs[];  // res entries
    __shared__ uint32_t words[3 * kObsThreads];
    const uint32_t perRow = QUADS ? res / 4u : res;
    const uint32_t perEnv = perRow * res;
    const uint32_t blockFirst = blockIdx.x * kObsThreads;
    const uint32_t valid = perEnv - blockFirst < kObsThreads ? perEnv - blockFirst : kObsThreads;
    const float denom = (float)(res - 1u);
    __shared__ float4 shs[2][6];     // QUADS: this and the next environment's shapes
    for (uint32_t j = threadIdx.x; j < res; j += kObsThreads) offs[j] = (float)j / denom - 0.5f;
    if (QUADS && threadIdx.x < 6u && blockIdx.y < numEnvs)
        shs[0][threadIdx.x] = shapes[6 * (size_t)blockIdx.y + threadIdx.x];
    __syncthreads();
    // row and column of this thread's first pixel (quad index / row length)
    const uint32_t i = blockFirst + threadIdx.x;
    uint32_t py = i / perRow;
    const uint32_t px0 = (QUADS ? 4u : 1u) * (i - py * perRow);
    uint32_t buf = 0;
    for (uint32_t e = blockIdx.y; e < numEnvs; e += gridDim.y, buf ^= 1u) {
        float4 s0, s1, s2, s3, s4, s5;
        if (QUADS) {
            // six threads fetch the next environment's shapes into the other
            // buffer (last read an iteration ago, before that iteration's
            // barriers); they are visible after this iteration's barriers
            const uint32_t en = e + gridDim.y;
            if (threadIdx.x < 6u && en < numEnvs) shs[buf ^ 1u][threadIdx.x] = shapes[6 * (size_t)en + threadIdx.x];
            s0 = shs[buf][0]; s1 = shs[buf][1]; s2 = shs[buf][2]; s3 = shs[buf][3]; s4 = shs[buf][4]; s5 = shs[buf][5];
        } else {
            const float4* S = shapes + 6 * (size_t)e;
            s0 = S[0]; s1 = S[1]; s2 = S[2]; s3 = S[3]; s4 = S[4]; s5 = S[5];
        }
        uint32_t kinds = 0;  // 2 bits per pixel: 0 background, 1 goal, 2 block, 3 pusher
        if (threadIdx.x < valid) {
            constexpr int N = QUADS ? 4 : 1;
            const float wy = s4.y + offs[py] * s4.z;
            float wx[N];
#pragma unroll
            for (int k = 0; k < N; k++) wx[k] = s4.x + offs[px0 + k] * s4.z;
            const float cx = 0.5f * (wx[0] + wx[N - 1]);
            const bool gBar = near_(cx, wy, s0.x, s0.y, s4.w), gStem = near_(cx, wy, s0.z, s0.w, s5.x);
            const bool bBar = near_(cx, wy, s1.z, s1.w, s4.w), bStem = near_(cx, wy, s2.z, s2.w, s5.x);
            const bool tip = near_(cx, wy, s3.z, s3.w, s5.y);
            if (gBar || gStem || bBar || bStem || tip) {
#pragma unroll
                for (int k = 0; k < N; k++) {
                    uint32_t kind = 0;
                    if ((gBar && in_box(wx[k], wy, s0.x, s0.y, s1.x, s1.y, 0.5f, 0.125f)) ||
                        (gStem && in_box(wx[k], wy, s0.z, s0.w, s1.x, s1.y, 0.125f, 0.325f)))
                        kind = 1;
                    if (bBar && in_box(wx[k], wy, s1.z, s1.w, s2.x, s2.y, 0.5f, 0.125f)) kind = 2;
                    if (bStem && in_box(wx[k], wy, s2.z, s2.w, s3.x, s3.y, 0.125f, 0.325f)) kind = 2;
                    if (tip) {
                        const float dx = wx[k] - s3.z, dy = wy - s3.w;
                        if (sqrtf(dx * dx + dy * dy) < 0.13f) kind = 3;
                    }
                    kinds |= kind << (2 * k);
                }
            }
        }
        // the four palette entries as bytes
        const uint32_t pal[4][3] = {
            {to_byte(0.06f), to_byte(0.06f), to_byte(0.06f)},
            {to_byte(0.10f), to_byte(0.55f), to_byte(0.12f)},
            {to_byte(0.85f), to_byte(0.15f), to_byte(0.12f)},
            {to_byte(0.2f), to_byte(0.4f), to_byte(0.95f)}};
        if (QUADS) {
            uint32_t w0, w1, w2;
            if (kinds == 0u) {  // four background pixels
                const uint32_t g = pal[0][0];
                w0 = w1 = w2 = g | (g << 8) | (g << 16) | (g << 24);
            } else {
                uint32_t b[12];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const uint32_t kind = (kinds >> (2 * k)) & 3u;
                    b[3 * k] = pal[kind][0]; b[3 * k + 1] = pal[kind][1]; b[3 * k + 2] = pal[kind][2];
                }
                w0 = b[0] | (b[1] << 8) | (b[2] << 16) | (b[3] << 24);
                w1 = b[4] | (b[5] << 8) | (b[6] << 16) | (b[7] << 24);
                w2 = b[8] | (b[9] << 8) | (b[10] << 16) | (b[11] << 24);
            }
            __syncthreads();  // the previous environment's words are out
            words[3 * threadIdx.x] = w0;
            words[3 * threadIdx.x + 1] = w1;
            words[3 * threadIdx.x + 2] = w2;
            __syncthreads();
            // 3 * valid words from byte (e * res^2 + 4 * blockFirst) * 3
            uint32_t* dst = reinterpret_cast<uint32_t*>(out + ((size_t)e * res * res + 4u * (size_t)blockFirst) * 3u);
            const uint32_t nWords = 3u * valid, nVec = nWords / 4u;
            for (uint32_t v = threadIdx.x; v < nVec; v += kObsThreads)
                reinterpret_cast<uint4*>(dst)[v] =
                    make_uint4(words[4 * v], words[4 * v + 1], words[4 * v + 2], words[4 * v + 3]);
            for (uint32_t w = 4u * nVec + threadIdx.x; w < nWords; w += kObsThreads) dst[w] = words[w];
        } else if (threadIdx.x < valid) {
            const uint32_t kind = kinds & 3u;
            uint8_t* o = out + ((size_t)e * res * res + i) * 3u;
            o[0] = (uint8_t)pal[kind][0]; o[1] = (uint8_t)pal[kind][1]; o[2] = (uint8_t)pal[kind][2];
        }
    }
}

static uint32_t blocks_for(uint32_t n, uint32_t threads) { return n == 0 ? 1u : (n + threads - 1) / threads; }

void launch_build_instances(const DevPtrs& d, const uint32_t* ids, const float4* colors, uint32_t n,
                            uint32_t colorMode, float* out, cudaStream_t st) {
    if (n) k_build_instances<<<blocks_for(n, 128), 128, 0, st>>>(d, ids, colors, n, colorMode, out);
}

void launch_soft_normals(const DevPtrs& d, uint32_t numTris, const uint32_t* surfVerts, const uint32_t* vtStart,
                         const uint32_t* vtCount, const uint32_t* vtList, uint32_t numSurf, float4* faceN,
                         float clothScale, float4* out, cudaStream_t st) {
    if (!numTris || !numSurf) return;
    k_face_normals<<<blocks_for(numTris, 256), 256, 0, st>>>(d, numTris, faceN);
    k_vertex_normals<<<blocks_for(numSurf, 128), 128, 0, st>>>(d, surfVerts, vtStart, vtCount, vtList, numSurf,
                                                               faceN, clothScale, out);
}

void launch_skin_deform(const float4* posLin, const SkinBinding* b, uint32_t n, float4* out, cudaStream_t st) {
    if (n) k_skin_deform<<<blocks_for(n, 256), 256, 0, st>>>(posLin, b, n, out);
}

void launch_pusht_obs(const float4* posLin, const float4* posAng, const PushTDev* envs, uint32_t numEnvs,
                      uint32_t res, float4* shapes, uint8_t* out, cudaStream_t st) {
    if (!numEnvs) return;
    k_pusht_shapes<<<blocks_for(numEnvs, 128), 128, 0, st>>>(posLin, posAng, envs, numEnvs, res, shapes);
    const bool quads = res % 4u == 0u;
    const uint32_t perEnv = quads ? res * res / 4u : res * res;
    // about eight resident blocks per SM in all; each block walks several
    // environments so that its offset table is built once for many
    const uint32_t bx = blocks_for(perEnv, kObsThreads);
    uint32_t by = (148u * 8u + bx - 1u) / bx;
    by = by < numEnvs ? by : numEnvs;
    by = by < 65535u ? (by ? by : 1u) : 65535u;
    const dim3 grid(bx, by);
    const size_t smem = sizeof(float) * res;  // res <= 4096: at most 16 KB
    if (quads) k_pusht_obs<true><<<grid, kObsThreads, smem, st>>>(shapes, numEnvs, res, out);
    else k_pusht_obs<false><<<grid, kObsThreads, smem, st>>>(shapes, numEnvs, res, out);
}

}  // namespace avbd
