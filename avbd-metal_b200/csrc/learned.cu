// learned.cu — learned warm start: per-vertex features, a 32-128-128-128-16
// MLP (BF16 weights and activations, FP32 accumulation on the tensor cores)
// for inference and training, and the acceptance test that keeps a predicted
// warm start only when it is no worse than the plain gamma warm start.
//
// The MLP predicts the correction the solve applies to the plain warm start
// of every dynamic particle, in units of s = max(|g|, 1) dt^2:
//   x0 = x_plain + s * MLP(features)[0-2],
// and, when the model covers rigid bodies (Params::learnRigid), of every
// dynamic rigid body's pose, the rotation as the arc length it sweeps at the
// body's bounding radius r:
//   q0 = q_plain (+) (s / r) * MLP(features)[3-5]   (q_addw, tangent space).
// Learned rows list the particles first, then the rigid bodies.
// Features (32, normalised by per-feature mean and 1/std stored with the
// model): [0-2] inertial offset (x~ - x_start)/s, [3-5] plain warm-start
// offset (x_plain - x_start)/s, [6-8] previous-frame displacement
// v_prev dt / s, [9] incident contact count / 4, [10-12] summed oriented
// contact normal, [13] smallest contact gap / s (clipped), [14] log(1 +
// stiffness dt^2 / m) of the incident elements, [15] 1; rigid rows only
// (zeros for particles): [16] 1, [17-19] plain warm-start rotation
// q_sub(q_plain, q_start) r / s, [20-22] world up axis in the body frame,
// [23] log(1 + r / s) / 10, [24] incident position-PD hinge motors / 4,
// [28-30] the rotation those motors ask for at the plain warm start (sum
// of hinge axis x -(twist - target), as arc length at r in units of s),
// [31] log(1 + sum kp dt^2 / (m r^2)); 1-ring aggregates over the vertices sharing a tet or spring: [25]
// ring size / 10, [26] mean neighbour contact count / 4, [27] smallest
// neighbour contact gap / s (clipped).  Contacts are rigid manifolds and
// element contacts alike.
//
// Parameter block (fp32, also the layout of the gradients): W1[128][32], b1,
// W2[128][128], b2, W3[128][128], b3, W4[16][128], b4[16].  The weights are
// mirrored as BF16 for the tensor cores.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>

#include "../../include/avbd.h"
#include "dmath.cuh"
#include "kernels.h"

namespace avbd {

namespace mlp {
constexpr int DIN = 32, HID = 128, DOUT = 16, USED_OUT = 6;
constexpr uint32_t OW1 = 0, OB1 = OW1 + HID * DIN, OW2 = OB1 + HID, OB2 = OW2 + HID * HID, OW3 = OB2 + HID,
                   OB3 = OW3 + HID * HID, OW4 = OB3 + HID, OB4 = OW4 + DOUT * HID, NPARAM = OB4 + DOUT;
// bf16 weight mirror: W1 | W2 | W3 | W4
constexpr uint32_t HW1 = 0, HW2 = HW1 + HID * DIN, HW3 = HW2 + HID * HID, HW4 = HW3 + HID * HID,
                   NHALF = HW4 + DOUT * HID;
// normalisation block: xmean[32], xinvstd[32], ymean[16], ystd[16]
constexpr uint32_t NNORM = 96, NX_MEAN = 0, NX_INV = 32, NY_MEAN = 64, NY_STD = 80;
}  // namespace mlp

namespace {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}


// ---------------------------------------------------------------------------
// Fused inference on the Blackwell tensor cores (tcgen05): one CTA of four
// warps per 128-row tile, persistent over the batch.  The weights live in
// global memory as an image of their shared-memory form — the UMMA canonical
// K-major layout without swizzle (8-row x 16-byte core matrices: element
// (r, k) of an operand with row-group stride `sbo` at (r / 8) sbo + (k / 8)
// 128 + (r % 8) 16 + (k % 8) 2 bytes) — and each CTA stages them once with
// bulk asynchronous copies completing on an mbarrier; a layer is 2 (K = 32) or 8 (K = 128) tcgen05.mma instructions of
// M = 128, K = 16, issued by one thread, accumulating in TMEM (128 lanes =
// the tile's rows, N fp32 columns); each warp reads its 32 rows back with
// tcgen05.ld, adds the bias, applies ReLU, rounds to BF16 and writes the next
// layer's A operand in place.  Completion of every layer's MMAs is signalled
// by tcgen05.commit on an mbarrier; every wait on it is bounded and a
// timeout sets *status (the CTA then frees its TMEM and stops).
// ---------------------------------------------------------------------------
namespace tc {
constexpr uint32_t ROWS = 128;
constexpr uint32_t SBO_K128 = 2048, SBO_K32 = 512;      // row-group strides (K = 128, K = 32)
// shared memory: weight image | layer operand | biases b1 b2 b3 b4 (fp32) |
// normalisation block (fp32) | MMA barrier | staging barrier | TMEM address
constexpr uint32_t W1 = 0, W2 = W1 + 128 * 32 * 2, W3 = W2 + 128 * 128 * 2, W4 = W3 + 128 * 128 * 2,
                   ACT = W4 + 16 * 128 * 2, BIAS = ACT + ROWS * 128 * 2, NORM = BIAS + (3 * 128 + 16) * 4,
                   BAR = NORM + 96 * 4, WBAR = BAR + 8, TSLOT = WBAR + 8, SMEM = TSLOT + 8;
constexpr uint32_t WBYTES = ACT - W1;                    // the weight image: 77,824 bytes
constexpr uint32_t STAGED = WBYTES + (NORM - BIAS) + 96 * 4;   // every byte the staging barrier expects
constexpr uint32_t TMEM_COLS = 128;
constexpr uint64_t WAIT_NS = 1000000000ull;              // a wait gives up after one second

__device__ __forceinline__ uint32_t off(uint32_t r, uint32_t k, uint32_t sbo) {
    return (r >> 3) * sbo + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}
// shared-memory matrix descriptor: start address, LBO = 128 B (the second
// 8-element K chunk), SBO, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}
// instruction descriptor of kind::f16: F32 accumulator, BF16 A and B, both
// K-major, N >> 3, M >> 4
__host__ __device__ constexpr uint32_t idesc(uint32_t m, uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem), "l"(a), "l"(b), "r"(id), "r"(acc));
}
__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ uint64_t now_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// bounded wait for the mbarrier phase `parity`; false on timeout
__device__ __forceinline__ bool wait(uint32_t bar, uint32_t parity) {
    const uint64_t t0 = now_ns();
    for (uint32_t i = 0;; i++) {
        if ((i & 255u) == 255u && now_ns() - t0 > WAIT_NS) return false;
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
// bulk asynchronous copy global -> this CTA's shared memory (no multicast),
// completing `bytes` of the barrier's transaction count
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 32 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = __uint_as_float(r[j]);
}
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}
}  // namespace tc

__global__ void __launch_bounds__(128) k_mlp_infer_tc(const bf16* __restrict__ W, const float* __restrict__ prm,
                                                      const float* __restrict__ norm, const float* __restrict__ X,
                                                      uint32_t n, float* __restrict__ Y, uint32_t* status,
                                                      bool issue = true) {
    using namespace mlp;
    extern __shared__ __align__(128) unsigned char sm[];
    const uint32_t t = threadIdx.x, warp = t >> 5;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    const uint32_t bar = sbase + tc::BAR, wbar = sbase + tc::WBAR;
    // the weight image (already in the canonical layout), the biases and the
    // normalisation block: nine bulk copies on one barrier
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(wbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        tc::expect_tx(wbar, tc::STAGED);
        const unsigned char* img = reinterpret_cast<const unsigned char*>(W);
        tc::bulk_load(sbase + tc::W1, img + tc::W1, tc::W2 - tc::W1, wbar);
        tc::bulk_load(sbase + tc::W2, img + tc::W2, tc::W3 - tc::W2, wbar);
        tc::bulk_load(sbase + tc::W3, img + tc::W3, tc::W4 - tc::W3, wbar);
        tc::bulk_load(sbase + tc::W4, img + tc::W4, tc::ACT - tc::W4, wbar);
        tc::bulk_load(sbase + tc::BIAS, prm + OB1, 128 * 4, wbar);
        tc::bulk_load(sbase + tc::BIAS + 512, prm + OB2, 128 * 4, wbar);
        tc::bulk_load(sbase + tc::BIAS + 1024, prm + OB3, 128 * 4, wbar);
        tc::bulk_load(sbase + tc::BIAS + 1536, prm + OB4, 16 * 4, wbar);
        tc::bulk_load(sbase + tc::NORM, norm, 96 * 4, wbar);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + tc::TSLOT),
                     "r"(tc::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + tc::TSLOT);
    const uint32_t lane_addr = tmem + ((warp * 32u) << 16);   // this warp's 32 TMEM lanes
    const uint32_t row = t;                                    // tile row held by this thread
    uint32_t phase = 0;
    // the weights have landed (bounded wait; block-uniform outcome)
    bool ok = __syncthreads_and(tc::wait(wbar, 0) ? 1 : 0) != 0;
    if (!ok) tc::wait(wbar, 0);        // give copies still in flight one more bounded wait
    const float* sbias = reinterpret_cast<const float*>(sm + tc::BIAS);
    const float* snorm = reinterpret_cast<const float*>(sm + tc::NORM);
    const uint32_t tiles = (n + tc::ROWS - 1) / tc::ROWS;
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t r = tile * tc::ROWS + row;
        // layer-1 operand: normalised features, BF16 (the row's 128 bytes as
        // eight 16-byte loads, all in flight together)
        float4 xr[DIN / 4];
#pragma unroll
        for (uint32_t q = 0; q < DIN / 4; q++)
            xr[q] = r < n ? reinterpret_cast<const float4*>(X + (size_t)r * DIN)[q] : make_float4(0, 0, 0, 0);
#pragma unroll
        for (uint32_t kg = 0; kg < DIN / 8; kg++) {
            const float* xv = reinterpret_cast<const float*>(&xr[2 * kg]);
            uint32_t w[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const uint32_t c = kg * 8 + 2 * e;
                const float a = r < n ? (xv[2 * e] - snorm[NX_MEAN + c]) * snorm[NX_INV + c] : 0.0f;
                const float b = r < n ? (xv[2 * e + 1] - snorm[NX_MEAN + c + 1]) * snorm[NX_INV + c + 1] : 0.0f;
                w[e] = pack_bf16(a, b);
            }
            *reinterpret_cast<uint4*>(sm + tc::ACT + tc::off(row, kg * 8, tc::SBO_K128)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        for (int layer = 0; layer < 4 && ok; layer++) {
            tc::fence_proxy();          // the operand writes above are read by the tensor core
            tc::fence_before();
            __syncthreads();
            tc::fence_after();
            if (t == 0 && issue) {       // issue = false only in the timeout test: nothing ever arrives
                const uint32_t wbase = layer == 0 ? tc::W1 : (layer == 1 ? tc::W2 : (layer == 2 ? tc::W3 : tc::W4));
                const uint32_t wsbo = layer == 0 ? tc::SBO_K32 : tc::SBO_K128;
                const uint32_t steps = layer == 0 ? DIN / 16 : HID / 16;
                const uint32_t id = tc::idesc(128, layer == 3 ? DOUT : HID);
                for (uint32_t s = 0; s < steps; s++)
                    tc::mma(tmem, tc::desc(sbase + tc::ACT + 256u * s, tc::SBO_K128),
                            tc::desc(sbase + wbase + 256u * s, wsbo), id, s > 0 ? 1u : 0u);
                tc::commit(bar);
            }
            // block-uniform outcome: every thread leaves the loop together
            ok = __syncthreads_and(tc::wait(bar, phase) ? 1 : 0) != 0;
            phase ^= 1u;
            tc::fence_after();
            if (!ok) break;
            if (layer < 3) {
                // bias, ReLU, BF16: the next layer's operand, written in place
                const float* bias = sbias + 128 * layer;
#pragma unroll 1
                for (uint32_t c0 = 0; c0 < HID; c0 += 32) {
                    float v[32];
                    tc::ld32(lane_addr + c0, v);
#pragma unroll
                    for (uint32_t kg = 0; kg < 4; kg++) {
                        uint32_t w[4];
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const uint32_t j = kg * 8 + 2 * e;
                            w[e] = pack_bf16(fmaxf(v[j] + bias[c0 + j], 0.0f), fmaxf(v[j + 1] + bias[c0 + j + 1], 0.0f));
                        }
                        *reinterpret_cast<uint4*>(sm + tc::ACT + tc::off(row, c0 + kg * 8, tc::SBO_K128)) =
                            make_uint4(w[0], w[1], w[2], w[3]);
                    }
                }
            } else {
                float v[16];
                tc::ld16(lane_addr, v);
                if (r < n) {
#pragma unroll
                    for (uint32_t c = 0; c < (uint32_t)USED_OUT; c++) {
                        const float y = v[c] + sbias[3 * 128 + c];
                        Y[(size_t)r * USED_OUT + c] = y * snorm[NY_STD + c] + snorm[NY_MEAN + c];
                    }
                }
            }
        }
        // every lane's TMEM reads are done before the next tile's MMAs
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
    }
    if (!ok && t == 0) atomicCAS(status, 0u, (uint32_t)AVBD_FAIL_WAIT_TIMEOUT);
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tc::TMEM_COLS)
                     : "memory");
}

// ---------------------------------------------------------------------------
// Training GEMM on the tensor cores: C[M][N] (fp32) = op(A) op(B), BF16
// operands, FP32 accumulation in TMEM.  A is [M][K] (lda = K) or, with TA,
// stored [K][M]; B is [N][K] or, with TB, stored [K][N].  A CTA of four warps
// owns a 128-row x BN-column tile (BN = N rounded up to 16, at most 128;
// rows past M are zero): K runs in chunks of 64 through two shared-memory
// stages in the UMMA canonical K-major layout (row-group stride 1024 B),
// staged by all threads (transposing on the fly) while the previous chunk's
// four M = 128, K = 16 tcgen05.mma instructions run; each stage is reused
// only after the tcgen05.commit of its MMAs has arrived on its mbarrier.
// Every wait is bounded (one second); a timeout sets *status and the CTA
// frees its TMEM and stops.  Split-K writes one partial per z-slice
// (reduced in a fixed order by k_split_sum).
// ---------------------------------------------------------------------------
namespace tg {
constexpr uint32_t BK = 64, SBO = (BK / 8) * 128;          // chunk of K; row-group stride (1024 B)
constexpr uint32_t STAGE = 128 * BK * 2;                    // one operand tile (16 KiB)
constexpr uint32_t A0 = 0, B0 = A0 + 2 * STAGE, BAR = B0 + 2 * STAGE, TSLOT = BAR + 16, SMEM = TSLOT + 16;
constexpr uint32_t TMEM_COLS = 128;
}  // namespace tg

// one 8-element K group of row r of an operand tile: 16 bytes in the
// canonical layout; T: the operand is stored transposed ([K][rows], ld = rows)
template <bool T>
__device__ __forceinline__ uint4 stage_group(const bf16* __restrict__ X, uint32_t rows, uint32_t K, uint32_t row,
                                             uint32_t k, uint32_t kEnd) {
    uint32_t w[4];
    if (!T && row < rows && k + 8 <= kEnd && (K & 7u) == 0u)
        return *reinterpret_cast<const uint4*>(X + (size_t)row * K + k);
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const uint32_t k0 = k + 2 * e, k1 = k0 + 1;
        bf16 lo = __float2bfloat16(0.0f), hi = __float2bfloat16(0.0f);
        if (row < rows && k0 < kEnd) lo = T ? X[(size_t)k0 * rows + row] : X[(size_t)row * K + k0];
        if (row < rows && k1 < kEnd) hi = T ? X[(size_t)k1 * rows + row] : X[(size_t)row * K + k1];
        w[e] = (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(128) k_gemm_tc(const bf16* __restrict__ A, const bf16* __restrict__ B,
                                                 float* __restrict__ C, uint32_t M, uint32_t N, uint32_t K,
                                                 uint32_t kPerSplit, uint32_t bn, uint32_t* status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const uint32_t t = threadIdx.x, warp = t >> 5;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    const uint32_t m0 = blockIdx.y * 128u, n0 = blockIdx.x * bn;
    const uint32_t kBeg = blockIdx.z * kPerSplit, kEnd = min(K, kBeg + kPerSplit);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sbase + tg::BAR) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sbase + tg::BAR + 8) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + tg::TSLOT),
                     "r"(tg::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + tg::TSLOT);
    const uint32_t id = tc::idesc(128, bn);
    const uint32_t chunks = kEnd > kBeg ? (kEnd - kBeg + tg::BK - 1) / tg::BK : 0u;
    bool ok = true;
    for (uint32_t c = 0; c < chunks && ok; c++) {
        const uint32_t buf = c & 1u, bar = sbase + tg::BAR + 8u * buf;
        if (c >= 2) {
            // the MMAs that last read this stage have completed (block-uniform)
            ok = __syncthreads_and(tc::wait(bar, ((c >> 1) - 1u) & 1u) ? 1 : 0) != 0;
            if (!ok) break;
        }
        const uint32_t k0 = kBeg + c * tg::BK;
        unsigned char* sa = sm + tg::A0 + buf * tg::STAGE;
        unsigned char* sb = sm + tg::B0 + buf * tg::STAGE;
        // thread t stages row t of the A tile and (t < bn) row t of the B tile
#pragma unroll 2
        for (uint32_t kg = 0; kg < tg::BK / 8; kg++) {
            *reinterpret_cast<uint4*>(sa + tc::off(t, kg * 8, tg::SBO)) =
                stage_group<TA>(A, M, K, m0 + t, k0 + kg * 8, kEnd);
            if (t < bn)
                *reinterpret_cast<uint4*>(sb + tc::off(t, kg * 8, tg::SBO)) =
                    stage_group<TB>(B, N, K, n0 + t, k0 + kg * 8, kEnd);
        }
        tc::fence_proxy();               // generic-proxy writes, read by the tensor core
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        if (t == 0) {
            const uint32_t steps = min(tg::BK, kEnd - k0 + 15u) / 16u;
            const uint32_t a = sbase + tg::A0 + buf * tg::STAGE, b = sbase + tg::B0 + buf * tg::STAGE;
            for (uint32_t s = 0; s < steps; s++)
                tc::mma(tmem, tc::desc(a + 256u * s, tg::SBO), tc::desc(b + 256u * s, tg::SBO), id,
                        (c > 0 || s > 0) ? 1u : 0u);
            tc::commit(bar);
        }
    }
    if (ok && chunks) {
        // the last commit covers every MMA issued before it
        const uint32_t last = chunks - 1u;
        ok = __syncthreads_and(tc::wait(sbase + tg::BAR + 8u * (last & 1u), (last >> 1) & 1u) ? 1 : 0) != 0;
        tc::fence_after();
    }
    if (ok) {
        const uint32_t r = m0 + t;
        const uint32_t lane_addr = tmem + ((warp * 32u) << 16);
        float* Cz = C + (size_t)blockIdx.z * M * N;
        for (uint32_t c0 = 0; c0 < bn; c0 += 16) {
            float v[16];
            if (chunks) {
                tc::ld16(lane_addr + c0, v);
            } else {
#pragma unroll
                for (int j = 0; j < 16; j++) v[j] = 0.0f;
            }
            if (r < M) {
#pragma unroll
                for (uint32_t j = 0; j < 16; j++)
                    if (n0 + c0 + j < N) Cz[(size_t)r * N + n0 + c0 + j] = v[j];
            }
        }
    } else if (t == 0) {
        atomicCAS(status, 0u, (uint32_t)AVBD_FAIL_WAIT_TIMEOUT);
    }
    if (!ok) {
        // let MMAs still in flight finish (bounded) before the TMEM is freed
        for (uint32_t b = 0; b < 2; b++) tc::wait(sbase + tg::BAR + 8u * b, 0u);
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tg::TMEM_COLS)
                     : "memory");
}

__global__ void k_split_sum(const float* part, uint32_t splits, uint32_t count, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float s = 0.0f;
    for (uint32_t z = 0; z < splits; z++) s += part[(size_t)z * count + i];
    out[i] = s;
}

// H = bf16(relu(Z + b)) for Z [rows][cols]
__global__ void k_bias_relu(const float* Z, const float* b, uint32_t rows, uint32_t cols, bf16* H) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    H[i] = __float2bfloat16(fmaxf(Z[i] + b[i % cols], 0.0f));
}

// normalised inputs as BF16 [rows][16]
__global__ void k_norm_input(const float* X, const float* norm, uint32_t rows, bf16* Xb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * mlp::DIN) return;
    const uint32_t c = i % mlp::DIN;
    Xb[i] = __float2bfloat16((X[i] - norm[mlp::NX_MEAN + c]) * norm[mlp::NX_INV + c]);
}

// Output layer and loss: Y = Z + b4; dY = 2 (Y - Tn) / rows on the used
// columns (Tn: targets normalised by ymean, ystd), 0 elsewhere; loss sums.
__global__ void k_loss_grad(const float* Z, const float* b4, const float* T, const float* norm, uint32_t rows,
                            float* dY, bf16* dYb, float* lossPart) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < rows * mlp::DOUT) {
        const uint32_t r = i / mlp::DOUT, c = i % mlp::DOUT;
        float g = 0.0f;
        if (c < (uint32_t)mlp::USED_OUT) {
            const float y = Z[i] + b4[c];
            const float t = (T[r * mlp::USED_OUT + c] - norm[mlp::NY_MEAN + c]) / norm[mlp::NY_STD + c];
            const float e = y - t;
            l = e * e;
            g = 2.0f * e / (float)rows;
        }
        dY[i] = g;
        dYb[i] = __float2bfloat16(g);
    }
    // block sum of the squared errors (fixed order)
    __shared__ float red[256];
    red[threadIdx.x] = l;
    __syncthreads();
    for (uint32_t w = blockDim.x >> 1; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) lossPart[blockIdx.x] = red[0];
}

// dH = bf16(G * (H > 0)), G fp32 [rows][cols]; also keeps fp32 for bias sums
__global__ void k_relu_back(const float* G, const bf16* H, uint32_t n, float* dH, bf16* dHb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = __bfloat162float(H[i]) > 0.0f ? G[i] : 0.0f;
    dH[i] = v;
    dHb[i] = __float2bfloat16(v);
}

// column sums of G [rows][cols] in a fixed order (one thread per column)
__global__ void k_col_sum(const float* G, uint32_t rows, uint32_t cols, float* out) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (uint32_t r = 0; r < rows; r++) s += G[(size_t)r * cols + c];
    out[c] = s;
}

// fixed-order sum of n values, times `scale`
__global__ void k_fixed_sum(const float* v, uint32_t n, float scale, float* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float s = 0.0f;
    for (uint32_t i = 0; i < n; i++) s += v[i];
    *out = s * scale;
}

// Adam on the fp32 parameters; refreshes the BF16 weight mirror.
__global__ void k_adam(float* prm, const float* grad, float* m, float* v, uint32_t step, float lr, float b1,
                       float b2, float eps, bf16* half) {
    using namespace mlp;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NPARAM) return;
    const float gi = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.0f - powf(b1, (float)step));
    const float vh = vi / (1.0f - powf(b2, (float)step));
    const float p = prm[i] - lr * mh / (sqrtf(vh) + eps);
    prm[i] = p;
    int h = -1;
    if (i < OB1) h = (int)(HW1 + i);
    else if (i >= OW2 && i < OB2) h = (int)(HW2 + i - OW2);
    else if (i >= OW3 && i < OB3) h = (int)(HW3 + i - OW3);
    else if (i >= OW4 && i < OB4) h = (int)(HW4 + i - OW4);
    if (h >= 0) half[h] = __float2bfloat16(p);
}

__global__ void k_mirror(const float* prm, bf16* half) {
    using namespace mlp;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NPARAM) return;
    int h = -1;
    if (i < OB1) h = (int)(HW1 + i);
    else if (i >= OW2 && i < OB2) h = (int)(HW2 + i - OW2);
    else if (i >= OW3 && i < OB3) h = (int)(HW3 + i - OW3);
    else if (i >= OW4 && i < OB4) h = (int)(HW4 + i - OW4);
    if (h >= 0) half[h] = __float2bfloat16(prm[i]);
}

// BF16 weight image of the inference kernel: W1..W4 in the UMMA canonical
// K-major layout, byte for byte the kernel's shared-memory weight region.
__global__ void k_mirror_umma(const float* prm, unsigned char* img) {
    using namespace mlp;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NHALF) return;
    uint32_t src, base, cols, sbo, j;
    if (i < HW2) { j = i - HW1; src = OW1; base = tc::W1; cols = DIN; sbo = tc::SBO_K32; }
    else if (i < HW3) { j = i - HW2; src = OW2; base = tc::W2; cols = HID; sbo = tc::SBO_K128; }
    else if (i < HW4) { j = i - HW3; src = OW3; base = tc::W3; cols = HID; sbo = tc::SBO_K128; }
    else { j = i - HW4; src = OW4; base = tc::W4; cols = HID; sbo = tc::SBO_K128; }
    const uint32_t r = j / cols, k = j % cols;
    *reinterpret_cast<bf16*>(img + base + tc::off(r, k, sbo)) = __float2bfloat16(prm[src + j]);
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side of training (forward with saved activations, backward, Adam).
// Workspace layout for a batch of B rows (all offsets 256-byte aligned).
// ---------------------------------------------------------------------------
namespace {
constexpr uint32_t kSplits = 32;
struct Work {
    bf16 *Xb, *H1, *H2, *H3, *dYb, *dH3b, *dH2b, *dH1b, *half;
    float *Z, *dY, *dH, *part, *grad, *lossPart;
    uint32_t* status;        // nonzero when a tensor-core wait gave up
};
size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
size_t work_layout(uint32_t B, char* base, Work* w) {
    using namespace mlp;
    size_t off = 0;
    auto take = [&](size_t bytes) { char* p = base ? base + off : nullptr; off += align256(bytes); return p; };
    const size_t Bp = (size_t)B;
    char* p;
    p = take(Bp * DIN * 2); if (w) w->Xb = (bf16*)p;
    p = take(Bp * HID * 2); if (w) w->H1 = (bf16*)p;
    p = take(Bp * HID * 2); if (w) w->H2 = (bf16*)p;
    p = take(Bp * HID * 2); if (w) w->H3 = (bf16*)p;
    p = take(Bp * DOUT * 2); if (w) w->dYb = (bf16*)p;
    p = take(Bp * HID * 2); if (w) w->dH3b = (bf16*)p;
    p = take(Bp * HID * 2); if (w) w->dH2b = (bf16*)p;
    p = take(Bp * HID * 2); if (w) w->dH1b = (bf16*)p;
    p = take((size_t)NHALF * 2); if (w) w->half = (bf16*)p;
    p = take(Bp * HID * 4); if (w) w->Z = (float*)p;
    p = take(Bp * DOUT * 4); if (w) w->dY = (float*)p;
    p = take(Bp * HID * 4); if (w) w->dH = (float*)p;
    p = take((size_t)kSplits * HID * HID * 4); if (w) w->part = (float*)p;
    p = take((size_t)NPARAM * 4); if (w) w->grad = (float*)p;
    p = take(((Bp * DOUT + 255) / 256) * 4 + 4); if (w) w->lossPart = (float*)p;
    p = take(4); if (w) w->status = (uint32_t*)p;
    return off;
}

// 64 KiB of dynamic shared memory for the two stages (set once per device)
template <bool TA, bool TB>
void gemm_attributes() {
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load() & bit) return;
    cudaFuncSetAttribute(k_gemm_tc<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tg::SMEM);
    done.fetch_or(bit);
}

template <bool TA, bool TB>
void launch_gemm_tc(dim3 grid, const bf16* A, const bf16* B, float* dst, uint32_t M, uint32_t N, uint32_t K,
                    uint32_t kPer, uint32_t bn, uint32_t* status, cudaStream_t st) {
    gemm_attributes<TA, TB>();
    k_gemm_tc<TA, TB><<<grid, 128, tg::SMEM, st>>>(A, B, dst, M, N, K, kPer, bn, status);
}

void gemm(const bf16* A, bool ta, const bf16* B, bool tb, float* C, uint32_t M, uint32_t N, uint32_t K,
          uint32_t splits, float* part, uint32_t* status, cudaStream_t st) {
    const uint32_t kPer = ((K + splits - 1) / splits + 63) / 64 * 64;
    splits = (K + kPer - 1) / kPer;
    // 64-column tiles: two column blocks for the 128-wide layers (more CTAs
    // for the batch-row GEMMs, which have only 64 row blocks at batch 8,192)
    const uint32_t bn = std::min<uint32_t>(64u, (N + 15u) / 16u * 16u);
    dim3 grid((N + bn - 1) / bn, (M + 127) / 128, splits);
    float* dst = splits > 1 ? part : C;
    if (!ta && !tb) launch_gemm_tc<false, false>(grid, A, B, dst, M, N, K, kPer, bn, status, st);
    else if (!ta && tb) launch_gemm_tc<false, true>(grid, A, B, dst, M, N, K, kPer, bn, status, st);
    else if (ta && !tb) launch_gemm_tc<true, false>(grid, A, B, dst, M, N, K, kPer, bn, status, st);
    else launch_gemm_tc<true, true>(grid, A, B, dst, M, N, K, kPer, bn, status, st);
    if (splits > 1) k_split_sum<<<(M * N + 255) / 256, 256, 0, st>>>(part, splits, M * N, C);
}

inline uint32_t blocks(size_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

// Forward with saved activations, loss and full gradient into w.grad.
void forward_backward(const float* prm, const float* norm, const float* X, const float* T, uint32_t B, Work& w,
                      cudaStream_t st) {
    using namespace mlp;
    k_mirror<<<blocks(NPARAM, 256), 256, 0, st>>>(prm, w.half);
    k_norm_input<<<blocks((size_t)B * DIN, 256), 256, 0, st>>>(X, norm, B, w.Xb);
    // forward: Z = Hprev W^T (W stored [out][in] = [N][K])
    gemm(w.Xb, false, w.half + HW1, false, w.Z, B, HID, DIN, 1, w.part, w.status, st);
    k_bias_relu<<<blocks((size_t)B * HID, 256), 256, 0, st>>>(w.Z, prm + OB1, B, HID, w.H1);
    gemm(w.H1, false, w.half + HW2, false, w.Z, B, HID, HID, 1, w.part, w.status, st);
    k_bias_relu<<<blocks((size_t)B * HID, 256), 256, 0, st>>>(w.Z, prm + OB2, B, HID, w.H2);
    gemm(w.H2, false, w.half + HW3, false, w.Z, B, HID, HID, 1, w.part, w.status, st);
    k_bias_relu<<<blocks((size_t)B * HID, 256), 256, 0, st>>>(w.Z, prm + OB3, B, HID, w.H3);
    gemm(w.H3, false, w.half + HW4, false, w.Z, B, DOUT, HID, 1, w.part, w.status, st);
    const uint32_t lb = blocks((size_t)B * DOUT, 256);
    k_loss_grad<<<lb, 256, 0, st>>>(w.Z, prm + OB4, T, norm, B, w.dY, w.dYb, w.lossPart);
    k_fixed_sum<<<1, 32, 0, st>>>(w.lossPart, lb, 1.0f / (float)B, w.lossPart + lb);   // mean over the batch
    // backward.  dW = dH^T Hprev: A = dH stored [B][out] = [K][M] (TA),
    // B-operand = Hprev stored [B][in] = [K][N] (TB).  dHprev = dH W:
    // A = dH [B][out] = [M][K], B-operand W stored [out][in] = [K][N] (TB).
    gemm(w.dYb, true, w.H3, true, w.grad + OW4, DOUT, HID, B, kSplits, w.part, w.status, st);
    k_col_sum<<<1, DOUT, 0, st>>>(w.dY, B, DOUT, w.grad + OB4);
    gemm(w.dYb, false, w.half + HW4, true, w.Z, B, HID, DOUT, 1, w.part, w.status, st);
    k_relu_back<<<blocks((size_t)B * HID, 256), 256, 0, st>>>(w.Z, w.H3, B * HID, w.dH, w.dH3b);
    k_col_sum<<<1, HID, 0, st>>>(w.dH, B, HID, w.grad + OB3);
    gemm(w.dH3b, true, w.H2, true, w.grad + OW3, HID, HID, B, kSplits, w.part, w.status, st);
    gemm(w.dH3b, false, w.half + HW3, true, w.Z, B, HID, HID, 1, w.part, w.status, st);
    k_relu_back<<<blocks((size_t)B * HID, 256), 256, 0, st>>>(w.Z, w.H2, B * HID, w.dH, w.dH2b);
    k_col_sum<<<1, HID, 0, st>>>(w.dH, B, HID, w.grad + OB2);
    gemm(w.dH2b, true, w.H1, true, w.grad + OW2, HID, HID, B, kSplits, w.part, w.status, st);
    gemm(w.dH2b, false, w.half + HW2, true, w.Z, B, HID, HID, 1, w.part, w.status, st);
    k_relu_back<<<blocks((size_t)B * HID, 256), 256, 0, st>>>(w.Z, w.H1, B * HID, w.dH, w.dH1b);
    k_col_sum<<<1, HID, 0, st>>>(w.dH, B, HID, w.grad + OB1);
    gemm(w.dH1b, true, w.Xb, true, w.grad + OW1, HID, DIN, B, kSplits, w.part, w.status, st);
}
}  // namespace

// ---------------------------------------------------------------------------
// Solver integration
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ float step_scale(const Params& P) { return fmaxf(fabsf(P.gravity), 1.0f) * P.dt * P.dt; }

// bounding radius of a rigid body (the rotation's length scale)
__device__ __forceinline__ float learn_radius(const DevPtrs& d, uint32_t v) { return fmaxf(d.shape[v].w, 1e-6f); }

// Pose of learned row i moved by its prediction y from the plain warm start
// (xp, qp).  A zero rotation prediction keeps qp bit for bit.
__device__ __forceinline__ void learn_pose(const Params& P, const DevPtrs& d, uint32_t i, uint32_t v, float4 xp,
                                           float4 qp, float4& x, float4& q) {
    const float s = step_scale(P);
    const float* y = d.learnPred + (size_t)i * mlp::USED_OUT;
    x = mk4(xyz(xp) + mk3(y[0], y[1], y[2]) * s, xp.w);
    q = qp;
    if (i >= P.learnParticles && (y[3] != 0.0f || y[4] != 0.0f || y[5] != 0.0f))
        q = q_addw(qp, mk3(y[3], y[4], y[5]) * (s / learn_radius(d, v)));
}

// Per-vertex features at the plain warm start (see the file comment).  The
// contact features walk the body's per-frame segment (manifolds, element
// contacts), the stiffness feature its static segments (springs; tets,
// membranes, bends).
// Contact state of every learned vertex: count of contact points, closest
// gap and summed oriented normal of its manifolds and element contacts.
__global__ void k_learn_contacts(const Params P, const DevPtrs d, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t v = d.learnIdx[i];
    float count = 0.0f, gap = 1e30f;
    float3 nsum = s3(0);
    const uint32_t ds = d.dynStart[v], dc = d.dynCount[v];
    for (uint32_t k = 0; k < dc; k++) {
        const uint32_t e = d.dynList[ds + k];
        const uint32_t kind = e >> ADJ_KIND_SHIFT;
        if (kind == FK_MANIFOLD) {
            const ManifoldGPU& m = d.manifolds[e & ADJ_INDEX_MASK];
            const float sg = m.header.x == v ? 1.0f : -1.0f;
            nsum += xyz(m.basisN) * sg;
            for (uint32_t c = 0; c < m.header.z; c++) {
                count += 1.0f;
                gap = fminf(gap, m.contacts[c].C0.x);
            }
        } else if (kind == FK_SOFT) {
            // element contact: the vertex's side of the stencil gives the sign
            const SoftContactGPU& sc = d.soft[e & ADJ_INDEX_MASK];
            const float w = sc.ids.x == v ? sc.weights.x : (sc.ids.y == v ? sc.weights.y
                                                            : (sc.ids.z == v ? sc.weights.z : sc.weights.w));
            nsum += xyz(sc.normal) * (w >= 0.0f ? 1.0f : -1.0f);
            count += 1.0f;
            gap = fminf(gap, sc.C0.x);
        }
    }
    d.learnStat[i] = mk4(nsum, count);
    d.learnGap[i] = gap;
}

// Features of every learned vertex.  The static parts (incident stiffness,
// the 1-ring of vertices sharing a tet or spring with its multiplicities)
// are precomputed at upload; the ring's contact state sums the neighbours'
// contact counts (times their multiplicity) and takes their closest gap.
__global__ void k_learn_features(const Params P, const DevPtrs d, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t v = d.learnIdx[i];
    const float s = step_scale(P);
    const float4 pl = d.posLin[v];
    const float3 x0 = xyz(d.initLin[v]);
    const float3 fi = (xyz(d.inertLin[v]) - x0) / s;
    const float3 fp = (xyz(pl) - x0) / s;
    const float3 fv = xyz(d.prevVelLin[v]) * (P.dt / s);
    const float4 st = d.learnStat[i];
    const float3 nsum = xyz(st);
    const float count = st.w, gap = d.learnGap[i];
    const float stiff = d.learnStiff[i];
    const float ringN = d.learnRingN[i];
    float ringContacts = 0.0f, ringGap = 1e30f;
    const uint32_t r1 = d.learnRingStart[i + 1];
    for (uint32_t k = d.learnRingStart[i]; k < r1; k++) {
        const uint2 e = d.learnRing[k];
        ringContacts += d.learnStat[e.x].w * (float)e.y;
        ringGap = fminf(ringGap, d.learnGap[e.x]);
    }
    const float inv = ringN > 0.0f ? 1.0f / ringN : 0.0f;
    float* f = d.learnFeat + (size_t)i * mlp::DIN;
    for (int k = 16; k < 25; k++) f[k] = 0.0f;          // rigid slots, reserved
    if (i >= P.learnParticles) {
        const float r = learn_radius(d, v);
        const float4 q = d.posAng[v];
        const float3 wq = q_sub(q, d.initAng[v]) * (r / s);
        const float3 up = q_rotate(q_conj(q), mk3(0, 0, 1));
        f[16] = 1.0f;
        f[17] = wq.x; f[18] = wq.y; f[19] = wq.z;
        f[20] = up.x; f[21] = up.y; f[22] = up.z;
        f[23] = 0.1f * log1pf(r / s);
    }
    f[25] = ringN * 0.1f;
    f[26] = ringContacts * inv * 0.25f;
    f[27] = ringContacts > 0.0f ? fminf(fmaxf(ringGap / s, -10.0f), 10.0f) : 10.0f;
    f[28] = 0.0f; f[29] = 0.0f; f[30] = 0.0f; f[31] = 0.0f;
    if (i >= P.learnParticles) {
        // position-PD hinge motors acting on the body (they are in its
        // static segment): the rotation each asks for, and their gains
        const float r = learn_radius(d, v);
        const uint4 sg = d.staticSeg[v];
        float motors = 0.0f, gain = 0.0f;
        float3 want = s3(0.0f);
        for (uint32_t k = 0; k < sg.y; k++) {
            const uint32_t e = d.preList[sg.x + k];
            if ((e >> ADJ_KIND_SHIFT) != FK_JOINT) continue;
            const JointGPU& j = d.joints[e & ADJ_INDEX_MASK];
            const uint32_t mode = j.header.w & MOTOR_MODE_MASK;
            if (!(j.motor.y > 0.0f) || j.hingeAxis.w == 0.0f || mode == MOTOR_EXPLICIT || mode == MOTOR_VELOCITY)
                continue;
            const uint32_t a = j.header.x, b = j.header.y;
            const float4 qA = a == WORLD_BODY ? make_float4(0, 0, 0, 1) : d.posAng[a];
            const float4 qB = d.posAng[b];
            const float3 axis = xyz(j.hingeAxis);
            const float Cm = wrap_pi(twist_angle(q_mul(qA, tof(j.restRel)), qB, axis) - j.motor.x);
            want += q_rotate(qB, axis) * (v == a ? Cm : -Cm);
            motors += 1.0f;
            gain += j.motor.w;
        }
        const float3 w = want * (r / s);
        f[24] = motors * 0.25f;
        f[28] = w.x; f[29] = w.y; f[30] = w.z;
        f[31] = log1pf(gain * P.dt * P.dt / fmaxf(pl.w * r * r, 1e-12f));
    }
    f[0] = fi.x; f[1] = fi.y; f[2] = fi.z;
    f[3] = fp.x; f[4] = fp.y; f[5] = fp.z;
    f[6] = fv.x; f[7] = fv.y; f[8] = fv.z;
    f[9] = count * 0.25f;
    f[10] = nsum.x; f[11] = nsum.y; f[12] = nsum.z;
    f[13] = count > 0.0f ? fminf(fmaxf(gap / s, -10.0f), 10.0f) : 10.0f;
    f[14] = log1pf(stiff * P.dt * P.dt / fmaxf(pl.w, 1e-12f));
    f[15] = 1.0f;
}

// x0 = x_plain + s * prediction for every learned row
__global__ void k_learn_apply(const Params P, const DevPtrs d, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t v = d.learnIdx[i];
    learn_pose(P, d, i, v, d.learnSaveLin[v], d.learnSaveAng[v], d.posLin[v], d.posAng[v]);
}

// keep the prediction when its residual after the trial sweeps is no worse
__global__ void k_learn_select(const Params P, const DevPtrs d, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool accept = d.learnResid[1] <= d.learnResid[0];
    if (i == 0 && accept) atomicAdd(d.learnAccepted, 1u);
    if (i >= n || !accept) return;
    const uint32_t v = d.learnIdx[i];
    learn_pose(P, d, i, v, d.learnSaveLin[v], d.learnSaveAng[v], d.posLin[v], d.posAng[v]);
}

// Pose buffers of the predicted branch: the solver's pose with every
// learned row (the first n slots) moved by its prediction.
__global__ void k_learn_branch(const Params P, const DevPtrs d, uint32_t nb, uint32_t n) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const uint32_t slot = d.learnSlot[b];
    if (slot < n) {
        learn_pose(P, d, slot, b, d.posLin[b], d.posAng[b], d.learnSweptLin[b], d.learnSweptAng[b]);
    } else {
        d.learnSweptLin[b] = d.posLin[b];
        d.learnSweptAng[b] = d.posAng[b];
    }
}

// After both trial sweeps: adopt the predicted branch's swept pose when its
// residual is no worse; otherwise the plain branch's pose stays.
__global__ void k_learn_adopt(const Params P, const DevPtrs d, uint32_t nb) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    const bool accept = d.learnResid[1] <= d.learnResid[0];
    if (b == 0 && accept) atomicAdd(d.learnAccepted, 1u);
    // the kept trial sweep is the first pass: its OGC bound-exceeder count
    // moves to the first pass's slot
    if (b == 0 && P.ogc) d.counters->ogcSlots[0] = d.counters->ogcSlots[accept ? 3 : 2];
    if (b >= nb || !accept) return;
    d.posLin[b] = d.learnSweptLin[b];
    d.posAng[b] = d.learnSweptAng[b];
}

// training target: the solve's correction of the plain warm start (the
// rotation part zero for particles)
__global__ void k_learn_target(const Params P, const DevPtrs d, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t v = d.learnIdx[i];
    const float s = step_scale(P);
    const float3 t = (xyz(d.posLin[v]) - xyz(d.learnSaveLin[v])) / s;
    const float3 w = i >= P.learnParticles ? q_sub(d.posAng[v], d.learnSaveAng[v]) * (learn_radius(d, v) / s)
                                           : s3(0.0f);
    float* y = d.learnTarget + (size_t)i * mlp::USED_OUT;
    y[0] = t.x; y[1] = t.y; y[2] = t.z;
    y[3] = w.x; y[4] = w.y; y[5] = w.z;
}

__global__ void k_copy_double(const double* src, double* dst) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = *src;
}

}  // namespace

void launch_learn_features(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    if (!z.numLearn) return;
    k_learn_contacts<<<(z.numLearn + 127) / 128, 128, 0, st>>>(P, d, z.numLearn);
    k_learn_features<<<(z.numLearn + 127) / 128, 128, 0, st>>>(P, d, z.numLearn);
}
void launch_learn_apply(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    if (z.numLearn) k_learn_apply<<<(z.numLearn + 127) / 128, 128, 0, st>>>(P, d, z.numLearn);
}
void launch_learn_select(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    k_learn_select<<<(z.numLearn + 128) / 128, 128, 0, st>>>(P, d, z.numLearn);
}
void launch_learn_branch(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    k_learn_branch<<<(z.numBodies + 127) / 128, 128, 0, st>>>(P, d, z.numBodies, z.numLearn);
}
void launch_learn_adopt(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    k_learn_adopt<<<(z.numBodies + 127) / 128, 128, 0, st>>>(P, d, z.numBodies);
}
void launch_learn_target(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    if (z.numLearn) k_learn_target<<<(z.numLearn + 127) / 128, 128, 0, st>>>(P, d, z.numLearn);
}
void launch_copy_double(const double* src, double* dst, cudaStream_t st) { k_copy_double<<<1, 32, 0, st>>>(src, dst); }

// weights, one activation tile, biases and normalisation: 110 KiB of shared
// memory (set once per device)
static void mlp_infer_attributes() {
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load() & bit) return;
    cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM);
    done.fetch_or(bit);
}

void launch_mlp_infer(const void* halfW, const float* prm, const float* norm, const float* X, uint32_t n, float* Y,
                      uint32_t* status, cudaStream_t st) {
    if (n == 0) return;
    mlp_infer_attributes();
    // two CTAs per SM (110 KiB of shared memory and 128 TMEM columns each),
    // every CTA walking 128-row tiles
    const uint32_t tiles = (n + tc::ROWS - 1) / tc::ROWS;
    const uint32_t blocks = std::min<uint32_t>(tiles, 2u * 148u);
    k_mlp_infer_tc<<<blocks, 128, tc::SMEM, st>>>(static_cast<const bf16*>(halfW), prm, norm, X, n, Y, status);
}

void launch_mlp_mirror(const float* prm, void* halfW, cudaStream_t st) {
    k_mirror_umma<<<blocks(mlp::NHALF, 256), 256, 0, st>>>(prm, static_cast<unsigned char*>(halfW));
}

uint32_t mlp_param_count() { return mlp::NPARAM; }
uint32_t mlp_half_count() { return mlp::NHALF; }
uint32_t mlp_norm_count() { return mlp::NNORM; }

}  // namespace avbd

// ---------------------------------------------------------------------------
// C ABI of the training kernels (no counterpart in the reference: the learned
// warm start is new).  Every pointer is device memory; `stream` is a
// cudaStream_t or null.
// ---------------------------------------------------------------------------
using namespace avbd;
extern "C" {

uint32_t avbd_mlp_param_count(void) { return mlp::NPARAM; }

size_t avbd_mlp_workspace_bytes(uint32_t batch) { return work_layout(batch, nullptr, nullptr); }

// status word of a workspace: cleared, or read after a synchronisation
static int workspace_status(const Work& w, cudaStream_t st) {
    uint32_t h = 0;
    if (cudaMemcpyAsync(&h, w.status, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return AVBD_ERR_RUNTIME_FAILURE;
    return h == 0 ? AVBD_OK : AVBD_ERR_RUNTIME_FAILURE;
}

static int gradients(const float* params, const float* norm, const float* features, const float* targets,
                     uint32_t batch, void* workspace, float* grad_out, float* loss_out, cudaStream_t st,
                     bool check) {
    if (!params || !norm || !features || !targets || !workspace || batch == 0) return AVBD_ERR_INVALID_ARGUMENT;
    Work w{};
    work_layout(batch, static_cast<char*>(workspace), &w);
    if (check) cudaMemsetAsync(w.status, 0, sizeof(uint32_t), st);
    forward_backward(params, norm, features, targets, batch, w, st);
    const uint32_t lb = blocks((size_t)batch * mlp::DOUT, 256);
    if (grad_out) cudaMemcpyAsync(grad_out, w.grad, sizeof(float) * mlp::NPARAM, cudaMemcpyDeviceToDevice, st);
    if (loss_out) cudaMemcpyAsync(loss_out, w.lossPart + lb, sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (cudaGetLastError() != cudaSuccess) return AVBD_ERR_RUNTIME_FAILURE;
    // a tensor-core wait that gave up fails the call (the GEMM kernels latch
    // it in the workspace's status word)
    return check ? workspace_status(w, st) : AVBD_OK;
}

int avbd_mlp_gradients(const float* params, const float* norm, const float* features, const float* targets,
                       uint32_t batch, void* workspace, float* grad_out, float* loss_out, void* stream) {
    return gradients(params, norm, features, targets, batch, workspace, grad_out, loss_out,
                     static_cast<cudaStream_t>(stream), true);
}

int avbd_mlp_workspace_status(const void* workspace, uint32_t batch, void* stream) {
    if (!workspace || batch == 0) return AVBD_ERR_INVALID_ARGUMENT;
    Work w{};
    work_layout(batch, static_cast<char*>(const_cast<void*>(workspace)), &w);
    return workspace_status(w, static_cast<cudaStream_t>(stream));
}

int avbd_mlp_train_step(float* params, const float* norm, const float* features, const float* targets,
                        uint32_t batch, float* adam_m, float* adam_v, uint32_t step, float lr, void* workspace,
                        float* loss_out, void* stream) {
    if (!params || !adam_m || !adam_v || step == 0) return AVBD_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Work w{};
    if (workspace && batch) {
        work_layout(batch, static_cast<char*>(workspace), &w);
        if (step == 1) cudaMemsetAsync(w.status, 0, sizeof(uint32_t), st);   // sticky from here on
    }
    int rc = gradients(params, norm, features, targets, batch, workspace, nullptr, loss_out, st, false);
    if (rc != AVBD_OK) return rc;
    k_adam<<<blocks(mlp::NPARAM, 256), 256, 0, st>>>(params, w.grad, adam_m, adam_v, step, lr, 0.9f, 0.999f, 1e-8f,
                                                     w.half);
    return cudaGetLastError() == cudaSuccess ? AVBD_OK : AVBD_ERR_RUNTIME_FAILURE;
}

static int mlp_infer(const float* params, const float* norm, const float* features, uint32_t n, float* out,
                     void* workspace, void* stream, bool issue) {
    if (!params || !norm || !features || !out || !workspace) return AVBD_ERR_INVALID_ARGUMENT;
    // bulk copies and vector loads read the weight image, the biases, the
    // normalisation block and the feature rows in 16-byte units
    if ((reinterpret_cast<uintptr_t>(workspace) | reinterpret_cast<uintptr_t>(features) |
         reinterpret_cast<uintptr_t>(params) | reinterpret_cast<uintptr_t>(norm)) & 15u)
        return AVBD_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the BF16 weight mirror, then the kernel's status word
    uint32_t* status = reinterpret_cast<uint32_t*>(static_cast<char*>(workspace) +
                                                   ((sizeof(bf16) * mlp::NHALF + 255) / 256) * 256);
    cudaMemsetAsync(status, 0, sizeof(uint32_t), st);
    launch_mlp_mirror(params, workspace, st);
    if (issue) {
        launch_mlp_infer(workspace, params, norm, features, n, out, status, st);
    } else if (n) {
        mlp_infer_attributes();
        k_mlp_infer_tc<<<1, 128, tc::SMEM, st>>>(static_cast<const bf16*>(workspace), params, norm, features, n, out,
                                                 status, false);
    }
    uint32_t h = 0;
    if (cudaMemcpyAsync(&h, status, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return AVBD_ERR_RUNTIME_FAILURE;
    return h == 0 ? AVBD_OK : AVBD_ERR_RUNTIME_FAILURE;
}

int avbd_mlp_infer(const float* params, const float* norm, const float* features, uint32_t n, float* out,
                   void* workspace, void* stream) {
    return mlp_infer(params, norm, features, n, out, workspace, stream, true);
}

int avbd_mlp_infer_wait_timeout_for_testing(const float* params, const float* norm, const float* features,
                                            uint32_t n, float* out, void* workspace, void* stream) {
    return mlp_infer(params, norm, features, n, out, workspace, stream, false);
}

}  // extern "C"
