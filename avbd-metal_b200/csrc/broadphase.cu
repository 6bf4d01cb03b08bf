// broadphase.cu — exclusive scan, counting-sort spatial hash and
// deterministic candidate-pair generation.
//
// Follows Shaders/10_scan.metal and Shaders/20_broadphase.metal:69-131,
// :287-512.  The hash grid is a counting sort (count -> scan -> scatter ->
// per-bucket sort by collider id); pairs are produced in two passes (count
// per producer, scan, emit in producer/cell order) so the pair list — and
// with it the manifold index of every pair — is the same on every run.
#include <mutex>

#include "../../include/avbd.h"
#include "dmath.cuh"
#include "kernels.h"

namespace avbd {

// ---------------------------------------------------------------------------
// Exclusive scan: 1024 words per block (256 threads x 4), a single-block scan
// of the block sums, then a uniform add.
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_GRAIN = 4;
constexpr int SCAN_BLOCK = SCAN_THREADS * SCAN_GRAIN;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warpSums,
                                                         uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t w = lane < nw ? warpSums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) warpSums[lane] = w;   // inclusive warp prefix
    }
    __syncthreads();
    uint32_t warpBase = warp > 0 ? warpSums[warp - 1] : 0u;
    total = warpSums[(blockDim.x >> 5) - 1];
    return warpBase + x - v;
}

__global__ void k_scan_blocks(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                              uint32_t* __restrict__ blockSums, uint32_t n) {
    __shared__ uint32_t warpSums[32];
    const uint32_t base = blockIdx.x * SCAN_BLOCK + threadIdx.x * SCAN_GRAIN;
    uint32_t v[SCAN_GRAIN];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_GRAIN; i++) {
        v[i] = base + i < n ? in[base + i] : 0u;
        sum += v[i];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, warpSums, total);
#pragma unroll
    for (int i = 0; i < SCAN_GRAIN; i++) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

__global__ void k_scan_block_sums(uint32_t* __restrict__ blockSums, uint32_t nblocks) {
    __shared__ uint32_t warpSums[32];
    // nblocks <= SCAN_BLOCK: each thread owns up to 4 consecutive sums
    const uint32_t base = threadIdx.x * SCAN_GRAIN;
    uint32_t v[SCAN_GRAIN];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_GRAIN; i++) {
        v[i] = base + i < nblocks ? blockSums[base + i] : 0u;
        sum += v[i];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, warpSums, total);
#pragma unroll
    for (int i = 0; i < SCAN_GRAIN; i++) {
        if (base + i < nblocks) blockSums[base + i] = run;
        run += v[i];
    }
}

__global__ void k_scan_add(uint32_t* __restrict__ out, const uint32_t* __restrict__ blockSums,
                           uint32_t n) {
    const uint32_t add = blockSums[blockIdx.x];
    const uint32_t base = blockIdx.x * SCAN_BLOCK + threadIdx.x * SCAN_GRAIN;
#pragma unroll
    for (int i = 0; i < SCAN_GRAIN; i++)
        if (base + i < n) out[base + i] += add;
}

void launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch,
                           cudaStream_t st) {
    if (n == 0) return;
    const uint32_t nblocks = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
    k_scan_blocks<<<nblocks, SCAN_THREADS, 0, st>>>(in, out, scratch, n);
    if (nblocks > 1) {
        k_scan_block_sums<<<1, SCAN_THREADS, 0, st>>>(scratch, nblocks);
        k_scan_add<<<nblocks, SCAN_THREADS, 0, st>>>(out, scratch, n);
    }
}

// Any n < 2^30: scan blocks of 1024, scan the block sums recursively in
// place (each thread reads its words before writing them), add back.
void launch_exclusive_scan_large(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch,
                                 cudaStream_t st) {
    if (n == 0) return;
    const uint32_t nblocks = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
    k_scan_blocks<<<nblocks, SCAN_THREADS, 0, st>>>(in, out, scratch, n);
    if (nblocks > 1) {
        launch_exclusive_scan_large(scratch, scratch, nblocks, scratch + nblocks, st);
        k_scan_add<<<nblocks, SCAN_THREADS, 0, st>>>(out, scratch, n);
    }
}

size_t scan_large_scratch_words(uint32_t n) {
    size_t words = 64;
    for (uint32_t m = n; m > 1;) {
        m = (m + SCAN_BLOCK - 1) / SCAN_BLOCK;
        words += m;
    }
    return words;
}

// ---------------------------------------------------------------------------
// Spatial hash
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 collider_center(const DevPtrs& d, uint32_t c) {
    const uint32_t b = d.colOwner[c];
    return xyz(d.posLin[b]) + q_rotate(d.posAng[b], xyz(d.colLocalPos[c]));
}

__global__ void k_bp_count(const Params P, const DevPtrs d) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.numHashed) return;
    const uint32_t c = d.hashedIdx[i];
    int x, y, z;
    cell_coord(collider_center(d, c), P.cellSize, x, y, z);
    const uint32_t h = cell_hash(x, y, z, d.colGroup[c], P.gridHashSize);
    const uint32_t slot = atomicAdd(&d.cellCount[h], 1u);
    d.bodyCellSlot[i] = make_uint2(h, slot);
    if (d.colShape[c].w >= 0.0f) d.cellRigid[h] = 1u;
}

__global__ void k_bp_scatter(const Params P, const DevPtrs d) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.numHashed) return;
    const uint2 cs = d.bodyCellSlot[i];
    d.cellTmp[d.cellStart[cs.x] + cs.y] = d.hashedIdx[i];
}

static uint32_t stride_blocks_bp(uint32_t threads, int T) {
    const uint32_t need = (threads + T - 1) / T;
    const uint32_t cap = 148u * 16u;
    return need == 0 ? 1u : (need < cap ? need : cap);
}

// Collider order inside each bucket: one warp per bucket places every entry
// at its rank (the number of smaller ids; ids are distinct).  Dense buckets —
// a cloth sheet puts hundreds of particles in one cell — cost n^2/32 compares
// per lane instead of a serial insertion sort.
__global__ void k_bp_sort_cells(const Params P, const DevPtrs d) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; h < P.gridHashSize; h += warps) {
        const uint32_t n = d.cellCount[h];
        if (n == 0) continue;
        const uint32_t s = d.cellStart[h];
        const uint32_t* src = d.cellTmp + s;
        for (uint32_t i = lane; i < n; i += 32) {
            const uint32_t v = src[i];
            uint32_t rank = 0;
            for (uint32_t j = 0; j < n; j++) rank += src[j] < v ? 1u : 0u;
            d.cellBodies[s + rank] = v;
        }
    }
}

__device__ __forceinline__ bool pair_excluded(const uint32_t* ex, uint32_t count, uint32_t a,
                                              uint32_t b) {
    uint32_t lo = 0, hi = count;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t ea = ex[2 * mid], eb = ex[2 * mid + 1];
        if (ea < a || (ea == a && eb < b)) lo = mid + 1; else hi = mid;
    }
    return lo < count && ex[2 * lo] == a && ex[2 * lo + 1] == b;
}

__device__ __forceinline__ bool domains_compatible(uint32_t ga, uint32_t gb, uint32_t sa,
                                                   uint32_t sb) {
    if (!(ga == 0u || gb == 0u || ga == gb)) return false;
    if (ga == 0u && gb != 0u) return sb != 0u;
    if (gb == 0u && ga != 0u) return sa != 0u;
    return true;
}

// Per-frame collider record: world center and |radius|, plus the metadata
// the pair filters need, so a candidate test is two 16-byte loads.
__global__ void k_bp_prep(const Params P, const DevPtrs d, uint32_t numColliders) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= numColliders) return;
    const uint32_t owner = d.colOwner[c];
    const float4 pl = d.posLin[owner];
    const float3 center = xyz(pl) + q_rotate(d.posAng[owner], xyz(d.colLocalPos[c]));
    d.colCenter[c] = mk4(center, fabsf(d.colShape[c].w));
    d.colMeta[c] = make_uint4(owner, d.colGroup[c], d.colShared[c] | (pl.w > 0.0f ? 2u : 0u),
                              d.clothGroup[owner]);
}

// Candidate pairs of one producer collider (20_broadphase.metal:287-424),
// one warp per producer: lane s < 27 scans neighbour cell s in (dz, dy, dx)
// order, lane 27 scans the global list.  A cell whose hash equals an earlier
// lane's is skipped (the reference's visited-bucket check).  Lane counts are
// prefix-summed, so pairs come out in exactly the serial order: cells in
// order, each bucket in collider order, then globals.
template <bool EMIT>
__global__ void k_bp_pairs(const Params P, const DevPtrs d, uint32_t producers) {
    const uint32_t producer = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (producer >= producers) return;                     // warp-uniform
    uint32_t count = 0;
    const bool hashedProducer = producer < P.numHashed;
    const uint32_t a = hashedProducer ? d.hashedIdx[producer] : d.globalIdx[producer - P.numHashed];
    const float4 ca = d.colCenter[a];
    const uint4 ma = d.colMeta[a];
    const float3 pa = xyz(ca);
    const float ra = ca.w;
    const uint32_t ownerA = ma.x, groupA = ma.y, sharedA = ma.z & 1u, ga = ma.w;
    const bool aDyn = (ma.z & 2u) != 0;
    // first output slot of this lane: producer start + counts of lower lanes
    uint32_t slot = 0;
    // --- lane work: count (and in EMIT mode write) this lane's candidates
    auto visit = [&](uint32_t b, uint32_t outA, uint32_t outB, bool emit) -> bool {
        const uint4 mb = d.colMeta[b];
        if (!domains_compatible(groupA, mb.y, sharedA, mb.z & 1u)) return false;
        const uint32_t ownerB = mb.x;
        if (ownerA == ownerB) return false;
        if (!aDyn && (mb.z & 2u) == 0) return false;
        const float4 cb = d.colCenter[b];
        const float3 dp = pa - xyz(cb);
        const float r = ra + cb.w;
        if (dot(dp, dp) > r * r) return false;
        if (pair_excluded(d.exclusions, P.numExclusions, min(ownerA, ownerB), max(ownerA, ownerB))) return false;
        if (emit && slot + count < P.maxPairs) d.pairs[slot + count] = make_uint2(outA, outB);
        return true;
    };
    auto run_lane = [&](bool emit) {
        count = 0;
        if (hashedProducer) {
            if (lane < 27) {
                if (!(ga != 0 && P.numHashedRigid == 0)) {
                    int cx, cy, cz;
                    cell_coord(pa, P.cellSize, cx, cy, cz);
                    const int dz = (int)(lane / 9) - 1, dy = (int)((lane / 3) % 3) - 1, dx = (int)(lane % 3) - 1;
                    const uint32_t h = cell_hash(cx + dx, cy + dy, cz + dz, groupA, P.gridHashSize);
                    const unsigned same = __match_any_sync(0x07FFFFFFu, h);
                    const bool dup = (same & ((1u << lane) - 1u)) != 0u;
                    if (!dup && !(ga != 0 && d.cellRigid[h] == 0)) {
                        const uint32_t s0 = d.cellStart[h], e0 = s0 + d.cellCount[h];
                        for (uint32_t k = s0; k < e0; k++) {
                            const uint32_t b = d.cellBodies[k];
                            if (b <= a) continue;
                            // soft surface vs soft surface belongs to element contacts
                            if (ga != 0 && d.colMeta[b].w != 0) continue;
                            if (visit(b, a, b, emit)) count++;
                        }
                    }
                }
            } else if (lane == 27) {
                for (uint32_t g = 0; g < P.numGlobals; g++) {
                    const uint32_t b = d.globalIdx[g];
                    if (ga != 0 && d.colMeta[b].w == ga) continue;
                    if (visit(b, min(a, b), max(a, b), emit)) count++;
                }
            }
        } else if (lane == 27) {
            const uint32_t gp = producer - P.numHashed;
            for (uint32_t g = gp + 1; g < P.numGlobals; g++) {
                const uint32_t b = d.globalIdx[g];
                if (ga != 0 && d.colMeta[b].w == ga) continue;
                if (visit(b, min(a, b), max(a, b), emit)) count++;
            }
        }
    };
    if (!EMIT) {
        run_lane(false);
        d.pairLaneCount[(size_t)producer * 32 + lane] = count;
        uint32_t total = count;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
        if (lane == 0) d.pairCount[producer] = total;
    } else {
        const uint32_t mine = d.pairLaneCount[(size_t)producer * 32 + lane];
        uint32_t x = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        slot = d.pairStart[producer] + x - mine;
        run_lane(true);
    }
}

__global__ void k_bp_finalize(const Params P, const DevPtrs d, uint32_t producers) {
    const uint32_t n = producers == 0 ? 0u : d.pairStart[producers - 1] + d.pairCount[producers - 1];
    d.counters->pairCandidates = n;
    d.counters->numPairs = n < P.maxPairs ? n : P.maxPairs;
}

void launch_broadphase(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    cudaMemsetAsync(d.cellCount, 0, sizeof(uint32_t) * P.gridHashSize, st);
    cudaMemsetAsync(d.cellRigid, 0, sizeof(uint32_t) * P.gridHashSize, st);
    const int T = 128;
    if (P.numHashed > 0) {
        k_bp_count<<<(P.numHashed + T - 1) / T, T, 0, st>>>(P, d);
        launch_exclusive_scan(d.cellCount, d.cellStart, P.gridHashSize, d.scanScratch, st);
        k_bp_scatter<<<(P.numHashed + T - 1) / T, T, 0, st>>>(P, d);
        k_bp_sort_cells<<<stride_blocks_bp(P.gridHashSize * 32u, T), T, 0, st>>>(P, d);
    }
    if (z.producers > 0) {
        k_bp_prep<<<(z.numColliders + T - 1) / T, T, 0, st>>>(P, d, z.numColliders);
        const uint32_t warpsPerBlock = T / 32;
        const uint32_t blocks = (z.producers + warpsPerBlock - 1) / warpsPerBlock;
        k_bp_pairs<false><<<blocks, T, 0, st>>>(P, d, z.producers);
        launch_exclusive_scan(d.pairCount, d.pairStart, z.producers, d.scanScratch, st);
        k_bp_pairs<true><<<blocks, T, 0, st>>>(P, d, z.producers);
    }
    k_bp_finalize<<<1, 1, 0, st>>>(P, d, z.producers);
}

// ---------------------------------------------------------------------------
// Allocation-free exclusive scan (avbd_exclusive_scan_noalloc).
//
// Some callers cannot call cudaMalloc: an arena or pool that must own every
// device allocation, a real-time loop with an allocation ban, a host whose
// allocator must see every device allocation.  For them the scan's block sums
// live in this fixed device array instead of solver- or caller-allocated
// memory.  The array is part of the library's device image, so every GPU that
// loads the library holds these 4 KiB until the process exits.  Host code may
// not use the array's name as a device address (it is a host-side stand-in);
// the real address is looked up once per device with cudaGetSymbolAddress.
// ---------------------------------------------------------------------------
constexpr uint32_t kNoAllocScratchWords = SCAN_BLOCK;                        // 1024 block sums
constexpr uint32_t kNoAllocMaxElements = SCAN_BLOCK * kNoAllocScratchWords;  // 1,048,576 words

static __device__ __align__(256) uint32_t g_noalloc_scan_block_sums[kNoAllocScratchWords];

namespace {
constexpr int kMaxDevices = 256;
std::mutex g_noalloc_mutex;
uint32_t* g_noalloc_scratch[kMaxDevices] = {};   // device address per device ordinal
}  // namespace

void set_thread_error(const char* msg);

}  // namespace avbd

extern "C" int avbd_exclusive_scan_noalloc(const uint32_t* d_in, uint32_t* d_out, uint32_t n,
                                           void* cuda_stream) {
    using namespace avbd;
    if (n == 0) return AVBD_OK;
    if (!d_in || !d_out) {
        set_thread_error("avbd_exclusive_scan_noalloc: null device pointer");
        return AVBD_ERR_INVALID_ARGUMENT;
    }
    if (n > kNoAllocMaxElements) {
        set_thread_error("avbd_exclusive_scan_noalloc: n exceeds the 1,048,576-element limit "
                         "of its fixed 4 KiB scratch");
        return AVBD_ERR_INVALID_ARGUMENT;
    }
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_thread_error("avbd_exclusive_scan_noalloc: no current CUDA device");
        return AVBD_ERR_NO_DEVICE;
    }
    uint32_t* scratch = nullptr;
    {
        // once per device, with that device current: the device address of
        // the fixed scratch array
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_scratch[dev]) {
            void* addr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scan_block_sums);
            if (e != cudaSuccess || !addr) {
                set_thread_error("avbd_exclusive_scan_noalloc: cudaGetSymbolAddress failed");
                return AVBD_ERR_KERNEL_MISSING;
            }
            g_noalloc_scratch[dev] = static_cast<uint32_t*>(addr);
        }
        scratch = g_noalloc_scratch[dev];
    }
    // k_scan_blocks writes block sum b before k_scan_block_sums and k_scan_add
    // read it, so the shared scratch needs no clearing between calls.
    launch_exclusive_scan(d_in, d_out, n, scratch, static_cast<cudaStream_t>(cuda_stream));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_thread_error(cudaGetErrorString(e));
        return AVBD_ERR_RUNTIME_FAILURE;
    }
    return AVBD_OK;
}
