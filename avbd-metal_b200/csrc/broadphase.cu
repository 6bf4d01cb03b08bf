// broadphase.cu — exclusive scan, counting-sort spatial hash and
// deterministic candidate-pair generation.
//
// Follows Shaders/10_scan.metal and Shaders/20_broadphase.metal:69-131,
// :287-512.  The hash grid is a counting sort (count -> scan -> scatter ->
// per-bucket sort by collider id); pairs are produced in two passes (count
// per producer, scan, emit in producer/cell order) so the pair list — and
// with it the manifold index of every pair — is the same on every run.
#include <mutex>

#include "bucket_sort.cuh"
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

// Every hashed collider into its bucket (cell hash with its collision group);
// cellRigid counts the rigid colliders of a bucket.  With the particle grid
// on (P.fineBP), particle colliders are also binned into fine cells of twice
// the largest particle radius (hash without group).
__global__ void k_bp_count(const Params P, const DevPtrs d) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.numHashed) return;
    const uint32_t c = d.hashedIdx[i];
    int x, y, z;
    const float3 p = collider_center(d, c);
    cell_coord(p, P.cellSize, x, y, z);
    const uint32_t h = cell_hash(x, y, z, d.colGroup[c], P.gridHashSize);
    const uint32_t slot = atomicAdd(&d.cellCount[h], 1u);
    d.bodyCellSlot[i] = make_uint2(h, slot);
    d.colBucket[c] = h;
    if (d.colShape[c].w >= 0.0f) {
        atomicAdd(&d.cellRigid[h], 1u);
    } else if (P.fineBP) {
        cell_coord(p, P.fineCellSize, x, y, z);
        const uint32_t hf = cell_hash(x, y, z, 0u, P.fineHashSize);
        d.fineSlot[i] = make_uint2(hf, atomicAdd(&d.fineCount[hf], 1u));
    }
}

__global__ void k_bp_scatter(const Params P, const DevPtrs d) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.numHashed) return;
    const uint2 cs = d.bodyCellSlot[i];
    const uint32_t c = d.hashedIdx[i];
    d.cellTmp[d.cellStart[cs.x] + cs.y] = c;
    if (P.fineBP && d.colShape[c].w < 0.0f) {
        const uint2 fs = d.fineSlot[i];
        d.fineTmp[d.fineStart[fs.x] + fs.y] = c;
    }
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
__global__ void k_bp_sort_cells(const uint32_t* count, const uint32_t* start, const uint32_t* tmp, uint32_t* out,
                                uint32_t buckets) {
    rank_sort_buckets(count, start, tmp, out, buckets);
}

// The rigid colliders of every bucket, in bucket (collider) order: a warp
// reads a group of buckets' rigid counts at once (bucket_group) and
// compacts each bucket that has any, one after another.
__global__ void k_bp_rigid_compact(const Params P, const DevPtrs d) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    // a group of buckets' rigid counts per coalesced load, then one bucket
    // at a time
    const uint32_t G = bucket_group(P.gridHashSize, warps);
    for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * G; base < P.gridHashSize;
         base += warps * G) {
        const uint32_t hl = base + lane;
        uint32_t live = __ballot_sync(0xffffffffu, lane < G && hl < P.gridHashSize && d.cellRigid[hl] != 0u);
        while (live) {
            const uint32_t h = base + (uint32_t)(__ffs(live) - 1);
            live &= live - 1u;
            const uint32_t s = d.cellStart[h], n = d.cellCount[h];
            uint32_t out = d.rigidStart[h];
            for (uint32_t k0 = 0; k0 < n; k0 += 32) {
                const uint32_t k = k0 + lane;
                uint32_t c = 0;
                bool rigid = false;
                if (k < n) {
                    c = d.cellBodies[s + k];
                    rigid = d.colShape[c].w >= 0.0f;
                }
                const uint32_t ballot = __ballot_sync(0xffffffffu, rigid);
                if (rigid) d.rigidCells[out + __popc(ballot & ((1u << lane) - 1u))] = c;
                out += __popc(ballot);
            }
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

// Boxes of every chunk of 32 global colliders: collider spheres (pair
// kernels) and owner bounding spheres (rigid-triangle emission).  A chunk
// that a query ball misses cannot hold a candidate, so the global scans skip
// it; the candidates they keep, and their order, are unchanged.
__global__ void k_global_chunks(const Params P, const DevPtrs d) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t chunk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t g = chunk * 32u + lane;
    if (chunk * 32u >= P.numGlobals) return;                // warp-uniform
    const float big = 3.0e38f;
    float3 clo = s3(big), chi = s3(-big), blo = s3(big), bhi = s3(-big);
    if (g < P.numGlobals) {
        const uint32_t c = d.globalIdx[g];
        const float4 cc = d.colCenter[c];
        clo = xyz(cc) - s3(cc.w);
        chi = xyz(cc) + s3(cc.w);
        const uint32_t o = d.colOwner[c];
        const float4 shp = d.shape[o];
        const float3 po = xyz(d.posLin[o]);
        const float rb = fabsf(shp.w);
        // the owner's pose and shape in one record for the global scans
        d.globalRec[3 * (size_t)g] = mk4(po, shp.w);
        d.globalRec[3 * (size_t)g + 1] = d.posAng[o];
        d.globalRec[3 * (size_t)g + 2] = mk4(xyz(shp), __uint_as_float(d.bodyShape[o]));
        blo = po - s3(rb);
        bhi = po + s3(rb);
        // a non-finite member makes the chunk unbounded (never skipped)
        if (!(finite3(clo) && finite3(chi))) { clo = s3(-big); chi = s3(big); }
        if (!(finite3(blo) && finite3(bhi))) { blo = s3(-big); bhi = s3(big); }
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        clo = mk3(fminf(clo.x, __shfl_xor_sync(0xffffffffu, clo.x, off)), fminf(clo.y, __shfl_xor_sync(0xffffffffu, clo.y, off)),
                  fminf(clo.z, __shfl_xor_sync(0xffffffffu, clo.z, off)));
        chi = mk3(fmaxf(chi.x, __shfl_xor_sync(0xffffffffu, chi.x, off)), fmaxf(chi.y, __shfl_xor_sync(0xffffffffu, chi.y, off)),
                  fmaxf(chi.z, __shfl_xor_sync(0xffffffffu, chi.z, off)));
        blo = mk3(fminf(blo.x, __shfl_xor_sync(0xffffffffu, blo.x, off)), fminf(blo.y, __shfl_xor_sync(0xffffffffu, blo.y, off)),
                  fminf(blo.z, __shfl_xor_sync(0xffffffffu, blo.z, off)));
        bhi = mk3(fmaxf(bhi.x, __shfl_xor_sync(0xffffffffu, bhi.x, off)), fmaxf(bhi.y, __shfl_xor_sync(0xffffffffu, bhi.y, off)),
                  fmaxf(bhi.z, __shfl_xor_sync(0xffffffffu, bhi.z, off)));
    }
    if (lane == 0) {
        float4* out = d.globalChunk + 4 * (size_t)chunk;
        out[0] = mk4(clo, 0.0f);
        out[1] = mk4(chi, 0.0f);
        out[2] = mk4(blo, 0.0f);
        out[3] = mk4(bhi, 0.0f);
    }
}

// Candidate pairs of one producer collider (20_broadphase.metal:287-424),
// one warp per producer: lane s < 27 scans neighbour cell s in (dz, dy, dx)
// order, lane 27 scans the global list.  A cell whose hash equals an earlier
// lane's is skipped (the reference's visited-bucket check).  Lane counts are
// prefix-summed, so pairs come out in exactly the serial order: cells in
// order, each bucket in collider order, then globals.
//
// With the particle grid on (P.fineBP: large rigid colliders make the cells
// far coarser than the particles), a particle producer takes its rigid
// candidates from the rigid sublists of its buckets and its particle
// candidates from the 27 fine cells around it, keeps exactly the candidates
// the bucket scan would accept (bucket in its visit list, the same filters)
// and sorts them into the serial order: by the visit rank of the candidate's
// bucket, then by collider index.
template <bool EMIT>
__global__ void __launch_bounds__(128) k_bp_pairs(const Params P, const DevPtrs d, uint32_t producers) {
    __shared__ uint32_t visitH[4][27];
    const uint32_t producer = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
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
    const bool fine = P.fineBP && hashedProducer && d.colShape[a].w < 0.0f;
    // rigid producers next to the particle grid scan their (large) buckets
    // with a warp per bucket in k_bp_heavy; here they only total the counts
    const bool heavy = P.fineBP && hashedProducer && !fine;
    if (heavy) {
        if (!EMIT) {
            const uint32_t c = lane < 28 ? d.pairLaneCount[(size_t)producer * 32 + lane] : 0u;
            if (lane >= 28) d.pairLaneCount[(size_t)producer * 32 + lane] = 0u;
            uint32_t total = c;
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
            if (lane == 0) d.pairCount[producer] = total;
        }
        return;
    }
    // this lane's bucket (NONE when an earlier lane visits the same bucket)
    uint32_t h = 0xFFFFFFFFu, hf = 0xFFFFFFFFu;
    if (hashedProducer) {
        int cx = 0, cy = 0, cz = 0;
        cell_coord(pa, P.cellSize, cx, cy, cz);
        const int dz = (int)(lane / 9) - 1, dy = (int)((lane / 3) % 3) - 1, dx = (int)(lane % 3) - 1;
        const uint32_t hh = cell_hash(cx + dx, cy + dy, cz + dz, groupA, P.gridHashSize);
        const unsigned same = __match_any_sync(0xffffffffu, lane < 27 ? hh : 0xFFFFFFFFu);
        if (lane < 27 && (same & ((1u << lane) - 1u)) == 0u) h = hh;
        if (fine) {
            cell_coord(pa, P.fineCellSize, cx, cy, cz);
            const uint32_t hfh = cell_hash(cx + dx, cy + dy, cz + dz, 0u, P.fineHashSize);
            const unsigned sameF = __match_any_sync(0xffffffffu, lane < 27 ? hfh : 0xFFFFFFFFu);
            if (lane < 27 && (sameF & ((1u << lane) - 1u)) == 0u) hf = hfh;
            if (lane < 27) visitH[warp][lane] = h;
            __syncwarp();
        }
    }
    auto visit_rank = [&](uint32_t hb) -> uint32_t {
        for (uint32_t s = 0; s < 27; s++)
            if (visitH[warp][s] == hb) return s;
        return 0xFFFFFFFFu;
    };
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
                    if (h != 0xFFFFFFFFu && !(ga != 0 && d.cellRigid[h] == 0)) {
                        // the whole bucket, or only its rigid colliders when
                        // the particle grid supplies the particles
                        const uint32_t* list = fine ? d.rigidCells + d.rigidStart[h] : d.cellBodies + d.cellStart[h];
                        const uint32_t n = fine ? d.cellRigid[h] : d.cellCount[h];
                        for (uint32_t k = 0; k < n; k++) {
                            const uint32_t b = list[k];
                            if (b <= a) continue;
                            // soft surface vs soft surface belongs to element contacts
                            if (ga != 0 && d.colMeta[b].w != 0) continue;
                            if (visit(b, a, b, emit)) count++;
                        }
                    }
                    if (fine && hf != 0xFFFFFFFFu) {
                        const uint32_t s0 = d.fineStart[hf], e0 = s0 + d.fineCount[hf];
                        for (uint32_t k = s0; k < e0; k++) {
                            const uint32_t b = d.fineCells[k];
                            if (b <= a) continue;
                            if (ga != 0 && d.colMeta[b].w != 0) continue;
                            const uint32_t hb = d.colBucket[b];
                            if (ga != 0 && d.cellRigid[hb] == 0) continue;
                            if (visit_rank(hb) == 0xFFFFFFFFu) continue;
                            if (visit(b, a, b, emit)) count++;
                        }
                    }
                }
            }
        }
        // the global list, counted for lane 27: the whole warp tests 32
        // globals at a time and ranks the accepted ones by ballot
        const uint32_t g0 = hashedProducer ? 0u : producer - P.numHashed + 1u;
        const uint32_t gslot = __shfl_sync(0xffffffffu, slot, 27);
        const uint32_t below = (1u << lane) - 1u;
        uint32_t gcount = 0;
        // chunks whose boxes the producer's ball misses are skipped; lane l
        // tests chunk c0 + l, 32 chunks per load, and the kept ones are
        // visited in order
        const uint32_t chunks = (P.numGlobals + 31u) / 32u;
        for (uint32_t c0 = g0 >> 5; c0 < chunks; c0 += 32) {
            bool keep = c0 + lane < chunks;
            if (keep && P.numGlobals > 32) {
                const float4* box = d.globalChunk + 4 * (size_t)(c0 + lane);
                keep = !ball_misses_box(pa, ra, box[0], box[1]);
            }
            uint32_t live = __ballot_sync(0xffffffffu, keep);
            while (live) {
                const uint32_t gb = (c0 + (uint32_t)(__ffs(live) - 1)) * 32u;
                live &= live - 1u;
                const uint32_t g = gb + lane;
                uint32_t b = 0;
                bool pass = false;
                if (g >= g0 && g < P.numGlobals) {
                    b = d.globalIdx[g];
                    if (!(ga != 0 && d.colMeta[b].w == ga)) pass = visit(b, 0u, 0u, false);
                }
                const uint32_t ballot = __ballot_sync(0xffffffffu, pass);
                if (emit && pass) {
                    const uint32_t o = gslot + gcount + __popc(ballot & below);
                    if (o < P.maxPairs) d.pairs[o] = make_uint2(min(a, b), max(a, b));
                }
                gcount += __popc(ballot);
            }
        }
        if (lane == 27) count = gcount;
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
        if (fine) {
            // bucket pairs (lanes 0-26) into the serial order; the global
            // pairs of lane 27 already follow them in order
            const uint32_t first = __shfl_sync(0xffffffffu, slot, 0);
            const uint32_t end = min(__shfl_sync(0xffffffffu, slot, 27), P.maxPairs);
            __syncwarp();
            if (lane == 0 && end > first + 1) {
                auto key = [&](uint2 p) { return (visit_rank(d.colBucket[p.y]) << 24) | p.y; };
                for (uint32_t i = first + 1; i < end; i++) {
                    const uint2 v = d.pairs[i];
                    const uint32_t kv = key(v);
                    uint32_t j = i;
                    while (j > first && key(d.pairs[j - 1]) > kv) { d.pairs[j] = d.pairs[j - 1]; j--; }
                    d.pairs[j] = v;
                }
            }
        }
    }
}

// One rigid producer's bucket s (s < 27) or its global list (s == 27) with a
// whole warp: entries in chunks of 32, emitted in order by ballot rank.
template <bool EMIT>
__global__ void __launch_bounds__(128) k_bp_heavy(const Params P, const DevPtrs d, const uint32_t* list, uint32_t n) {
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (w >= n * 28u) return;                               // warp-uniform
    const uint32_t producer = list[w / 28u], s = w % 28u;
    const uint32_t a = d.hashedIdx[producer];
    const float4 ca = d.colCenter[a];
    const uint4 ma = d.colMeta[a];
    const float3 pa = xyz(ca);
    const float ra = ca.w;
    const uint32_t ownerA = ma.x, groupA = ma.y, sharedA = ma.z & 1u, ga = ma.w;
    const bool aDyn = (ma.z & 2u) != 0;
    const uint32_t below = (1u << lane) - 1u;
    uint32_t slot = 0;
    if (EMIT) {
        const uint32_t c = lane < s ? d.pairLaneCount[(size_t)producer * 32 + lane] : 0u;
        uint32_t x = c;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        slot = d.pairStart[producer] + x;
    }
    auto accept = [&](uint32_t b) -> bool {
        const uint4 mb = d.colMeta[b];
        if (!domains_compatible(groupA, mb.y, sharedA, mb.z & 1u)) return false;
        const uint32_t ownerB = mb.x;
        if (ownerA == ownerB) return false;
        if (!aDyn && (mb.z & 2u) == 0) return false;
        const float4 cb = d.colCenter[b];
        const float3 dp = pa - xyz(cb);
        const float r = ra + cb.w;
        if (dot(dp, dp) > r * r) return false;
        return !pair_excluded(d.exclusions, P.numExclusions, min(ownerA, ownerB), max(ownerA, ownerB));
    };
    uint32_t count = 0;
    if (s < 27) {
        int cx, cy, cz;
        cell_coord(pa, P.cellSize, cx, cy, cz);
        const int dz = (int)(lane / 9) - 1, dy = (int)((lane / 3) % 3) - 1, dx = (int)(lane % 3) - 1;
        const uint32_t hh = cell_hash(cx + dx, cy + dy, cz + dz, groupA, P.gridHashSize);
        const unsigned same = __match_any_sync(0xffffffffu, lane < 27 ? hh : 0xFFFFFFFFu);
        const bool dupMine = lane < 27 && (same & below) != 0u;
        const uint32_t h = __shfl_sync(0xffffffffu, hh, s);
        const bool dup = __shfl_sync(0xffffffffu, dupMine ? 1u : 0u, s) != 0u;
        if (!(ga != 0 && P.numHashedRigid == 0) && !dup && !(ga != 0 && d.cellRigid[h] == 0)) {
            const uint32_t s0 = d.cellStart[h], nb = d.cellCount[h];
            for (uint32_t k0 = 0; k0 < nb; k0 += 32) {
                const uint32_t k = k0 + lane;
                uint32_t b = 0;
                bool pass = false;
                if (k < nb) {
                    b = d.cellBodies[s0 + k];
                    pass = b > a && !(ga != 0 && d.colMeta[b].w != 0) && accept(b);
                }
                const uint32_t ballot = __ballot_sync(0xffffffffu, pass);
                if (EMIT && pass) {
                    const uint32_t o = slot + count + __popc(ballot & below);
                    if (o < P.maxPairs) d.pairs[o] = make_uint2(a, b);
                }
                count += __popc(ballot);
            }
        }
    } else {
        // kept chunks in order, 32 chunk boxes tested per load (as above)
        const uint32_t chunks = (P.numGlobals + 31u) / 32u;
        for (uint32_t c0 = 0; c0 < chunks; c0 += 32) {
            bool keep = c0 + lane < chunks;
            if (keep && P.numGlobals > 32) {
                const float4* box = d.globalChunk + 4 * (size_t)(c0 + lane);
                keep = !ball_misses_box(pa, ra, box[0], box[1]);
            }
            uint32_t live = __ballot_sync(0xffffffffu, keep);
            while (live) {
                const uint32_t g0 = (c0 + (uint32_t)(__ffs(live) - 1)) * 32u;
                live &= live - 1u;
                const uint32_t g = g0 + lane;
                uint32_t b = 0;
                bool pass = false;
                if (g < P.numGlobals) {
                    b = d.globalIdx[g];
                    pass = !(ga != 0 && d.colMeta[b].w == ga) && accept(b);
                }
                const uint32_t ballot = __ballot_sync(0xffffffffu, pass);
                if (EMIT && pass) {
                    const uint32_t o = slot + count + __popc(ballot & below);
                    if (o < P.maxPairs) d.pairs[o] = make_uint2(min(a, b), max(a, b));
                }
                count += __popc(ballot);
            }
        }
    }
    if (!EMIT && lane == 0) d.pairLaneCount[(size_t)producer * 32 + s] = count;
}

__global__ void k_bp_finalize(const Params P, const DevPtrs d, uint32_t producers) {
    const uint32_t n = producers == 0 ? 0u : d.pairStart[producers - 1] + d.pairCount[producers - 1];
    d.counters->pairCandidates = n;
    d.counters->numPairs = n < P.maxPairs ? n : P.maxPairs;
}

void launch_broadphase(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    cudaMemsetAsync(d.cellCount, 0, sizeof(uint32_t) * P.gridHashSize, st);
    cudaMemsetAsync(d.cellRigid, 0, sizeof(uint32_t) * P.gridHashSize, st);
    if (P.fineBP) cudaMemsetAsync(d.fineCount, 0, sizeof(uint32_t) * P.fineHashSize, st);
    const int T = 128;
    if (P.numHashed > 0) {
        k_bp_count<<<(P.numHashed + T - 1) / T, T, 0, st>>>(P, d);
        launch_exclusive_scan(d.cellCount, d.cellStart, P.gridHashSize, d.scanScratch, st);
        if (P.fineBP) launch_exclusive_scan(d.fineCount, d.fineStart, P.fineHashSize, d.scanScratch, st);
        k_bp_scatter<<<(P.numHashed + T - 1) / T, T, 0, st>>>(P, d);
        k_bp_sort_cells<<<stride_blocks_bp(P.gridHashSize * 32u, T), T, 0, st>>>(d.cellCount, d.cellStart, d.cellTmp,
                                                                                   d.cellBodies, P.gridHashSize);
        if (P.numHashedRigid > 0) {
            launch_exclusive_scan(d.cellRigid, d.rigidStart, P.gridHashSize, d.scanScratch, st);
            k_bp_rigid_compact<<<stride_blocks_bp(P.gridHashSize * 32u, T), T, 0, st>>>(P, d);
        }
        if (P.fineBP)
            k_bp_sort_cells<<<stride_blocks_bp(P.fineHashSize * 32u, T), T, 0, st>>>(d.fineCount, d.fineStart, d.fineTmp,
                                                                                       d.fineCells, P.fineHashSize);
    }
    if (z.producers > 0) {
        k_bp_prep<<<(z.numColliders + T - 1) / T, T, 0, st>>>(P, d, z.numColliders);
        if (P.numGlobals > 32) {
            const uint32_t chunks = (P.numGlobals + 31) / 32;
            k_global_chunks<<<(chunks + 3) / 4, 128, 0, st>>>(P, d);
        }
        const uint32_t warpsPerBlock = T / 32;
        const uint32_t blocks = (z.producers + warpsPerBlock - 1) / warpsPerBlock;
        const uint32_t nh = z.numHeavyProducers;
        const uint32_t hblocks = (nh * 28u + warpsPerBlock - 1) / warpsPerBlock;
        if (nh) k_bp_heavy<false><<<hblocks, T, 0, st>>>(P, d, d.heavyProducers, nh);
        k_bp_pairs<false><<<blocks, T, 0, st>>>(P, d, z.producers);
        launch_exclusive_scan(d.pairCount, d.pairStart, z.producers, d.scanScratch, st);
        if (nh) k_bp_heavy<true><<<hblocks, T, 0, st>>>(P, d, d.heavyProducers, nh);
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
// the real address is looked up once per CUDA context with
// cudaGetSymbolAddress.
// ---------------------------------------------------------------------------
constexpr uint32_t kNoAllocScratchWords = SCAN_BLOCK;                        // 1024 block sums
constexpr uint32_t kNoAllocMaxElements = SCAN_BLOCK * kNoAllocScratchWords;  // 1,048,576 words

static __device__ __align__(256) uint32_t g_noalloc_scan_block_sums[kNoAllocScratchWords];

// In-place first pass (d_in == d_out): the same block scan as k_scan_blocks
// with one pointer, no __restrict__.  Each thread loads its own words before
// the block scan's barriers and stores to the same words after them.
__global__ void k_scan_blocks_inplace(uint32_t* data, uint32_t* blockSums, uint32_t n) {
    __shared__ uint32_t warpSums[32];
    const uint32_t base = blockIdx.x * SCAN_BLOCK + threadIdx.x * SCAN_GRAIN;
    uint32_t v[SCAN_GRAIN];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_GRAIN; i++) {
        v[i] = base + i < n ? data[base + i] : 0u;
        sum += v[i];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, warpSums, total);
#pragma unroll
    for (int i = 0; i < SCAN_GRAIN; i++) {
        if (base + i < n) data[base + i] = run;
        run += v[i];
    }
    if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

namespace {
// The array's device address, looked up once per CUDA context: a __device__
// symbol is loaded separately into every context, so a caller that makes a
// non-primary context current (cuCtxCreate / cuCtxSetCurrent) gets that
// context's copy, not the primary context's.
struct ScratchEntry { void* ctx; uint32_t* addr; };
constexpr int kMaxContexts = 64;
std::mutex g_noalloc_mutex;
ScratchEntry g_noalloc_scratch[kMaxContexts] = {};
int g_noalloc_entries = 0;
using CtxGetCurrentFn = int (*)(void**);
CtxGetCurrentFn g_ctx_get_current = nullptr;
bool g_ctx_lookup_done = false;

// The current driver context (cuCtxGetCurrent through the runtime's entry
// point table, so the library needs no link against libcuda), or null.
void* current_context() {
    if (!g_ctx_lookup_done) {
        g_ctx_lookup_done = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    }
    void* ctx = nullptr;
    if (!g_ctx_get_current || g_ctx_get_current(&ctx) != 0) return nullptr;
    return ctx;
}
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
    const uintptr_t inLo = reinterpret_cast<uintptr_t>(d_in), outLo = reinterpret_cast<uintptr_t>(d_out);
    const uintptr_t bytes = (uintptr_t)n * sizeof(uint32_t);
    const bool inPlace = inLo == outLo;
    if (!inPlace && inLo < outLo + bytes && outLo < inLo + bytes) {
        set_thread_error("avbd_exclusive_scan_noalloc: d_in and d_out overlap without being equal");
        return AVBD_ERR_INVALID_ARGUMENT;
    }
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        set_thread_error("avbd_exclusive_scan_noalloc: no current CUDA device");
        return AVBD_ERR_NO_DEVICE;
    }
    uint32_t* scratch = nullptr;
    {
        // once per context, with it current: the device address of the
        // fixed scratch array
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        void* ctx = current_context();
        for (int i = 0; i < g_noalloc_entries && ctx; i++)
            if (g_noalloc_scratch[i].ctx == ctx) scratch = g_noalloc_scratch[i].addr;
        if (!scratch) {
            void* addr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scan_block_sums);
            if (e != cudaSuccess || !addr) {
                set_thread_error("avbd_exclusive_scan_noalloc: cudaGetSymbolAddress failed");
                return AVBD_ERR_KERNEL_MISSING;
            }
            scratch = static_cast<uint32_t*>(addr);
            if (ctx && g_noalloc_entries < kMaxContexts) g_noalloc_scratch[g_noalloc_entries++] = {ctx, scratch};
        }
    }
    // The first pass writes block sum b before the block-sum scan and the
    // uniform add read it, so the shared scratch needs no clearing between calls.
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    if (inPlace) {
        const uint32_t nblocks = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
        k_scan_blocks_inplace<<<nblocks, SCAN_THREADS, 0, st>>>(d_out, scratch, n);
        if (nblocks > 1) {
            k_scan_block_sums<<<1, SCAN_THREADS, 0, st>>>(scratch, nblocks);
            k_scan_add<<<nblocks, SCAN_THREADS, 0, st>>>(d_out, scratch, n);
        }
    } else {
        launch_exclusive_scan(d_in, d_out, n, scratch, st);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_thread_error(cudaGetErrorString(e));
        return AVBD_ERR_RUNTIME_FAILURE;
    }
    return AVBD_OK;
}
