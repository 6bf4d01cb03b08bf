// bucket_sort.cuh — in-bucket ordering of counting-sorted hash grids.
#pragma once
#include <cstdint>

namespace avbd {

// Buckets a warp takes at a time: 32 when the grid has many more buckets
// than the launch has warps (sparse grids), fewer down to one when it has
// few, so that every warp still gets a group.
__device__ __forceinline__ uint32_t bucket_group(uint32_t buckets, uint32_t warps) {
    uint32_t g = 32u;
    while (g > 1u && (uint64_t)warps * g > (uint64_t)buckets) g >>= 1;
    return g;
}

// Every bucket's entries in ascending order (ids within a bucket are
// distinct): a warp takes a group of consecutive buckets (bucket_group),
// one count per lane in a single coalesced load, and then places the
// entries of each non-empty one of them at their rank (the number of
// smaller ids) — one dependent count load per group instead of one per
// bucket, which dominated the sparse grids (millions of buckets, a few
// thousand in use).  Dense buckets cost n^2/32 compares per lane.
__device__ __forceinline__ void rank_sort_buckets(const uint32_t* __restrict__ count,
                                                  const uint32_t* __restrict__ start,
                                                  const uint32_t* __restrict__ tmp, uint32_t* __restrict__ out,
                                                  uint32_t buckets) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t G = bucket_group(buckets, warps);
    for (uint32_t base = warp * G; base < buckets; base += warps * G) {
        const uint32_t h = base + lane;
        const uint32_t myN = (lane < G && h < buckets) ? count[h] : 0u;
        const uint32_t myS = myN ? start[h] : 0u;
        uint32_t live = __ballot_sync(0xffffffffu, myN != 0u);
        while (live) {
            const int b = __ffs(live) - 1;
            live &= live - 1u;
            const uint32_t n = __shfl_sync(0xffffffffu, myN, b);
            const uint32_t s = __shfl_sync(0xffffffffu, myS, b);
            const uint32_t* src = tmp + s;
            for (uint32_t i = lane; i < n; i += 32) {
                const uint32_t v = src[i];
                uint32_t rank = 0;
                for (uint32_t j = 0; j < n; j++) rank += src[j] < v ? 1u : 0u;
                out[s + rank] = v;
            }
        }
    }
}

}  // namespace avbd
