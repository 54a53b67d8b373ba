// Ordering of one cell's entries by value with one warp, shared by the
// engine's re-sort and the allocation-free cell sort.
#pragma once

#include <cstdint>

namespace sphb {

// Entries per lane the warp ranks in registers: cells of up to
// 32 * kCellRankPer entries are ordered by warp_rank_order.
constexpr int kCellRankPer = 16;
constexpr unsigned kCellRankMax = 32u * kCellRankPer;

// Orders vals[b .. b+n) ascending (the values are distinct) with the calling
// warp: the lanes hold the entries in registers and each entry's rank is the
// number of smaller ones, counted over warp shuffles.  n <= kCellRankMax;
// every lane of the warp calls it with the same b and n.
__device__ __forceinline__ void warp_rank_order(uint32_t *vals, unsigned b, unsigned n,
                                                unsigned lane)
{
    const unsigned kn = (n + 31u) >> 5;   // occupied register rows
    unsigned v[kCellRankPer], rk[kCellRankPer];
#pragma unroll
    for (int k = 0; k < kCellRankPer; ++k) {
        const unsigned idx = lane + 32u * k;
        v[k] = ((unsigned)k < kn && idx < n) ? __ldcg(&vals[b + idx]) : 0xffffffffu;
        rk[k] = 0;
    }
#pragma unroll
    for (int k2 = 0; k2 < kCellRankPer; ++k2) {
        if ((unsigned)k2 >= kn) break;
        for (unsigned src = 0; src < 32u; ++src) {
            const unsigned w = __shfl_sync(0xffffffffu, v[k2], src);
            if (32u * k2 + src >= n) break;
#pragma unroll
            for (int k = 0; k < kCellRankPer; ++k)
                if ((unsigned)k < kn) rk[k] += w < v[k] ? 1u : 0u;
        }
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kCellRankPer; ++k) {
        const unsigned idx = lane + 32u * k;
        if ((unsigned)k < kn && idx < n) vals[b + rk[k]] = v[k];
    }
}

}  // namespace sphb
