// Cell sort of one simulation's particles by a group of thread blocks
// (the reference's calcParticleCellID + thrust::sort_by_key +
// reorderArrays, src/sorting.cuh:25-132, src/device.cu:1066-1114).
//
// The particle arrays stay in sorted order between steps and are re-sorted
// only when some particle's cell changed.  A stable sort of unchanged keys
// is the identity, so skipping it is exact.  The sort is a bucket sort on
// cells: count per cell, exclusive scan (cellStart/cellEnd), atomic
// scatter, then each cell's few entries are ordered by original index,
// which gives exactly the stable (cellID, index) order.  The phases are
// separated by a barrier over the group (a grid barrier for a cooperative
// launch, a group barrier inside the persistent step kernel).
#pragma once

#include "dem_state.h"
#include "cell_order.cuh"

namespace sphb {

// Block-wide exclusive scan of one value per thread (blockDim a multiple of
// 32, at most 1024).
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned &total)
{
    __shared__ unsigned warp_tot[32];
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned x = v;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned w = lane < nw ? warp_tot[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (unsigned)o) w += y;
        }
        if (lane < nw) warp_tot[lane] = w;  // inclusive warp prefix
    }
    __syncthreads();
    unsigned before = wid ? warp_tot[wid - 1] : 0;
    total = warp_tot[nw - 1];
    __syncthreads();
    return before + x - v;
}

// Per-particle scratch arrays of a re-sort (carved from one byte buffer).
struct PermScratch {
    double4 *x, *vel, *angvel, *angpos, *acc, *angacc, *xyzsum;
    double *es, *ev;
    uint32_t *cell;
};

__host__ __device__ inline PermScratch make_perm_scratch(unsigned char *p, size_t n)
{
    auto take = [&](size_t bytes) {
        unsigned char *q = p;
        p += (bytes + 255) & ~(size_t)255;
        return q;
    };
    PermScratch W;
    W.x = (double4 *)take(n * 32); W.vel = (double4 *)take(n * 32);
    W.angvel = (double4 *)take(n * 32); W.angpos = (double4 *)take(n * 32);
    W.acc = (double4 *)take(n * 32); W.angacc = (double4 *)take(n * 32);
    W.xyzsum = (double4 *)take(n * 32);
    W.es = (double *)take(n * 8); W.ev = (double *)take(n * 8);
    W.cell = (uint32_t *)take(n * 4);
    return W;
}

inline size_t perm_scratch_bytes(size_t n)
{
    return 7 * ((n * 32 + 255) & ~(size_t)255) + 2 * ((n * 8 + 255) & ~(size_t)255) +
           ((n * 4 + 255) & ~(size_t)255) + 256;
}

// Re-sorts S in place.  The group has `nranks` blocks; this block is
// `rank`; `bar()` is the group barrier (returns false when it gave up).
// With refresh_f the FP32 velocity copies of the mixed mode are rewritten
// from the permuted FP64 velocities.  Returns false when a barrier failed.
template <class Bar>
__device__ bool resort_group(const DevParams &P, const DevState &S, const PermScratch &W,
                             unsigned nranks, unsigned rank, Bar &&bar, bool refresh_f)
{
    const unsigned G = nranks;
    const unsigned gtid = rank * blockDim.x + threadIdx.x;
    const unsigned gstride = G * blockDim.x;
    const unsigned np = P.np, ncells = P.ncells;

    // 1. zero the per-cell counts
    for (unsigned c = gtid; c < ncells; c += gstride) S.count[c] = 0;
    if (!bar()) return false;
    // 2. count particles per cell
    for (unsigned k = gtid; k < np; k += gstride) atomicAdd(&S.count[__ldcg(&S.cell_new[k])], 1u);
    if (!bar()) return false;
    // 3. exclusive scan of the counts over contiguous chunks of cells
    const unsigned chunk = (ncells + G - 1) / G;
    const unsigned c0 = min(rank * chunk, ncells), c1 = min(c0 + chunk, ncells);
    {
        unsigned s = 0;
        for (unsigned c = c0 + threadIdx.x; c < c1; c += blockDim.x) s += __ldcg(&S.count[c]);
        unsigned tot;
        (void)block_exclusive_scan(s, tot);
        if (threadIdx.x == 0) S.block_sums[rank] = tot;
    }
    if (!bar()) return false;
    if (rank == 0) {
        // exclusive scan of the G chunk sums, blockDim at a time
        unsigned run = 0;
        for (unsigned base = 0; base < G; base += blockDim.x) {
            unsigned i = base + threadIdx.x;
            unsigned v = i < G ? __ldcg(&S.block_sums[i]) : 0, tot;
            unsigned ex = block_exclusive_scan(v, tot);
            if (i < G) S.block_sums[i] = run + ex;
            run += tot;
            __syncthreads();
        }
    }
    if (!bar()) return false;
    {
        unsigned run = __ldcg(&S.block_sums[rank]);
        for (unsigned base = c0; base < c1; base += blockDim.x) {
            unsigned c = base + threadIdx.x;
            unsigned v = c < c1 ? __ldcg(&S.count[c]) : 0, tot;
            unsigned ex = block_exclusive_scan(v, tot);
            if (c < c1) {
                unsigned st = run + ex;
                S.cell_start[c] = v ? st : 0xffffffffu;
                S.cell_end[c] = st + v;
                S.fill[c] = 0;
            }
            run += tot;
            __syncthreads();
        }
    }
    if (!bar()) return false;
    // 4. scatter original indices into their cell ranges
    for (unsigned k = gtid; k < np; k += gstride) {
        unsigned c = __ldcg(&S.cell_new[k]);
        unsigned pos = __ldcg(&S.cell_end[c]) - __ldcg(&S.count[c]) + atomicAdd(&S.fill[c], 1u);
        S.vals[pos] = __ldcg(&S.orig_of[k]);
    }
    if (!bar()) return false;
    // 5. order each cell by original index (stable sort order), one warp
    // per cell (warp_rank_order).  Cells of more than kCellRankMax entries
    // fall back to an insertion sort by one lane.
    {
        const unsigned lane = threadIdx.x & 31u;
        const unsigned gwarp = gtid >> 5, nwarps = gstride >> 5;
        for (unsigned c = gwarp; c < ncells; c += nwarps) {
            const unsigned n = __ldcg(&S.count[c]);
            if (n < 2) continue;
            const unsigned b = __ldcg(&S.cell_end[c]) - n;
            if (n <= kCellRankMax) {
                warp_rank_order(S.vals, b, n, lane);
            } else if (lane == 0) {
                for (unsigned i = b + 1; i < b + n; ++i) {
                    unsigned v = __ldcg(&S.vals[i]);
                    unsigned j = i;
                    while (j > b && __ldcg(&S.vals[j - 1]) > v) {
                        S.vals[j] = __ldcg(&S.vals[j - 1]);
                        --j;
                    }
                    S.vals[j] = v;
                }
            }
        }
    }
    if (!bar()) return false;
    // 6. gather the particle arrays into the new order
    for (unsigned j = gtid; j < np; j += gstride) {
        unsigned o = __ldcg(&S.vals[j]);
        unsigned k = __ldcg(&S.pos_of[o]);
        W.x[j] = ldcg4(&S.x[k]);
        W.vel[j] = ldcg4(&S.vel[k]);
        W.angvel[j] = ldcg4(&S.angvel[k]);
        W.angpos[j] = ldcg4(&S.angpos[k]);
        W.acc[j] = ldcg4(&S.acc[k]);
        W.angacc[j] = ldcg4(&S.angacc[k]);
        W.xyzsum[j] = ldcg4(&S.xyzsum[k]);
        W.es[j] = __ldcg(&S.es[k]);
        W.ev[j] = __ldcg(&S.ev[k]);
        W.cell[j] = __ldcg(&S.cell_new[k]);
    }
    if (!bar()) return false;
    // 7. commit
    for (unsigned j = gtid; j < np; j += gstride) {
        unsigned o = __ldcg(&S.vals[j]);
        double4 v = ldcg4(&W.vel[j]), w = ldcg4(&W.angvel[j]);
        S.x[j] = ldcg4(&W.x[j]);
        S.vel[j] = v;
        S.angvel[j] = w;
        S.angpos[j] = ldcg4(&W.angpos[j]);
        S.acc[j] = ldcg4(&W.acc[j]);
        S.angacc[j] = ldcg4(&W.angacc[j]);
        S.xyzsum[j] = ldcg4(&W.xyzsum[j]);
        S.es[j] = __ldcg(&W.es[j]);
        S.ev[j] = __ldcg(&W.ev[j]);
        unsigned c = __ldcg(&W.cell[j]);
        S.cell_of[j] = c;
        S.cell_new[j] = c;
        S.orig_of[j] = o;
        S.pos_of[o] = j;
        if (refresh_f && S.vel_f) {
            S.vel_f[j] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
            S.angvel_f[j] = make_float4((float)w.x, (float)w.y, (float)w.z, 0.0f);
        }
    }
    return true;
}

}  // namespace sphb
