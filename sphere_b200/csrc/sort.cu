// Cell sort of the particles (the reference's calcParticleCellID +
// thrust::sort_by_key + reorderArrays, src/sorting.cuh:25-132,
// src/device.cu:1066-1114), as one cooperative kernel.
//
// The reference sorts (cellID, index) pairs with a stable radix sort every
// step.  Here the particle arrays stay in sorted order between steps and
// are re-sorted only when some particle's cell changed (the integration
// kernel raises DevCtl::resort).  A stable sort of unchanged keys is the
// identity, so skipping it is exact.  The sort itself is a bucket sort on
// cells: count per cell, exclusive scan (cellStart/cellEnd), atomic
// scatter, then each cell's few entries are ordered by original index,
// which gives exactly the stable (cellID, index) order.
#include "dem_state.h"
#include "dem_launch.h"

#include <cooperative_groups.h>

namespace sphb {

// Grid-wide barrier for a cooperative launch, with a bounded wait: after
// ~2^24 polls (well over a second) it records DERR_TIMEOUT and returns
// false instead of spinning forever.
__device__ bool grid_barrier(DevCtl *ctl, unsigned nblocks)
{
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        volatile unsigned *gen = &ctl->barrier_gen;
        unsigned g = *gen;
        __threadfence();
        unsigned arrived = atomicAdd(&ctl->barrier_count, 1u);
        ok = 1;
        if (arrived == nblocks - 1) {
            ctl->barrier_count = 0;
            __threadfence();
            atomicAdd(&ctl->barrier_gen, 1u);
        } else {
            unsigned spins = 0;
            while (*gen == g) {
                if (++spins > (1u << 24)) {
                    raise_err(ctl, DERR_TIMEOUT, -1);
                    ok = 0;
                    break;
                }
                if (((volatile int *)&ctl->err)[0] == DERR_TIMEOUT) { ok = 0; break; }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Block-wide exclusive scan of one value per thread (256 threads).
__device__ unsigned block_exclusive_scan(unsigned v, unsigned &total)
{
    __shared__ unsigned warp_tot[8];
    unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned x = v;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned w = lane < 8 ? warp_tot[lane] : 0;
        for (int o = 1; o < 8; o <<= 1) {
            unsigned y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (unsigned)o) w += y;
        }
        if (lane < 8) warp_tot[lane] = w;  // inclusive warp prefix
    }
    __syncthreads();
    unsigned before = wid ? warp_tot[wid - 1] : 0;
    total = warp_tot[7];
    __syncthreads();
    return before + x - v;
}

struct PermScratch {
    double4 *x, *vel, *angvel, *angpos, *acc, *angacc, *xyzsum, *f_p;
    double *es, *ev;
    uint32_t *cell;
};

__global__ void __launch_bounds__(256) k_resort(DevParams P, DevState S, PermScratch W, int force)
{
    DevCtl *ctl = S.ctl;
    if (ctl->err) return;
    if (!force && !ctl->resort) return;
    const unsigned G = gridDim.x;
    const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned gstride = G * blockDim.x;
    const unsigned np = P.np, ncells = P.ncells;

    // 1. zero the per-cell counts
    for (unsigned c = gtid; c < ncells; c += gstride) S.count[c] = 0;
    if (!grid_barrier(ctl, G)) return;
    // 2. count particles per cell
    for (unsigned k = gtid; k < np; k += gstride) atomicAdd(&S.count[S.cell_new[k]], 1u);
    if (!grid_barrier(ctl, G)) return;
    // 3. exclusive scan of the counts over contiguous chunks of cells
    const unsigned chunk = (ncells + G - 1) / G;
    const unsigned c0 = min(blockIdx.x * chunk, ncells), c1 = min(c0 + chunk, ncells);
    {
        __shared__ unsigned red[256];
        unsigned s = 0;
        for (unsigned c = c0 + threadIdx.x; c < c1; c += blockDim.x) s += S.count[c];
        red[threadIdx.x] = s;
        __syncthreads();
        for (unsigned i = 128; i; i >>= 1) {
            if (threadIdx.x < i) red[threadIdx.x] += red[threadIdx.x + i];
            __syncthreads();
        }
        if (threadIdx.x == 0) S.block_sums[blockIdx.x] = red[0];
    }
    if (!grid_barrier(ctl, G)) return;
    if (blockIdx.x == 0) {
        // exclusive scan of the G block sums, 256 at a time
        unsigned run = 0;
        for (unsigned base = 0; base < G; base += blockDim.x) {
            unsigned i = base + threadIdx.x;
            unsigned v = i < G ? S.block_sums[i] : 0, tot;
            unsigned ex = block_exclusive_scan(v, tot);
            if (i < G) S.block_sums[i] = run + ex;
            run += tot;
            __syncthreads();
        }
    }
    if (!grid_barrier(ctl, G)) return;
    {
        unsigned run = S.block_sums[blockIdx.x];
        for (unsigned base = c0; base < c1; base += blockDim.x) {
            unsigned c = base + threadIdx.x;
            unsigned v = c < c1 ? S.count[c] : 0, tot;
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
    if (!grid_barrier(ctl, G)) return;
    // 4. scatter original indices into their cell ranges
    for (unsigned k = gtid; k < np; k += gstride) {
        unsigned c = S.cell_new[k];
        unsigned pos = S.cell_end[c] - S.count[c] + atomicAdd(&S.fill[c], 1u);
        S.vals[pos] = S.orig_of[k];
    }
    if (!grid_barrier(ctl, G)) return;
    // 5. order each cell by original index (stable sort order)
    for (unsigned c = gtid; c < ncells; c += gstride) {
        unsigned n = S.count[c];
        if (n < 2) continue;
        unsigned b = S.cell_end[c] - n;
        for (unsigned i = b + 1; i < b + n; ++i) {
            unsigned v = S.vals[i];
            unsigned j = i;
            while (j > b && S.vals[j - 1] > v) {
                S.vals[j] = S.vals[j - 1];
                --j;
            }
            S.vals[j] = v;
        }
    }
    if (!grid_barrier(ctl, G)) return;
    // 6. gather the particle arrays into the new order
    for (unsigned j = gtid; j < np; j += gstride) {
        unsigned o = S.vals[j];
        unsigned k = S.pos_of[o];
        W.x[j] = S.x[k];
        W.vel[j] = S.vel[k];
        W.angvel[j] = S.angvel[k];
        W.angpos[j] = S.angpos[k];
        W.acc[j] = S.acc[k];
        W.angacc[j] = S.angacc[k];
        W.xyzsum[j] = S.xyzsum[k];
        W.es[j] = S.es[k];
        W.ev[j] = S.ev[k];
        W.cell[j] = S.cell_new[k];
    }
    if (!grid_barrier(ctl, G)) return;
    // 7. commit
    for (unsigned j = gtid; j < np; j += gstride) {
        unsigned o = S.vals[j];
        S.x[j] = W.x[j];
        S.vel[j] = W.vel[j];
        S.angvel[j] = W.angvel[j];
        S.angpos[j] = W.angpos[j];
        S.acc[j] = W.acc[j];
        S.angacc[j] = W.angacc[j];
        S.xyzsum[j] = W.xyzsum[j];
        S.es[j] = W.es[j];
        S.ev[j] = W.ev[j];
        S.cell_of[j] = W.cell[j];
        S.cell_new[j] = W.cell[j];
        S.orig_of[j] = o;
        S.pos_of[o] = j;
    }
    if (gtid == 0) {
        ctl->resort = 0;
        ctl->resorts += 1;
        ctl->nl_rebuild = 1;   // sorted indices changed
    }
}

static int g_resort_grid = 0;

cudaError_t launch_resort(const DevParams &P, const DevState &S, unsigned char *scratch,
                          int force, cudaStream_t st)
{
    if (P.np == 0) return cudaSuccess;
    if (g_resort_grid == 0) {
        int dev, sms, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_resort, 256, 0);
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        g_resort_grid = sms * (per_sm < 4 ? per_sm : 4);
    }
    PermScratch W;
    size_t n = P.np;
    unsigned char *p = scratch;
    auto take = [&](size_t bytes) {
        unsigned char *q = p;
        p += (bytes + 255) & ~(size_t)255;
        return q;
    };
    W.x = (double4 *)take(n * 32); W.vel = (double4 *)take(n * 32);
    W.angvel = (double4 *)take(n * 32); W.angpos = (double4 *)take(n * 32);
    W.acc = (double4 *)take(n * 32); W.angacc = (double4 *)take(n * 32);
    W.xyzsum = (double4 *)take(n * 32); W.f_p = (double4 *)take(n * 32);
    W.es = (double *)take(n * 8); W.ev = (double *)take(n * 8);
    W.cell = (uint32_t *)take(n * 4);
    unsigned grid = g_resort_grid;
    unsigned need = (P.np + 255) / 256;
    if (need < grid) grid = need < 1 ? 1 : need;
    DevParams Pc = P;
    DevState Sc = S;
    void *args[] = {(void *)&Pc, (void *)&Sc, (void *)&W, (void *)&force};
    return cudaLaunchCooperativeKernel((void *)k_resort, dim3(grid), dim3(256), args, 0, st);
}

size_t resort_scratch_bytes(size_t np)
{
    return 8 * ((np * 32 + 255) & ~(size_t)255) + 2 * ((np * 8 + 255) & ~(size_t)255) +
           ((np * 4 + 255) & ~(size_t)255) + 256;
}

}  // namespace sphb
