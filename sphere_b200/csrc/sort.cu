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
#include "resort_device.cuh"
#include "dem_device.cuh"

#include <cooperative_groups.h>

namespace sphb {

// Grid-wide barrier for a cooperative launch, with a bounded wait: after
// ~2^24 polls (well over a second) it records DERR_TIMEOUT and returns
// false instead of spinning forever.  With `inject` no block releases it and
// every block gives up after kInjectPolls polls.
__device__ bool grid_barrier(DevCtl *ctl, unsigned nblocks, bool inject)
{
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        volatile unsigned *gen = &ctl->barrier_gen;
        unsigned g = *gen;
        __threadfence();
        unsigned arrived = atomicAdd(&ctl->barrier_count, 1u);
        ok = 1;
        if (arrived == nblocks - 1 && !inject) {
            ctl->barrier_count = 0;
            __threadfence();
            atomicAdd(&ctl->barrier_gen, 1u);
        } else {
            unsigned spins = 0;
            const unsigned limit = inject ? kInjectPolls : (1u << 24);
            while (inject || *gen == g) {
                if (++spins > limit) {
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

// The pre-contact work of a step in one launch: the re-sort when a
// particle changed cell (or `force`), then, with `with_nl`, the neighbour
// lists when they are stale or the sort changed the indices.  Both flags
// come from the previous step's integration, so every block reads the same
// decision.
__global__ void __launch_bounds__(256, 3) k_resort(DevParams P, DevState S, PermScratch W, int force,
                                                int with_nl)
{
    DevCtl *ctl = S.ctl;
    if (ctl->err) return;
    const bool resort = force || ctl->resort;
    const bool nl = with_nl && (resort || ctl->nl_rebuild);
    if (!resort && !nl) return;
    const bool inject = (P.inject & kInjectResort) != 0;
    auto bar = [&]() { return grid_barrier(ctl, gridDim.x, inject); };
    if (resort) {
        // the FP32 velocity copies of the mixed mode follow the permutation
        if (!resort_group(P, S, W, gridDim.x, blockIdx.x, bar, true)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ctl->resort = 0;
            ctl->resorts += 1;
            ctl->nl_rebuild = 1;   // sorted indices changed (k_contacts clears it)
        }
        if (nl && !bar()) return;
    }
    if (nl) {
        const unsigned stride = gridDim.x * blockDim.x;
        for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < P.np; k += stride)
            nl_build_particle(P, S, k);
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->nl_builds += 1;
    }
}

static int g_resort_grid = 0;

cudaError_t launch_resort(const DevParams &P, const DevState &S, unsigned char *scratch,
                          int force, cudaStream_t st, int with_nl)
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
    PermScratch W = make_perm_scratch(scratch, P.np);
    unsigned grid = g_resort_grid;
    unsigned need = (P.np + 255) / 256;
    if (need < grid) grid = need < 1 ? 1 : need;
    DevParams Pc = P;
    DevState Sc = S;
    void *args[] = {(void *)&Pc, (void *)&Sc, (void *)&W, (void *)&force, (void *)&with_nl};
    return cudaLaunchCooperativeKernel((void *)k_resort, dim3(grid), dim3(256), args, 0, st);
}

size_t resort_scratch_bytes(size_t np) { return perm_scratch_bytes(np); }

}  // namespace sphb
