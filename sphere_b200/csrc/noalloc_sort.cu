// Cell sort of particle positions that allocates nothing: sph_sort_cells_noalloc.
//
// Same result as the engine's cell sort (stable order by (cell, original
// index), cellStart/cellEnd), but every scratch word it needs -- per-cell
// counts, per-cell fill counters, per-tile sums and an error flag -- sits in
// one file-scope device array below.  The caller passes the positions and
// the four output arrays; nothing here calls cudaMalloc, cudaFree or an
// allocating library routine.
#include <cstdint>
#include <cstdio>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/sphere_b200.h"
#include "cell_order.cuh"

namespace sphb {
namespace {

constexpr uint32_t kMaxCells = SPH_NOALLOC_MAX_CELLS;
constexpr uint32_t kTile = 1024;                      // cells per scan tile
constexpr uint32_t kMaxTiles = kMaxCells / kTile;     // 1024
// layout (32-bit words): count[kMaxCells] | fill[kMaxCells] | tiles[kMaxTiles] | err, err_index
constexpr size_t kOffCount = 0;
constexpr size_t kOffFill = kMaxCells;
constexpr size_t kOffTiles = 2 * (size_t)kMaxCells;
constexpr size_t kOffErr = kOffTiles + kMaxTiles;
constexpr size_t kWords = kOffErr + 64;
static_assert(kCellRankMax == SPH_NOALLOC_MAX_PER_CELL, "per-cell limit of the header");

// Scratch shared by every call of sph_sort_cells_noalloc on a device.  It is
// resident on every GPU that loads this library (about 8.4 MB) until exit.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kWords];

struct Grid {
    double origo[3], cell[3];
    uint32_t num[3];
    uint32_t ncells;
};

__device__ __forceinline__ bool cell_of(const Grid &g, const double *x4, uint32_t i, uint32_t &c)
{
    double p[3] = {x4[4 * (size_t)i], x4[4 * (size_t)i + 1], x4[4 * (size_t)i + 2]};
    uint32_t ic[3];
    for (int d = 0; d < 3; ++d) {
        double f = floor((p[d] - g.origo[d]) / g.cell[d]);
        if (!(f >= 0.0) || f >= (double)g.num[d]) return false;
        ic[d] = (uint32_t)f;
    }
    c = (ic[2] * g.num[1]) * g.num[0] + ic[1] * g.num[0] + ic[0];
    return true;
}

__global__ void k_na_clear(uint32_t *scr, uint32_t ncells)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ncells) {
        scr[kOffCount + i] = 0;
        scr[kOffFill + i] = 0;
    }
    if (i == 0) {
        scr[kOffErr] = 0;
        scr[kOffErr + 1] = 0xffffffffu;
    }
}

__global__ void k_na_count(const double *x4, uint32_t np, Grid g, uint32_t *scr)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    uint32_t c;
    if (!cell_of(g, x4, i, c)) {
        if (atomicCAS(&scr[kOffErr], 0u, 1u) == 0u) scr[kOffErr + 1] = i;
        return;
    }
    atomicAdd(&scr[kOffCount + c], 1u);
}

// inclusive scan of one value per thread over a 1024-thread block
__device__ uint32_t block_incl_scan(uint32_t v, uint32_t *warp_tot)
{
    uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (uint32_t)o) v += y;
    }
    if (lane == 31) warp_tot[wid] = v;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = warp_tot[lane];
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        warp_tot[lane] = w;
    }
    __syncthreads();
    uint32_t r = v + (wid ? warp_tot[wid - 1] : 0);
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(1024) k_na_tile_sums(uint32_t *scr, uint32_t ncells)
{
    __shared__ uint32_t warp_tot[32];
    uint32_t c = blockIdx.x * kTile + threadIdx.x;
    uint32_t v = c < ncells ? scr[kOffCount + c] : 0;
    uint32_t s = block_incl_scan(v, warp_tot);
    if (threadIdx.x == kTile - 1) scr[kOffTiles + blockIdx.x] = s;
}

__global__ void __launch_bounds__(1024) k_na_scan_tiles(uint32_t *scr, uint32_t ntiles)
{
    __shared__ uint32_t warp_tot[32];
    uint32_t t = threadIdx.x;
    uint32_t v = t < ntiles ? scr[kOffTiles + t] : 0;
    uint32_t s = block_incl_scan(v, warp_tot);
    if (t < ntiles) scr[kOffTiles + t] = s - v;  // exclusive
}

__global__ void __launch_bounds__(1024) k_na_apply(uint32_t *scr, uint32_t ncells,
                                                    uint32_t *cell_start, uint32_t *cell_end)
{
    __shared__ uint32_t warp_tot[32];
    uint32_t c = blockIdx.x * kTile + threadIdx.x;
    uint32_t v = c < ncells ? scr[kOffCount + c] : 0;
    uint32_t s = block_incl_scan(v, warp_tot);
    if (c < ncells) {
        uint32_t st = scr[kOffTiles + blockIdx.x] + s - v;
        cell_start[c] = v ? st : 0xffffffffu;
        cell_end[c] = st + v;
    }
}

__global__ void k_na_scatter(const double *x4, uint32_t np, Grid g, uint32_t *scr,
                             const uint32_t *cell_end, uint32_t *index)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np || scr[kOffErr]) return;
    uint32_t c;
    if (!cell_of(g, x4, i, c)) return;
    uint32_t pos = cell_end[c] - scr[kOffCount + c] + atomicAdd(&scr[kOffFill + c], 1u);
    index[pos] = i;
}

// Orders each cell's entries by original index (the stable sort order),
// one warp per cell with the engine's register ranks, and writes the sorted
// cell keys.  A cell of more than kCellRankMax entries is not ordered: it
// raises error 2 (a grid far coarser than the contact search uses), so no
// call runs a quadratic loop over a crowded cell.
__global__ void k_na_cells(uint32_t *scr, uint32_t ncells, const uint32_t *cell_end,
                           uint32_t *index, uint32_t *cellid)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= ncells || scr[kOffErr]) return;
    const uint32_t n = scr[kOffCount + c];
    if (n == 0) return;
    const uint32_t b = cell_end[c] - n;
    if (n > kCellRankMax) {
        if (lane == 0 && atomicCAS(&scr[kOffErr], 0u, 2u) == 0u) scr[kOffErr + 1] = c;
        return;
    }
    if (n > 1) warp_rank_order(index, b, n, lane);
    for (uint32_t i = b + lane; i < b + n; i += 32u) cellid[i] = c;
}

// Device address of g_noalloc_scratch, looked up once per device.
std::mutex g_mu;
uint32_t *g_scratch_ptr[64] = {};
// message of the calling thread's last failure
thread_local char g_err[256];

int scratch_for_current_device(uint32_t **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        std::snprintf(g_err, sizeof g_err, "no usable current CUDA device (%s)",
                      cudaGetErrorString(e));
        return SPH_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            std::snprintf(g_err, sizeof g_err, "cudaGetSymbolAddress failed on device %d: %s",
                          dev, cudaGetErrorString(e));
            return SPH_ERR_CUDA;
        }
        g_scratch_ptr[dev] = (uint32_t *)p;
    }
    *out = g_scratch_ptr[dev];
    return SPH_OK;
}

}  // namespace
}  // namespace sphb

extern "C" int sph_sort_cells_noalloc(const double *x4, uint32_t np, const double origo[3],
                                      const double L[3], const uint32_t num[3], uint32_t *cellid,
                                      uint32_t *index, uint32_t *cell_start, uint32_t *cell_end,
                                      void *stream)
{
    using namespace sphb;
    if (!origo || !L || !num || (np && (!x4 || !cellid || !index)) || !cell_start || !cell_end) {
        std::snprintf(g_err, sizeof g_err, "null pointer argument");
        return SPH_ERR_ARG;
    }
    uint64_t ncells = (uint64_t)num[0] * num[1] * num[2];
    if (ncells == 0 || ncells > kMaxCells) {
        std::snprintf(g_err, sizeof g_err,
                      "grid of %llu cells is outside 1..%u, the size of the built-in scratch",
                      (unsigned long long)ncells, kMaxCells);
        return SPH_ERR_ARG;
    }
    uint32_t *scr = nullptr;
    int rc = scratch_for_current_device(&scr);
    if (rc) return rc;
    Grid g;
    for (int d = 0; d < 3; ++d) {
        g.origo[d] = origo[d];
        g.cell[d] = L[d] / num[d];
        g.num[d] = num[d];
    }
    g.ncells = (uint32_t)ncells;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t nc = g.ncells, ntiles = (nc + kTile - 1) / kTile;
    k_na_clear<<<(nc + 255) / 256, 256, 0, st>>>(scr, nc);
    if (np) k_na_count<<<(np + 255) / 256, 256, 0, st>>>(x4, np, g, scr);
    k_na_tile_sums<<<ntiles, kTile, 0, st>>>(scr, nc);
    k_na_scan_tiles<<<1, kTile, 0, st>>>(scr, ntiles);
    k_na_apply<<<ntiles, kTile, 0, st>>>(scr, nc, cell_start, cell_end);
    if (np) k_na_scatter<<<(np + 255) / 256, 256, 0, st>>>(x4, np, g, scr, cell_end, index);
    k_na_cells<<<(unsigned)(((uint64_t)nc * 32 + 255) / 256), 256, 0, st>>>(scr, nc, cell_end, index,
                                                                               cellid);
    cudaError_t e = cudaGetLastError();
    uint32_t flag[2] = {0, 0};
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(flag, scr + kOffErr, sizeof flag, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        std::snprintf(g_err, sizeof g_err, "CUDA error: %s", cudaGetErrorString(e));
        return SPH_ERR_CUDA;
    }
    if (flag[0] == 2) {
        std::snprintf(g_err, sizeof g_err,
                      "cell %u holds more than %u particles: the grid is too coarse", flag[1],
                      kCellRankMax);
        return SPH_ERR_ARG;
    }
    if (flag[0]) {
        std::snprintf(g_err, sizeof g_err, "particle %u is outside the grid or not finite", flag[1]);
        return SPH_ERR_OUTSIDE;
    }
    return SPH_OK;
}

extern "C" const char *sph_noalloc_error(void) { return sphb::g_err; }
