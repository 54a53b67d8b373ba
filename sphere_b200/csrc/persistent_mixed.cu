// Persistent step kernel, mixed precision (FP64 overlaps and accumulation,
// FP32 contact laws), compiled with FMA contraction like the per-stage mixed
// contact kernel.
#include "persistent_launch.h"

namespace sphb {

namespace {

template <int MODEL, int NT, int MINB>
cudaError_t launch_t(const BatchArgs &A, unsigned grid, size_t smem, cudaStream_t st)
{
    auto fn = k_persistent<2, MODEL, NT, MINB>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    BatchArgs a = A;
    void *args[] = {(void *)&a};
    return cudaLaunchCooperativeKernel((void *)fn, dim3(grid), dim3(NT), args, smem, st);
}

template <int MODEL, int NT, int MINB>
int occ_t(size_t smem)
{
    auto fn = k_persistent<2, MODEL, NT, MINB>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, NT, smem) != cudaSuccess) return 0;
    return n;
}

template <int MODEL>
cudaError_t launch_shape(int shape, const BatchArgs &A, unsigned grid, size_t smem, cudaStream_t st)
{
    switch (shape) {
    case 0: return launch_t<MODEL, 64, 8>(A, grid, smem, st);
    case 1: return launch_t<MODEL, 128, 4>(A, grid, smem, st);
    case 2: return launch_t<MODEL, 256, 2>(A, grid, smem, st);
    case 3: return launch_t<MODEL, 128, 3>(A, grid, smem, st);
    default: return cudaErrorInvalidValue;
    }
}

template <int MODEL>
int occ_shape(int shape, size_t smem)
{
    switch (shape) {
    case 0: return occ_t<MODEL, 64, 8>(smem);
    case 1: return occ_t<MODEL, 128, 4>(smem);
    case 2: return occ_t<MODEL, 256, 2>(smem);
    case 3: return occ_t<MODEL, 128, 3>(smem);
    default: return 0;
    }
}

}  // namespace

cudaError_t persistent_launch_mixed(int model, int shape, const BatchArgs &A, unsigned grid,
                                    size_t smem, cudaStream_t st)
{
    return model == 2 ? launch_shape<2>(shape, A, grid, smem, st)
                      : launch_shape<1>(shape, A, grid, smem, st);
}

int persistent_blocks_per_sm_mixed(int model, int shape, size_t smem)
{
    return model == 2 ? occ_shape<2>(shape, smem) : occ_shape<1>(shape, smem);
}

}  // namespace sphb
