// Persistent step kernel, FP64 modes (faithful and true FP64), compiled with
// -fmad=false like the per-stage FP64 kernels so both paths round alike.
#include "persistent_launch.h"

namespace sphb {

namespace {

template <int PREC, int MODEL, int NT, int MINB>
cudaError_t launch_t(const BatchArgs &A, unsigned grid, size_t smem, cudaStream_t st)
{
    auto fn = k_persistent<PREC, MODEL, NT, MINB>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    BatchArgs a = A;
    void *args[] = {(void *)&a};
    return cudaLaunchCooperativeKernel((void *)fn, dim3(grid), dim3(NT), args, smem, st);
}

template <int PREC, int MODEL, int NT, int MINB>
int occ_t(size_t smem)
{
    auto fn = k_persistent<PREC, MODEL, NT, MINB>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, NT, smem) != cudaSuccess) return 0;
    return n;
}

template <int PREC, int MODEL>
cudaError_t launch_shape(int shape, const BatchArgs &A, unsigned grid, size_t smem, cudaStream_t st)
{
    switch (shape) {
    case 0: return launch_t<PREC, MODEL, 64, 8>(A, grid, smem, st);
    case 1: return launch_t<PREC, MODEL, 128, 4>(A, grid, smem, st);
    case 2: return launch_t<PREC, MODEL, 256, 2>(A, grid, smem, st);
    case 3: return launch_t<PREC, MODEL, 128, 3>(A, grid, smem, st);
    default: return cudaErrorInvalidValue;
    }
}

template <int PREC, int MODEL>
int occ_shape(int shape, size_t smem)
{
    switch (shape) {
    case 0: return occ_t<PREC, MODEL, 64, 8>(smem);
    case 1: return occ_t<PREC, MODEL, 128, 4>(smem);
    case 2: return occ_t<PREC, MODEL, 256, 2>(smem);
    case 3: return occ_t<PREC, MODEL, 128, 3>(smem);
    default: return 0;
    }
}

}  // namespace

cudaError_t persistent_launch_fp64(int prec, int model, int shape, const BatchArgs &A,
                                   unsigned grid, size_t smem, cudaStream_t st)
{
    if (prec == 0) return model == 2 ? launch_shape<0, 2>(shape, A, grid, smem, st)
                                     : launch_shape<0, 1>(shape, A, grid, smem, st);
    return model == 2 ? launch_shape<1, 2>(shape, A, grid, smem, st)
                      : launch_shape<1, 1>(shape, A, grid, smem, st);
}

int persistent_blocks_per_sm_fp64(int prec, int model, int shape, size_t smem)
{
    if (prec == 0) return model == 2 ? occ_shape<0, 2>(shape, smem) : occ_shape<0, 1>(shape, smem);
    return model == 2 ? occ_shape<1, 2>(shape, smem) : occ_shape<1, 1>(shape, smem);
}

cudaError_t persistent_launch(int prec, int model, int shape, const BatchArgs &A, unsigned grid,
                              size_t smem, cudaStream_t st)
{
    if (prec == 2) return persistent_launch_mixed(model, shape, A, grid, smem, st);
    return persistent_launch_fp64(prec, model, shape, A, grid, smem, st);
}

int persistent_blocks_per_sm(int prec, int model, int shape, size_t smem)
{
    if (prec == 2) return persistent_blocks_per_sm_mixed(model, shape, smem);
    return persistent_blocks_per_sm_fp64(prec, model, shape, smem);
}

}  // namespace sphb
