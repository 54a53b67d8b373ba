// Host entry points of the persistent step kernel (persistent.cuh).
#pragma once

#include <cuda_runtime.h>

#include "persistent.cuh"

namespace sphb {

// Block shapes the kernel is built for: threads per block and resident
// blocks per SM (the same 80-register budget).
struct PersistShape {
    int threads, minb;
};
constexpr PersistShape kPersistShapes[] = {{64, 12}, {128, 6}, {256, 3}};
constexpr int kNumPersistShapes = 3;

// prec: SPH_PREC_* (0 faithful, 1 FP64 in persistent_fp64.cu; 2 mixed in
// persistent_mixed.cu); model: 1 or 2; shape: index into kPersistShapes.
cudaError_t persistent_launch(int prec, int model, int shape, const BatchArgs &A, unsigned grid,
                              size_t smem, cudaStream_t st);
// Resident blocks per SM of that instantiation with `smem` dynamic bytes.
int persistent_blocks_per_sm(int prec, int model, int shape, size_t smem);

// per-translation-unit halves
cudaError_t persistent_launch_fp64(int prec, int model, int shape, const BatchArgs &A,
                                   unsigned grid, size_t smem, cudaStream_t st);
int persistent_blocks_per_sm_fp64(int prec, int model, int shape, size_t smem);
cudaError_t persistent_launch_mixed(int model, int shape, const BatchArgs &A, unsigned grid,
                                    size_t smem, cudaStream_t st);
int persistent_blocks_per_sm_mixed(int model, int shape, size_t smem);

// dynamic shared memory of a launch: slot rows, at least the 16 KB stage
inline size_t persistent_smem(int threads, unsigned nc)
{
    size_t rows = (size_t)threads * nc * 4;
    return rows > 16384 ? rows : 16384;
}

}  // namespace sphb
