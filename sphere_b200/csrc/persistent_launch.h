// Host entry points of the persistent step kernel (persistent.cuh).
#pragma once

#include <cuda_runtime.h>

#include "persistent.cuh"

namespace sphb {

// Block shapes the kernel is built for: threads per block and resident
// blocks per SM.  The fused step needs about 144 registers per thread; the
// first three shapes cap it at 128 (no spills to speak of), the last runs
// uncapped with fewer warps.
struct PersistShape {
    int threads, minb;
};
constexpr PersistShape kPersistShapes[] = {{64, 8}, {128, 4}, {256, 2}, {128, 3}};
constexpr int kNumPersistShapes = 4;

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

// The synchronisation block of a launch (zeroed before it): counters at
// 0 (next box), 4 (abort), 8 (any error); the sub-counter tree at 256; the
// group barriers after it.
constexpr size_t kSyncTreeOff = 256;
constexpr size_t kSyncGroupsOff = kSyncTreeOff + sizeof(GroupTree);
inline size_t sync_bytes(unsigned ngroups) { return kSyncGroupsOff + ngroups * sizeof(GroupSync); }
inline void set_sync_args(BatchArgs &A, unsigned char *sync)
{
    A.next = reinterpret_cast<unsigned *>(sync);
    A.abort = reinterpret_cast<int *>(sync + 4);
    A.any_err = reinterpret_cast<int *>(sync + 8);
    A.tree = reinterpret_cast<GroupTree *>(sync + kSyncTreeOff);
    A.groups = reinterpret_cast<GroupSync *>(sync + kSyncGroupsOff);
}

// dynamic shared memory of a launch: slot rows, at least the 16 KB stage
inline size_t persistent_smem(int threads, unsigned nc)
{
    size_t rows = (size_t)threads * nc * 4;
    return rows > 16384 ? rows : 16384;
}

}  // namespace sphb
