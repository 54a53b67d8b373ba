// Device-resident state of one engine.
//
// Particle arrays live in SORTED order (position k = k-th particle of the
// current cell sort) and are permuted only when some particle changes cell;
// contact history rows are keyed by ORIGINAL particle index, as in the
// reference (src/contactsearch.cuh:273,286), so they survive re-sorts.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dev_common.cuh"

namespace sphb {

struct DevState {
    // sorted particle storage (the reference's Float4 layout per particle)
    double4 *x, *vel, *angvel, *angpos, *acc, *angacc, *xyzsum, *force, *torque;
    double *es_dot, *es, *ev_dot, *ev, *p;
    uint32_t *orig_of;     // sorted position -> original index
    uint32_t *pos_of;      // original index -> sorted position
    uint32_t *cell_of;     // sorted position -> cell of the current sort
    uint32_t *cell_new;    // sorted position -> cell after the last integration
    uint32_t *cell_start, *cell_end;

    // contact history, np * nc slots keyed by original index
    uint32_t *contacts;    // partner original index, np = empty
    uint8_t *dmcode;       // periodic shift of the slot (dm_encode)
    double4 *delta_t;      // tangential displacement (x, y, z, 0)
    uint64_t *occ;         // occupied-slot bitmask per original index (nc <= 64)

    // mixed precision only (null otherwise): FP32 copies of the velocities
    // in sorted order and FP32 tangential history per slot
    float4 *vel_f, *angvel_f, *delta_t_f;

    // the other buffer of the ping-pong pairs the fused step integrates into
    // (the per-stage kernels integrate in place and never touch them)
    double4 *x_nx, *vel_nx, *angvel_nx;
    float4 *vel_f_nx, *angvel_f_nx;

    // neighbour lists in sorted order: entry j of particle k at nl[j*np + k]
    // = sorted index | periodic shift code << 28
    uint32_t *nl, *nl_count;
    float4 *x_ref;         // position at the last list build

    // walls
    double4 *wnx, *wmvfd;
    double *wacc;
    double *walls_force_pp;   // nw * np, ORIGINAL order (reduced like the reference)
    double *tau_pp;           // np, ORIGINAL order
    double *partials;         // nblocks256
    double *tau_partials;     // nblocks256

    // bonds (original particle indices)
    uint2 *bonds;
    double4 *bonds_delta, *bonds_omega;
    // per-particle bond lists (CSR over original index) for gather accumulation
    uint32_t *bond_ptr, *bond_list;

    // sort scratch
    uint32_t *count, *fill, *vals, *block_sums;
    // permutation scratch (raw bytes, sized for every per-particle array)
    unsigned char *perm_scratch;

    DevCtl *ctl;
};

}  // namespace sphb
