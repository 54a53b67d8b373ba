// Host-side launchers of the DEM kernels.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "dem_state.h"

namespace sphb {

// prec: 0 faithful FP64 (FP32 lengths), 1 FP64.  staged = 1: contact model 2
// reads its partners from the neighbour cells staged in shared memory
// (k_contacts_staged); 0 walks the neighbour lists through global memory
// (k_contacts).
cudaError_t launch_contacts(const DevParams &P, const DevState &S, int prec, cudaStream_t st,
                            int staged = 0);
// mixed precision: FP64 overlaps, FP32 contact laws, FP64 accumulation
cudaError_t launch_contacts_mixed(const DevParams &P, const DevState &S, cudaStream_t st,
                                  int staged = 0);
// Shared memory of the staged contact kernel: bytes per block and the
// staging capacity (particles) for nc slots per particle.
void staged_contact_shape(unsigned nc, size_t per_particle, size_t &smem, unsigned &cap);
// Contacts and particle integration of one step in one launch
// (k_contacts_integrate): reads the current buffers of S, integrates into
// S.x_nx / vel_nx / angvel_nx (and the FP32 copies).  Only for dry boxes
// without bonds or a shear-stress wall; launch_walls_step completes the step.
cudaError_t launch_contacts_integrate(const DevParams &P, const DevState &S, int prec,
                                      cudaStream_t st);
cudaError_t launch_contacts_integrate_mixed(const DevParams &P, const DevState &S, cudaStream_t st);
// wall reduction, wall update, loop counters and the next step's flags after
// launch_contacts_integrate
cudaError_t launch_walls_step(const DevParams &P, const DevState &S, cudaStream_t st);
cudaError_t launch_bonds(const DevParams &P, const DevState &S, int prec, double4 *bond_f,
                         double4 *bond_t, cudaStream_t st);
// shear-stress reduction (wmode 3), then one kernel: integration, wall
// reduction + wall integration, loop counters
cudaError_t launch_integrate(const DevParams &P, const DevState &S, cudaStream_t st);
cudaError_t launch_occ_from_rows(const DevParams &P, const DevState &S, cudaStream_t st);
cudaError_t launch_hash(const DevParams &P, const DevState &S, cudaStream_t st);
// positions from the host (ORIGINAL order, device memory) into the sorted
// storage, raising the re-sort and list flags where a particle changed cell,
// left its list skin or changed radius
cudaError_t launch_set_positions(const DevParams &P, const DevState &S, const double4 *src,
                                 cudaStream_t st);
// force = 1 sorts unconditionally; otherwise only when DevCtl::resort is
// set.  with_nl = 1 also rebuilds the neighbour lists in the same launch
// when they are stale (DevCtl::nl_rebuild) or the sort ran.
cudaError_t launch_resort(const DevParams &P, const DevState &S, unsigned char *scratch,
                          int force, cudaStream_t st, int with_nl = 0);
size_t resort_scratch_bytes(size_t np);

// Gathers sorted storage into original order: dst[orig_of[k]] = src[k].
cudaError_t launch_unsort(const void *src, void *dst, const uint32_t *orig_of, size_t np,
                          size_t elem_bytes, cudaStream_t st);
// Scatters original order into sorted storage: dst[k] = src[orig_of[k]].
cudaError_t launch_sort_into(const void *src, void *dst, const uint32_t *orig_of, size_t np,
                             size_t elem_bytes, cudaStream_t st);

}  // namespace sphb
