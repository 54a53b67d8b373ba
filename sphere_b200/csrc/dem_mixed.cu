// Mixed-precision DEM contact kernel: the shared contact kernel template
// instantiated with FP64 overlaps, FP32 contact laws and FP64 accumulation
// (compiled with FMA contraction, unlike the FP64 kernels).
#include "dem_device.cuh"
#include "contacts_staged.cuh"
#include "dem_launch.h"
#include "engine_internal.h"

namespace sphb {

cudaError_t launch_contacts_mixed(const DevParams &P, const DevState &S, cudaStream_t st,
                                  int staged)
{
    if (P.np == 0) return cudaSuccess;
    if (P.contactmodel == 2 && staged) {
        size_t smem;
        unsigned cap;
        staged_contact_shape(P.nc, stage_bytes_per_particle<2>(), smem, cap);
        static size_t attr = 0;
        if (attr < smem) {
            cudaFuncSetAttribute(k_contacts_staged<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            attr = smem;
        }
        dim3 grid((P.np + SPHB_STAGED_B - 1) / SPHB_STAGED_B);
        k_contacts_staged<2><<<grid, SPHB_STAGED_B, smem, st>>>(P, S, cap);
        return cudaGetLastError();
    }
    const unsigned B = SPHB_CONTACT_B;
    dim3 grid((P.np + B - 1) / B);
    if (P.contactmodel == 2) {
        size_t smem = (size_t)B * P.nc * sizeof(uint32_t);
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_contacts<2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)((size_t)B * 64 * sizeof(uint32_t)));
            attr = true;
        }
        k_contacts<2, 2><<<grid, B, smem, st>>>(P, S);
    } else {
        k_contacts<2, 1><<<grid, B, 0, st>>>(P, S);
    }
    return cudaGetLastError();
}

cudaError_t launch_contacts_integrate_mixed(const DevParams &P, const DevState &S, cudaStream_t st)
{
    if (P.np == 0) return cudaSuccess;
    const unsigned B = SPHB_CONTACT_B;
    dim3 grid((P.np + B - 1) / B);
    if (P.contactmodel == 2) {
        size_t smem = (size_t)B * P.nc * sizeof(uint32_t);
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_contacts_integrate<2, 2>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)((size_t)B * 64 * sizeof(uint32_t)));
            attr = true;
        }
        k_contacts_integrate<2, 2><<<grid, B, smem, st>>>(P, S);
    } else {
        k_contacts_integrate<2, 1><<<grid, B, 0, st>>>(P, S);
    }
    return cudaGetLastError();
}

int Engine::mixed_init() { return ST_OK; }

}  // namespace sphb
