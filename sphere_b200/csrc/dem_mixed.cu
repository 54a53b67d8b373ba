// Mixed-precision DEM contact kernel: the shared contact kernel template
// instantiated with FP64 overlaps, FP32 contact laws and FP64 accumulation
// (compiled with FMA contraction, unlike the FP64 kernels).
#include "dem_device.cuh"
#include "dem_launch.h"
#include "engine_internal.h"

namespace sphb {

cudaError_t launch_contacts_mixed(const DevParams &P, const DevState &S, cudaStream_t st)
{
    if (P.np == 0) return cudaSuccess;
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

int Engine::mixed_init() { return ST_OK; }

}  // namespace sphb
