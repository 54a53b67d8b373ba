/* Prelude of the host build of the reference's ray-tracing kernels
 * (src/raytracer.cuh, its __global__ kernels only) -- TEST INFRASTRUCTURE
 * ONLY.  The camera and the particle count are the reference's __constant__
 * symbols; in the host build they are globals defined (by constants.cuh)
 * in ref_host.cpp and declared here. */
#ifndef REF_RT_PRELUDE_H_
#define REF_RT_PRELUDE_H_
#include "ref_shim.h"
#include "helper_math.h"
#include "typedefs.h"
extern unsigned int devC_np;
extern float3 devC_u, devC_v, devC_w, devC_eye, devC_light;
extern float4 devC_imgplane;
extern float devC_d;
extern unsigned int devC_pixels;
#endif
