/* Stand-ins for reference members that the DEM step does not use but the
 * linked host sources reference -- TEST INFRASTRUCTURE ONLY. */
#include <cstdio>
#include <cstdlib>
#include "sphere.h"
#include <cstring>
#include <cuda_runtime_api.h>

static void unused(const char *what)
{
    std::fprintf(stderr, "reference host build: %s is not part of this build\n", what);
    std::abort();
}

/* Host stand-ins for the CUDA runtime calls the reference's device-memory
 * code makes (cudaMalloc/cudaMemcpy/...): "device" memory is host memory
 * in this build, so the reference's own transfer code runs unchanged. */
extern "C" {
cudaError_t cudaMalloc(void **p, size_t n) { *p = std::calloc(n ? n : 1, 1); return *p ? cudaSuccess : cudaErrorMemoryAllocation; }
cudaError_t cudaFree(void *p) { std::free(p); return cudaSuccess; }
cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) { std::memmove(d, s, n); return cudaSuccess; }
cudaError_t cudaMemset(void *d, int v, size_t n) { std::memset(d, v, n); return cudaSuccess; }
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
cudaError_t cudaPeekAtLastError(void) { return cudaSuccess; }
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaThreadSynchronize(void) { return cudaSuccess; }
const char *cudaGetErrorString(cudaError_t) { return "no error"; }
}
