// Darcy porosity-coupled pressure solver (cfd_solver 1).
#include "engine_internal.h"
#include "../../include/sphere_b200.h"

namespace sphb {

int Engine::darcy_init()
{
    if (!hs.fluid) return ST_OK;
    return fail(ST_UNSUPPORTED, "Darcy solver not built yet");
}
int64_t Engine::darcy_field_bytes(int) const { return -1; }
int Engine::darcy_get(int, void *, size_t) { return fail(ST_ARG, "unknown field"); }
int Engine::darcy_download() { return ST_OK; }
int Engine::step_with_fluid_log(uint64_t n) { return step(n); }
cudaError_t Engine::enqueue_fluid() { return cudaSuccess; }
void Engine::conv_open() {}
void Engine::conv_close() {}

}  // namespace sphb
