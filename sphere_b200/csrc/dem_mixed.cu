// Mixed-precision DEM step.
#include "engine_internal.h"

namespace sphb {

int Engine::mixed_init() { return fail(ST_UNSUPPORTED, "mixed precision not built yet"); }

}  // namespace sphb
