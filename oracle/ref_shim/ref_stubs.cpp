/* Stand-ins for reference members that the DEM step does not use but the
 * linked host sources reference -- TEST INFRASTRUCTURE ONLY. */
#include <cstdio>
#include <cstdlib>
#include "sphere.h"

static void unused(const char *what)
{
    std::fprintf(stderr, "reference host build: %s is not part of this build\n", what);
    std::abort();
}
void DEM::initNS() { unused("Navier-Stokes"); }
void DEM::initNSmem() { unused("Navier-Stokes"); }
void DEM::initNSmemDev() { unused("Navier-Stokes"); }
unsigned int DEM::idx(const int, const int, const int) { unused("Navier-Stokes"); return 0; }
