/* Self-written stand-in for the vector-operator header the reference
 * downloads at build time (src/CMakeLists.txt:11-13) -- TEST
 * INFRASTRUCTURE ONLY.  Only the operators the host build needs. */
#ifndef REF_SHIM_HELPER_MATH_H_
#define REF_SHIM_HELPER_MATH_H_
#include "ref_shim.h"
#endif
