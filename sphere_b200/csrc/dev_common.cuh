// Shared device definitions for the DEM kernels.
//
// Arithmetic in the FP64 kernels follows the reference's operation order
// exactly (src/vector_arithmetic.h, src/contactmodels.cuh,
// src/integration.cuh); those kernels are compiled with -fmad=false, the
// reference's --fmad=false, so every product and sum rounds separately.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sphb {

// The reference's PI (src/constants.h:15).
#define SPHB_PI 3.14159265358979

// Error flags in DevCtl::err.
enum DevErr : int {
    DERR_NONE = 0,
    DERR_OUTSIDE = 1,   // particle outside the grid or non-finite
    DERR_CAPACITY = 2,  // contact slot row full
    DERR_TIMEOUT = 3,   // bounded grid barrier gave up
    DERR_BOND = 4,      // bond index out of range
    DERR_NAN = 5,       // Darcy residual not finite
};

// Fault injection for tests (sph_opts.inject_timeout, values equal to
// SPH_INJECT_*): the bounded waits of the selected kernels wait for a value
// nothing writes and give up after kInjectPolls polls, so the error path of a
// timed-out wait runs without a real hang.
constexpr uint32_t kInjectResort = 1, kInjectPersistent = 2, kInjectDarcy = 4, kInjectNS = 8;
constexpr unsigned kInjectPolls = 1u << 10;

// Per-run constants, passed to every kernel by value.
struct DevParams {
    uint32_t np, nc, nw, nb0;
    uint32_t ncells, nblocks256;   // ceil(np/256): the reference's blocksPerGrid
    uint32_t num[3];
    int32_t periodic;
    uint32_t contactmodel;
    int32_t integrator;            // 3 or 2
    int32_t wmode[6];
    double origo[3], L[3];
    double dt;
    double g[3];
    double k_n, k_t, E, gamma_n, gamma_t, mu_s, mu_d;
    double gamma_wn, gamma_wt, mu_ws, mu_wd, rho;
    double kappa, db, V_b;
    double sigma0_A, sigma0_f, tau_x;
    double lambda_bar, sigma_b, tau_b;
    double skin;                   // neighbour-list skin [m]
    uint32_t nlmax;                // neighbour-list entries per particle
    uint32_t inject;               // kInject* mask (a test knob; 0 in normal use)
};

// Loop state that lives on the device so captured graphs can replay steps.
struct DevCtl {
    long long iter;            // the reference's `iter` (device.cu:926)
    double t_current;          // time.current
    int velocity_state;        // rate-state step (device.cu:1000-1005)
    int resort;                // 1: a particle changed cell, sort before contacts
    int err;                   // DevErr
    int err_index;             // particle / bond that raised err
    double tau_eff_x;          // sum of the wmode-3 shear-stress partials
    long long resorts;         // number of sorts performed
    unsigned barrier_count;    // grid barrier state
    unsigned barrier_gen;
    unsigned ticket;           // last-block-done counter
    int nl_rebuild;            // 1: rebuild the neighbour lists before contacts
    long long nl_builds;       // neighbour-list builds performed
    // flags raised by an integration that runs inside the contact launch
    // (k_contacts_integrate); k_walls_step moves them into resort /
    // nl_rebuild once that launch has finished
    int resort_next;
    int nl_next;
};

struct V3 {
    double x, y, z;
};

// L2-only (L1-bypassing) load of a double4, for data another block wrote
// earlier in the same kernel.
__device__ __forceinline__ double4 ldcg4(const double4 *p)
{
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = __ldcg(q), b = __ldcg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ V3 mk3(double x, double y, double z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 add3(V3 a, V3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
// Float * Float3 (b * a.x)
__device__ __forceinline__ V3 smul3(double b, V3 a) { return mk3(b * a.x, b * a.y, b * a.z); }
// Float3 * Float (a.x * b)
__device__ __forceinline__ V3 muls3(V3 a, double b) { return mk3(a.x * b, a.y * b, a.z * b); }
__device__ __forceinline__ V3 divs3(V3 a, double b) { return mk3(a.x / b, a.y / b, a.z / b); }
__device__ __forceinline__ V3 adds3(V3 a, double b) { return mk3(a.x + b, a.y + b, a.z + b); }
__device__ __forceinline__ V3 neg3(V3 a) { return mk3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross3(V3 a, V3 b)
{
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 xyz(double4 a) { return mk3(a.x, a.y, a.z); }

// Vector length.  PREC 0: FP32 square root of the FP64 dot product rounded
// to FP32 (src/vector_arithmetic.h:317-324, IEEE-rounded); PREC 1: FP64.
template <int PREC>
__device__ __forceinline__ double vlen(V3 v)
{
    double d = dot3(v, v);
    if (PREC == 0) return (double)__fsqrt_rn(__double2float_rn(d));
    return __dsqrt_rn(d);
}

// sqrtf() applied to a Float argument in the kernels.
template <int PREC>
__device__ __forceinline__ double ssqrt(double v)
{
    if (PREC == 0) return (double)__fsqrt_rn(__double2float_rn(v));
    return __dsqrt_rn(v);
}

// Integer cell coordinate along axis d (src/sorting.cuh:7-20); false when
// the position is outside [origo, origo + num*cell) or not finite.
__device__ __forceinline__ bool cell_coord(const DevParams &P, double x, int d, int &out)
{
    double f = floor((x - P.origo[d]) / (P.L[d] / P.num[d]));
    if (!(f >= 0.0) || f >= (double)P.num[d]) return false;
    out = (int)f;
    return true;
}

// Decoded periodic shift of a contact slot (src/contactsearch.cuh:12-83):
// bit 0/1 = +/-L along x, bit 2/3 = +/-L along y.
__device__ __forceinline__ uint8_t dm_encode(int sx, int sy)
{
    return (uint8_t)((sx > 0 ? 1 : 0) | (sx < 0 ? 2 : 0) | (sy > 0 ? 4 : 0) | (sy < 0 ? 8 : 0));
}

__device__ __forceinline__ V3 dm_decode(const DevParams &P, uint8_t c)
{
    V3 d = mk3(0.0, 0.0, 0.0);
    if (c & 1) d = add3(d, mk3(P.L[0], 0.0, 0.0));
    if (c & 2) d = sub3(d, mk3(P.L[0], 0.0, 0.0));
    if (c & 4) d = add3(d, mk3(0.0, P.L[1], 0.0));
    if (c & 8) d = sub3(d, mk3(0.0, P.L[1], 0.0));
    return d;
}

__device__ __forceinline__ void raise_err(DevCtl *ctl, int code, int index)
{
    if (atomicCAS(&ctl->err, 0, code) == 0) ctl->err_index = index;
}

}  // namespace sphb
