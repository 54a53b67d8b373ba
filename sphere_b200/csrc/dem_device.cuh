// Device code shared by the FP64 and the mixed-precision DEM kernels:
// contact laws, cell traversal, neighbour-list traversal, the slot policy
// and the contact kernel template.  The FP64 instantiations live in
// dem_kernels.cu (compiled with -fmad=false), the mixed one in dem_mixed.cu.
#pragma once

#include "dem_state.h"
#include "reduce_device.cuh"

namespace sphb {

// ---------------------------------------------------------------------
// contact laws
// ---------------------------------------------------------------------

// contactLinear_wall, src/contactmodels.cuh:10-114
template <int PREC>
__device__ double contact_wall(const DevParams &P, V3 &F, V3 &T, double &es_dot,
                               double &ev_dot, double &p, double ra, V3 vlin,
                               V3 angvel, V3 n, double delta, double wvel)
{
    V3 vel = adds3(add3(vlin, smul3(ra + delta / 2.0, cross3(n, angvel))), wvel);
    double vel_n = dot3(vlin, n);
    V3 vel_t = sub3(vel, muls3(n, dot3(n, vel)));
    double vel_t_length = vlen<PREC>(vel_t);
    double k_n = P.k_n;
    if (P.E > .001) k_n = 3.141592654 / 2.0 * P.E * ra;
    V3 f_n = smul3(fmax(0.0, -k_n * delta - P.gamma_wn * vel_n), n);
    double f_n_length = vlen<PREC>(f_n);
    ev_dot += P.gamma_wn * vel_n * vel_n;
    V3 f_t = mk3(0.0, 0.0, 0.0);
    if (vel_t_length > 0.0 && P.gamma_wt > 0.0) {
        V3 f_t_visc = smul3(P.gamma_wt, vel_t);
        double f_t_visc_length = vlen<PREC>(f_t_visc);
        double f_t_limit;
        if (vel_t_length > 0.0) f_t_limit = P.mu_wd * f_n_length;
        else f_t_limit = P.mu_ws * f_n_length;
        if (f_t_visc_length < f_t_limit) {
            f_t = smul3(-1.0, f_t_visc);
        } else {
            f_t = divs3(smul3(-f_t_limit, vel_t), vel_t_length);
            es_dot += vlen<PREC>(muls3(smul3(vlen<PREC>(f_t), vel_t), P.dt)) / P.dt;
        }
    }
    F = add3(F, add3(f_n, f_t));
    T = add3(T, cross3(smul3(-(ra + delta * 0.5), n), f_t));
    p += f_n_length / (4.0f * SPHB_PI * ra * ra);
    return dot3(f_n, n);
}

// contactLinear, src/contactmodels.cuh:241-408.  Returns the new
// tangential displacement (zero where the reference leaves it unassigned).
template <int PREC>
__device__ V3 contact_linear(const DevParams &P, V3 &F, V3 &T, double &es_dot,
                             double &ev_dot, double &p, double4 vel_a, V3 angvel_a,
                             double4 vel_b, V3 angvel_b, double4 dt0, double ra,
                             double rb, V3 x, double x_length, double delta)
{
    V3 delta_t0_uncor = xyz(dt0);
    V3 n = divs3(x, x_length);
    V3 vel_linear = mk3(vel_a.x - vel_b.x, vel_a.y - vel_b.y, vel_a.z - vel_b.z);
    V3 vel = add3(add3(vel_linear, smul3(ra + delta / 2.0, cross3(n, angvel_a))),
                  smul3(rb + delta / 2.0, cross3(n, angvel_b)));
    double vel_n = -dot3(vel_linear, n);
    V3 vel_t = sub3(vel, muls3(n, dot3(n, vel)));
    double vel_t_length = vlen<PREC>(vel_t);
    V3 delta_t0 = sub3(delta_t0_uncor, muls3(n, dot3(n, delta_t0_uncor)));
    double delta_t0_length = vlen<PREC>(delta_t0);
    V3 delta_t = mk3(0.0, 0.0, 0.0);
    double k_n = P.k_n, k_t = P.k_t;
    if (P.E > .001) {
        k_n = 3.141592654 / 2.0 * P.E * (ra + rb) / 2.;
        k_t = k_n;
    }
    V3 f_n = smul3(fmax(0.0, -k_n * delta + P.gamma_n * vel_n), n);
    double f_n_length = vlen<PREC>(f_n);
    ev_dot += 0.5 * P.gamma_n * vel_n * vel_n;
    V3 f_c = smul3(-P.kappa * ssqrt<PREC>(ra * rb), n);
    V3 f_t = mk3(0.0, 0.0, 0.0);
    if (delta_t0_length > 0.0 || vel_t_length > 0.0) {
        delta_t = add3(delta_t0, muls3(vel_t, P.dt));
        V3 f_t_elast = smul3(-k_t, delta_t);
        V3 f_t_visc = smul3(-P.gamma_t, vel_t);
        f_t = add3(f_t_elast, f_t_visc);
        double f_t_length = vlen<PREC>(f_t);
        double f_t_limit = P.mu_s * vlen<PREC>(sub3(f_n, f_c));
        ev_dot += 0.5 * P.gamma_t * vel_t_length * vel_t_length;
        if (f_t_length > f_t_limit) {
            V3 t = divs3(f_t, vlen<PREC>(f_t));
            f_t = smul3(f_t_limit, t);
            delta_t = smul3(-1.0 / k_t, add3(smul3(P.mu_d * vlen<PREC>(sub3(f_n, f_c)), t),
                                             smul3(P.gamma_t, vel_t)));
            es_dot += 0.5 * vlen<PREC>(muls3(smul3(vlen<PREC>(f_t), vel_t), P.dt)) / P.dt;
        }
    }
    F = add3(F, add3(add3(f_n, f_t), f_c));
    T = add3(T, cross3(smul3(-(ra + delta * 0.5), n), f_t));
    p += f_n_length / (4.0f * SPHB_PI * ra * ra);
    return delta_t;
}

// capillaryCohesion_exp, src/cohesion.cuh:237-277
template <int PREC>
__device__ void capillary_exp(const DevParams &P, V3 &N, double ra, double rb,
                              double delta_ab, V3 x_ab, double x_ab_length, double kappa)
{
    V3 n_ab = divs3(x_ab, x_ab_length);
    double r;
    if ((ra / rb) > (rb / ra)) r = ra / rb;
    else r = rb / ra;
    double h = -ssqrt<PREC>(r);
    double R_har = (2.0f * ra * rb) / (ra + rb);
    double R_geo = ssqrt<PREC>(ra * rb);
    double lambda = 0.9f * h * ssqrt<PREC>(P.V_b / R_har);
    double e = PREC == 0 ? (double)expf(__double2float_rn(-delta_ab / lambda))
                         : exp(-delta_ab / lambda);
    V3 f_c = smul3(-kappa * R_geo * e, n_ab);
    N = add3(N, f_c);
}

// contactLinearViscous, src/contactmodels.cuh:119-237
template <int PREC>
__device__ void contact_linear_viscous(const DevParams &P, V3 &F, V3 &T, double &p,
                                       double4 vel_a, V3 angvel_a, double4 vel_b,
                                       V3 angvel_b, double ra, double rb, V3 x_ab,
                                       double x_ab_length, double delta_ab, double kappa)
{
    V3 n_ab = divs3(x_ab, x_ab_length);
    V3 vel_ab_linear = mk3(vel_a.x - vel_b.x, vel_a.y - vel_b.y, vel_a.z - vel_b.z);
    V3 vel_ab = add3(add3(vel_ab_linear, smul3(ra + delta_ab / 2.0f, cross3(n_ab, angvel_a))),
                     smul3(rb + delta_ab / 2.0f, cross3(n_ab, angvel_b)));
    double vel_n_ab = dot3(vel_ab_linear, n_ab);
    V3 vel_t_ab = sub3(vel_ab, muls3(n_ab, dot3(vel_ab, n_ab)));
    double vel_t_ab_length = vlen<PREC>(vel_t_ab);
    double k_n = P.k_n;
    if (P.E > .001) k_n = 3.141592654 / 2.0 * P.E * (ra + rb) / 2.;
    V3 f_n = smul3(fmax(0.0, -k_n * delta_ab - P.gamma_n * vel_n_ab), n_ab);
    if (dot3(f_n, n_ab) < 0.0f) f_n = mk3(0.0f, 0.0f, 0.0f);
    double f_n_length = vlen<PREC>(f_n);
    V3 f_c = smul3(-kappa * ssqrt<PREC>(ra * rb), n_ab);
    V3 f_t = mk3(0.0, 0.0, 0.0);
    if (vel_t_ab_length > 0.0) {
        double f_t_visc = P.gamma_t * vel_t_ab_length;
        double f_t_limit;
        if (vel_t_ab_length > 0.001f) f_t_limit = P.mu_d * vlen<PREC>(sub3(f_n, f_c));
        else f_t_limit = P.mu_s * vlen<PREC>(sub3(f_n, f_c));
        if (f_t_visc < f_t_limit) f_t = divs3(smul3(-f_t_visc, vel_t_ab), vel_t_ab_length);
        else f_t = divs3(smul3(-f_t_limit, vel_t_ab), vel_t_ab_length);
    }
    F = add3(F, add3(add3(f_n, f_t), f_c));
    T = add3(T, smul3(-(ra + delta_ab / 2.0f), cross3(n_ab, f_t)));
    p += f_n_length / (4.0f * SPHB_PI * ra * ra);
}


// ---------------------------------------------------------------------
// mixed-precision contact laws: the same laws as contactLinear and
// contactLinear_wall (contactmodels.cuh:10-114, 241-408) evaluated in FP32
// from an FP64 overlap; the caller accumulates the results in FP64.
// ---------------------------------------------------------------------
struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 fadd(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ F3 fsub(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ F3 fmul(float s, F3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float fdot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 fcross(F3 a, F3 b)
{
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float flen(F3 a) { return sqrtf(fdot(a, a)); }
__device__ __forceinline__ F3 fxyz(float4 a) { return f3(a.x, a.y, a.z); }

__device__ __forceinline__ void mixed_pair(const DevParams &P, V3 &F, V3 &T, double &es_dot,
                                           double &ev_dot, double &p, float4 va, float4 wa,
                                           float4 vb, float4 wb, float4 &hist, double ra_d,
                                           double rb_d, V3 x_ab, double len, double delta_d)
{
    const float ra = (float)ra_d, rb = (float)rb_d, delta = (float)delta_d;
    const float inv = 1.0f / (float)len;
    const F3 n = f3((float)x_ab.x * inv, (float)x_ab.y * inv, (float)x_ab.z * inv);
    const F3 vel_linear = fsub(fxyz(va), fxyz(vb));
    const F3 vel = fadd(fadd(vel_linear, fmul(ra + 0.5f * delta, fcross(n, fxyz(wa)))),
                        fmul(rb + 0.5f * delta, fcross(n, fxyz(wb))));
    const float vel_n = -fdot(vel_linear, n);
    const F3 vel_t = fsub(vel, fmul(fdot(n, vel), n));
    const float vel_t_length = flen(vel_t);
    const F3 h0 = fxyz(hist);
    const F3 delta_t0 = fsub(h0, fmul(fdot(n, h0), n));
    const float delta_t0_length = flen(delta_t0);
    float k_n = (float)P.k_n, k_t = (float)P.k_t;
    if (P.E > .001) {
        k_n = (float)(1.5707963267948966 * P.E * (ra_d + rb_d) * 0.5);
        k_t = k_n;
    }
    const float gamma_n = (float)P.gamma_n, gamma_t = (float)P.gamma_t, dt = (float)P.dt;
    const float fn_mag = fmaxf(0.0f, -k_n * delta + gamma_n * vel_n);
    const F3 f_n = fmul(fn_mag, n);
    const float f_n_length = fabsf(fn_mag);
    double evd = 0.5 * (double)gamma_n * (double)vel_n * (double)vel_n;
    const F3 f_c = fmul(-(float)P.kappa * sqrtf(ra * rb), n);
    F3 f_t = f3(0.f, 0.f, 0.f), delta_t = f3(0.f, 0.f, 0.f);
    double esd = 0.0;
    if (delta_t0_length > 0.0f || vel_t_length > 0.0f) {
        delta_t = fadd(delta_t0, fmul(dt, vel_t));
        f_t = fsub(fmul(-k_t, delta_t), fmul(gamma_t, vel_t));
        const float f_t_length = flen(f_t);
        const float fnc = flen(fsub(f_n, f_c));
        const float f_t_limit = (float)P.mu_s * fnc;
        evd += 0.5 * (double)gamma_t * (double)vel_t_length * (double)vel_t_length;
        if (f_t_length > f_t_limit) {
            const F3 t = fmul(1.0f / f_t_length, f_t);
            f_t = fmul(f_t_limit, t);
            delta_t = fmul(-1.0f / k_t, fadd(fmul((float)P.mu_d * fnc, t), fmul(gamma_t, vel_t)));
            esd = 0.5 * (double)f_t_limit * (double)vel_t_length;
        }
    }
    ev_dot += evd;
    es_dot += esd;
    const F3 f = fadd(fadd(f_n, f_t), f_c);
    F = add3(F, mk3(f.x, f.y, f.z));
    const F3 tq = fcross(fmul(-(ra + 0.5f * delta), n), f_t);
    T = add3(T, mk3(tq.x, tq.y, tq.z));
    p += (double)f_n_length / (4.0 * SPHB_PI * ra_d * ra_d);
    hist = make_float4(delta_t.x, delta_t.y, delta_t.z, 0.0f);
}

__device__ __forceinline__ double mixed_wall(const DevParams &P, V3 &F, V3 &T, double &es_dot,
                                             double &ev_dot, double &p, double ra_d, V3 vlin_d,
                                             V3 angvel_d, V3 n_d, double delta_d, double wvel_d)
{
    const float ra = (float)ra_d, delta = (float)delta_d, wvel = (float)wvel_d;
    const F3 n = f3((float)n_d.x, (float)n_d.y, (float)n_d.z);
    const F3 vlin = f3((float)vlin_d.x, (float)vlin_d.y, (float)vlin_d.z);
    const F3 angvel = f3((float)angvel_d.x, (float)angvel_d.y, (float)angvel_d.z);
    F3 vel = fadd(vlin, fmul(ra + 0.5f * delta, fcross(n, angvel)));
    vel = f3(vel.x + wvel, vel.y + wvel, vel.z + wvel);
    const float vel_n = fdot(vlin, n);
    const F3 vel_t = fsub(vel, fmul(fdot(n, vel), n));
    const float vel_t_length = flen(vel_t);
    float k_n = (float)P.k_n;
    if (P.E > .001) k_n = (float)(1.5707963267948966 * P.E * ra_d);
    const float gamma_wn = (float)P.gamma_wn, gamma_wt = (float)P.gamma_wt;
    const float fn_mag = fmaxf(0.0f, -k_n * delta - gamma_wn * vel_n);
    const F3 f_n = fmul(fn_mag, n);
    const float f_n_length = fabsf(fn_mag) * flen(n);
    ev_dot += (double)gamma_wn * (double)vel_n * (double)vel_n;
    F3 f_t = f3(0.f, 0.f, 0.f);
    if (vel_t_length > 0.0f && gamma_wt > 0.0f) {
        const F3 f_t_visc = fmul(gamma_wt, vel_t);
        const float f_t_visc_length = flen(f_t_visc);
        const float f_t_limit = (float)P.mu_wd * f_n_length;
        if (f_t_visc_length < f_t_limit) {
            f_t = fmul(-1.0f, f_t_visc);
        } else {
            f_t = fmul(-f_t_limit / vel_t_length, vel_t);
            es_dot += (double)f_t_limit * (double)vel_t_length;
        }
    }
    const F3 f = fadd(f_n, f_t);
    F = add3(F, mk3(f.x, f.y, f.z));
    const F3 tq = fcross(fmul(-(ra + 0.5f * delta), n), f_t);
    T = add3(T, mk3(tq.x, tq.y, tq.z));
    p += (double)f_n_length / (4.0 * SPHB_PI * ra_d * ra_d);
    return (double)fdot(f_n, n);
}

// Wall contact in the precision of the step.
template <int PREC>
__device__ __forceinline__ double wall_law(const DevParams &P, V3 &F, V3 &T, double &es_dot,
                                           double &ev_dot, double &p, double ra, V3 vlin,
                                           V3 angvel, V3 n, double delta, double wvel)
{
    if constexpr (PREC == 2) return mixed_wall(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel, n, delta, wvel);
    else return contact_wall<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel, n, delta, wvel);
}

// findDistMod, src/contactsearch.cuh:12-83: returns false for a cell
// outside the grid; wraps periodic cells and sets the shift signs.
__device__ __forceinline__ bool wrap_cell(const DevParams &P, int &cx, int &cy, int cz,
                                          int &sx, int &sy)
{
    int nx = (int)P.num[0], ny = (int)P.num[1], nz = (int)P.num[2];
    sx = 0;
    sy = 0;
    if (P.periodic == 1) {
        if (cx < 0) { cx += nx; sx = 1; }
        if (cx >= nx) { cx -= nx; sx = -1; }
        if (cy < 0) { cy += ny; sy = 1; }
        if (cy >= ny) { cy -= ny; sy = -1; }
    }
    if (P.periodic == 2) {
        if (cx < 0) { cx += nx; sx = 1; }
        if (cx >= nx) { cx -= nx; sx = -1; }
        if (cy < 0 || cy >= ny) return false;
    }
    if (P.periodic > 2 || P.periodic < 1) {
        if (cx < 0 || cx >= nx) return false;
        if (cy < 0 || cy >= ny) return false;
    }
    return !(cz < 0 || cz >= nz);
}

__device__ __forceinline__ void grid_pos(const DevParams &P, double4 x, int &gx, int &gy, int &gz)
{
    gx = (int)floor((x.x - P.origo[0]) / (P.L[0] / P.num[0]));
    gy = (int)floor((x.y - P.origo[1]) / (P.L[1] / P.num[1]));
    gz = (int)floor((x.z - P.origo[2]) / (P.L[2] / P.num[2]));
}

// ---------------------------------------------------------------------
// contact search + forces: topology (contactsearch.cuh:329-371) and
// interact (contactsearch.cuh:385-726) for one particle per thread.
//
// Candidates come from a neighbour list built in the reference's visiting
// order (27 cells z, y, x; sorted order inside a cell) holding every pair
// closer than r_a + r_b + skin.  The list is rebuilt whenever the sort
// changed or a particle moved more than 0.45 skin since the build, so a
// pair missing from it cannot overlap: the overlap tests, and therefore the
// slot insertions, happen in exactly the reference's sequence.  The slot
// row is tracked with an occupancy bitmask so the slot policy and the force
// loop visit occupied slots only; empty slots keep zero history, which is
// what the reference rewrites into them every step.
// ---------------------------------------------------------------------
constexpr uint32_t NL_OVERFLOW = 0xffffffffu;

__device__ __forceinline__ V3 shift_vec(const DevParams &P, int sx, int sy)
{
    V3 dm = mk3(0.0, 0.0, 0.0);
    if (sx > 0) dm = add3(dm, mk3(P.L[0], 0.0, 0.0));
    if (sx < 0) dm = sub3(dm, mk3(P.L[0], 0.0, 0.0));
    if (sy > 0) dm = add3(dm, mk3(0.0, P.L[1], 0.0));
    if (sy < 0) dm = sub3(dm, mk3(0.0, P.L[1], 0.0));
    return dm;
}

// Visits every candidate of particle k in the reference's 27-cell order and
// calls f(b, sx, sy) with its sorted index and periodic shift signs.
template <class F>
__device__ __forceinline__ void for_each_cell_candidate(const DevParams &P, const DevState &S,
                                                        unsigned k, double4 xa, F &&f)
{
    int gx, gy, gz;
    grid_pos(P, xa, gx, gy, gz);
    for (int dz = -1; dz < 2; ++dz)
        for (int dy = -1; dy < 2; ++dy)
            for (int dx = -1; dx < 2; ++dx) {
                int cx = gx + dx, cy = gy + dy, cz = gz + dz, sx, sy;
                if (!wrap_cell(P, cx, cy, cz, sx, sy)) continue;
                unsigned cell = (unsigned)cx + (unsigned)cy * P.num[0] +
                                (P.num[0] * P.num[1]) * (unsigned)cz;
                unsigned start = S.cell_start[cell];
                if (start == 0xffffffffu) continue;
                unsigned end = S.cell_end[cell];
                for (unsigned b = start; b < end; ++b) {
                    if (b == k) continue;
                    if (!f(b, sx, sy)) return;
                }
            }
}


// The slot the reference's topology picks for partner b_orig
// (contactsearch.cuh:267-280): the first slot already holding b_orig, else
// the last empty slot, else nc.
__device__ __forceinline__ int pick_slot(uint64_t mask, uint64_t full, const uint32_t *srow,
                                         unsigned B, unsigned t, unsigned b_orig, int nc)
{
    uint64_t m = mask;
    while (m) {
        int i = __ffsll((long long)m) - 1;
        if (srow[i * B + t] == b_orig) return i;
        m &= m - 1;
    }
    uint64_t empty = ~mask & full;
    if (empty) return 63 - __clzll((long long)empty);
    return nc;
}

// Results of the contact search and force evaluation of one particle.
struct ContactOut {
    V3 F, T;
    double es_dot, ev_dot, p;
    double wf0, wf1, wf2, wf3, wf4;   // force on each dynamic wall (walls_force_pp)
};

// Wall contacts of one particle (contactsearch.cuh:602-701) after its
// particle contacts, and the results of both into out.
template <int PREC>
__device__ __forceinline__ void contact_walls(const DevParams &P, const DevState &S, double4 xa,
                                              double ra, double4 vel_a, V3 angvel_a, V3 F, V3 T,
                                              double es_dot, double ev_dot, double p,
                                              ContactOut &out)
{
    // walls beyond nw keep the reference's defaults (the domain faces); the
    // five walls are unrolled so their state stays in registers
    const unsigned nw = P.nw;
    const double4 wnx0 = nw > 0 ? S.wnx[0] : make_double4(0.0f, 0.0f, -1.0f, P.L[2]);
    const double4 wnx1 = nw > 1 ? S.wnx[1] : make_double4(-1.0f, 0.0f, 0.0f, P.L[0]);
    const double4 wnx2 = nw > 2 ? S.wnx[2] : make_double4(1.0f, 0.0f, 0.0f, 0.0f);
    const double4 wnx3 = nw > 3 ? S.wnx[3] : make_double4(0.0f, -1.0f, 0.0f, P.L[1]);
    const double4 wnx4 = nw > 4 ? S.wnx[4] : make_double4(0.0f, 1.0f, 0.0f, 0.0f);
    double wf0 = 0.0, wf1 = 0.0, wf2 = 0.0, wf3 = 0.0, wf4 = 0.0;
    V3 vlin = xyz(vel_a);
    double dw = wnx0.w - (xa.z + ra);
    if (dw < 0.0f)
        wf0 = wall_law<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a, xyz(wnx0), dw,
                             nw > 0 ? S.wmvfd[0].y : 0.0);
    dw = xa.z - ra - P.origo[2];
    if (dw < 0.0f)
        (void)wall_law<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a,
                                 mk3(0.0f, 0.0f, 1.0f), dw, 0.0);
    if (P.periodic == 0) {
        dw = wnx1.w - (xa.x + ra);
        if (dw < 0.0f)
            wf1 = wall_law<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a, xyz(wnx1), dw,
                                 nw > 1 ? S.wmvfd[1].y : 0.0);
        dw = xa.x - ra - wnx2.w;
        if (dw < 0.0f)
            wf2 = wall_law<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a, xyz(wnx2), dw,
                                 nw > 2 ? S.wmvfd[2].y : 0.0);
    }
    if (P.periodic == 0 || P.periodic == 2) {
        dw = wnx3.w - (xa.y + ra);
        if (dw < 0.0f)
            wf3 = wall_law<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a, xyz(wnx3), dw,
                                 nw > 3 ? S.wmvfd[3].y : 0.0);
        dw = xa.y - ra - wnx4.w;
        if (dw < 0.0f)
            wf4 = wall_law<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a, xyz(wnx4), dw,
                                 nw > 4 ? S.wmvfd[4].y : 0.0);
    }
    out.F = F;
    out.T = T;
    out.es_dot = es_dot;
    out.ev_dot = ev_dot;
    out.p = p;
    out.wf0 = wf0; out.wf1 = wf1; out.wf2 = wf2; out.wf3 = wf3; out.wf4 = wf4;
}

// Contact search + forces of sorted particle k (topology and interact of
// the reference, walls included).  srow is the thread's slot scratch in
// shared memory (entry i at srow[i * B + t]: the partner's original index).
// Returns false after raising a capacity error.
// PREC 0: faithful FP64, 1: FP64, 2: mixed (FP64 overlap, FP32 contact law,
// FP64 accumulation).
template <int PREC, int MODEL>
__device__ __forceinline__ bool contact_particle(const DevParams &P, const DevState &S, unsigned k,
                                                 uint32_t *srow, unsigned B, unsigned t,
                                                 ContactOut &out)
{
    constexpr int TP = PREC == 2 ? 1 : PREC;  // precision of overlap tests
    const unsigned NC = P.nc;
    const uint64_t full = NC >= 64 ? ~0ull : ((1ull << NC) - 1ull);
    const unsigned o = S.orig_of[k];
    const double4 xa = S.x[k];
    const double ra = xa.w;
    const double4 vel_a = S.vel[k];
    const V3 angvel_a = xyz(S.angvel[k]);
    double es_dot = 0.0, ev_dot = 0.0, p = 0.0;
    V3 F = mk3(0.0, 0.0, 0.0), T = mk3(0.0, 0.0, 0.0);
    const unsigned cnt = S.nl_count[k];
    const size_t np = P.np;

    if (MODEL == 2) {
        const size_t rowbase = (size_t)o * NC;
        uint64_t mask = S.occ[o];
        uint64_t written = 0;
        {
            uint64_t m = mask;
            while (m) {
                int i = __ffsll((long long)m) - 1;
                srow[i * B + t] = S.contacts[rowbase + i];
                m &= m - 1;
            }
        }
        // --- topology ---
        int nc = 0;
        bool ok = true;
        auto visit = [&](unsigned b, int sx, int sy) -> bool {
            double4 xb = S.x[b];
            double rb = xb.w;
            V3 xab = mk3(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z);
            xab = add3(xab, shift_vec(P, sx, sy));
            double len = vlen<TP>(xab);
            double delta = len - (ra + rb);
            if (delta < 0.0) {
                unsigned b_orig = S.orig_of[b];
                int cpos = pick_slot(mask, full, srow, B, t, b_orig, nc);
                if (cpos >= (int)NC || nc + 1 > (int)NC) {
                    raise_err(S.ctl, DERR_CAPACITY, (int)o);
                    ok = false;
                    return false;
                }
                srow[cpos * B + t] = b_orig;
                mask |= 1ull << cpos;
                written |= 1ull << cpos;
                S.dmcode[rowbase + cpos] = dm_encode(sx, sy);
                ++nc;
            }
            return true;
        };
        if (cnt != NL_OVERFLOW) {
            for (unsigned j = 0; j < cnt; ++j) {
                uint32_t e = S.nl[(size_t)j * np + k];
                uint32_t c = e >> 28;
                int sx = (c & 1) ? 1 : ((c & 2) ? -1 : 0);
                int sy = (c & 4) ? 1 : ((c & 8) ? -1 : 0);
                if (!visit(e & 0x0fffffffu, sx, sy)) break;
            }
        } else {
            for_each_cell_candidate(P, S, k, xa, visit);
        }
        if (!ok) return false;
        // --- interact, history contacts in slot order ---
        uint64_t m = mask;
        while (m) {
            const int i = __ffsll((long long)m) - 1;
            m &= m - 1;
            const unsigned b_orig = srow[i * B + t];
            if (b_orig >= P.np) { raise_err(S.ctl, DERR_CAPACITY, (int)o); return false; }
            const size_t mempos = rowbase + i;
            V3 dm = dm_decode(P, S.dmcode[mempos]);
            unsigned kb = S.pos_of[b_orig];
            double4 xb = S.x[kb];
            double rb = xb.w;
            V3 x_ab = mk3(xa.x - xb.x + dm.x, xa.y - xb.y + dm.y, xa.z - xb.z + dm.z);
            double len = vlen<TP>(x_ab);
            double delta_n = len - (ra + rb);
            if (delta_n < 0.0) {
                if constexpr (PREC == 2) {
                    float4 h = S.delta_t_f[mempos];
                    mixed_pair(P, F, T, es_dot, ev_dot, p, S.vel_f[k], S.angvel_f[k], S.vel_f[kb],
                               S.angvel_f[kb], h, ra, rb, x_ab, len, delta_n);
                    S.delta_t_f[mempos] = h;
                } else {
                    V3 dt_new = contact_linear<PREC>(P, F, T, es_dot, ev_dot, p, vel_a, angvel_a,
                                                     S.vel[kb], xyz(S.angvel[kb]),
                                                     S.delta_t[mempos], ra, rb, x_ab, len, delta_n);
                    S.delta_t[mempos] = make_double4(dt_new.x, dt_new.y, dt_new.z, 0.0);
                }
            } else {
                mask &= ~(1ull << i);
                written |= 1ull << i;
                if constexpr (PREC == 2) S.delta_t_f[mempos] = make_float4(0.f, 0.f, 0.f, 0.f);
                else S.delta_t[mempos] = make_double4(0.0, 0.0, 0.0, 0.0);
            }
        }
        if (written) {
            uint64_t w = written;
            while (w) {
                int i = __ffsll((long long)w) - 1;
                w &= w - 1;
                S.contacts[rowbase + i] = (mask >> i) & 1ull ? srow[i * B + t] : P.np;
            }
            S.occ[o] = mask;
        }
    } else if (MODEL == 1) {
        // findAndProcessContactsInCell, contactsearch.cuh:91-186
        auto visit = [&](unsigned b, int sx, int sy) -> bool {
            double4 xb = S.x[b];
            double rb = xb.w;
            V3 x_ab = mk3(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z);
            x_ab = add3(x_ab, shift_vec(P, sx, sy));
            double len = vlen<TP>(x_ab);
            double delta_ab = len - (ra + rb);
            if (delta_ab < 0.0f)
                contact_linear_viscous<TP>(P, F, T, p, vel_a, angvel_a, S.vel[b],
                                             xyz(S.angvel[b]), ra, rb, x_ab, len, delta_ab,
                                             P.kappa);
            else if (delta_ab < P.db)
                capillary_exp<TP>(P, F, ra, rb, delta_ab, x_ab, len, P.kappa);
            return true;
        };
        if (cnt != NL_OVERFLOW && !(P.db > 0.0 && P.kappa != 0.0)) {
            for (unsigned j = 0; j < cnt; ++j) {
                uint32_t e = S.nl[(size_t)j * np + k];
                uint32_t c = e >> 28;
                int sx = (c & 1) ? 1 : ((c & 2) ? -1 : 0);
                int sy = (c & 4) ? 1 : ((c & 8) ? -1 : 0);
                visit(e & 0x0fffffffu, sx, sy);
            }
        } else {
            for_each_cell_candidate(P, S, k, xa, visit);
        }
    }

    contact_walls<PREC>(P, S, xa, ra, vel_a, angvel_a, F, T, es_dot, ev_dot, p, out);
    return true;
}

// Write-back of one particle's contact results (contactsearch.cuh:706-724).
__device__ __forceinline__ void contact_writeback(const DevParams &P, const DevState &S, unsigned k,
                                                  const ContactOut &c)
{
    const unsigned o = S.orig_of[k];
    S.force[k] = make_double4(c.F.x, c.F.y, c.F.z, 0.0f);
    S.torque[k] = make_double4(c.T.x, c.T.y, c.T.z, 0.0f);
    S.es_dot[k] = c.es_dot;
    S.ev_dot[k] = c.ev_dot;
    S.es[k] += c.es_dot * P.dt;
    S.ev[k] += c.ev_dot * P.dt;
    S.p[k] = c.p;
    const size_t np = P.np;
    if (P.nw > 0) S.walls_force_pp[o] = c.wf0;
    if (P.nw > 1) S.walls_force_pp[o + np] = c.wf1;
    if (P.nw > 2) S.walls_force_pp[o + 2 * np] = c.wf2;
    if (P.nw > 3) S.walls_force_pp[o + 3 * np] = c.wf3;
    if (P.nw > 4) S.walls_force_pp[o + 4 * np] = c.wf4;
}

// Neighbour list of sorted particle k (defined below).
__device__ __forceinline__ void nl_build_particle(const DevParams &P, const DevState &S, unsigned k);

// 6 resident blocks of 128 threads per SM (80 registers): measured best
// between 1 and 8 on the dense-shear workload.
#ifndef SPHB_CONTACT_MINB
#define SPHB_CONTACT_MINB 6
#endif
// threads per block of the per-stage contact kernel
#ifndef SPHB_CONTACT_B
#define SPHB_CONTACT_B 128
#endif
// Contact search and forces of the per-stage path (after k_nl_build).
template <int PREC, int MODEL>
__global__ void __launch_bounds__(SPHB_CONTACT_B, SPHB_CONTACT_MINB) k_contacts(DevParams P, DevState S)
{
    extern __shared__ uint32_t srow[];   // blockDim * nc slot partners
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0 && S.ctl->nl_rebuild) S.ctl->nl_rebuild = 0;  // k_resort has rebuilt the lists
    if (S.ctl->err || k >= P.np) return;
    ContactOut c;
    if (!contact_particle<PREC, MODEL>(P, S, k, srow, blockDim.x, threadIdx.x, c)) return;
    contact_writeback(P, S, k, c);
}

// Neighbour list of sorted particle k: every candidate closer than
// r_a + r_b + skin, in the reference's visiting order; records the build
// position.
__device__ __forceinline__ void nl_build_particle(const DevParams &P, const DevState &S, unsigned k)
{
    double4 xa = S.x[k];
    const double ra = xa.w;
    unsigned n = 0;
    const size_t np = P.np;
    for_each_cell_candidate(P, S, k, xa, [&](unsigned b, int sx, int sy) {
        double4 xb = S.x[b];
        V3 dm = shift_vec(P, sx, sy);
        V3 xab = add3(mk3(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z), dm);
        double reach = ra + xb.w + P.skin;
        if (dot3(xab, xab) < reach * reach) {
            if (n < P.nlmax) S.nl[(size_t)n * np + k] = b | ((uint32_t)dm_encode(sx, sy) << 28);
            ++n;
        }
        return true;
    });
    S.nl_count[k] = n <= P.nlmax ? n : NL_OVERFLOW;
    S.x_ref[k] = make_float4((float)xa.x, (float)xa.y, (float)xa.z, 0.0f);
}

// Loop state an integration step reads (the values before the step).
struct StepClock {
    long long iter;
    double t_current;
    int velocity_state;
    double tau_eff_x;
};

// The inputs of one particle's integration step (its state before the step
// and the forces of the step).
struct IntegrateIn {
    double4 force, torque, x, vel, angvel, angpos, xyzsum, acc0, angacc0;
    float4 x_ref;      // position at the last neighbour-list build
    uint32_t cell;     // cell of the current sort
};

// integrate, src/integration.cuh:14-305 (TY3 default, TY2 selectable), for
// sorted particle k with the inputs `in` (acc0 / angacc0 are read only
// after the first step, as the reference does), followed by the cell hash
// of the new position (src/sorting.cuh:7-51).  Writes the new x, vel,
// angvel (and their FP32 copies when vel_f_out is set) to the *_out arrays
// -- S's own arrays for the in-place kernel, the other buffer of a ping-pong
// pair for the fused step -- and acc, angacc, angpos, xyzsum, cell_new to S.
// Raises *resort_flag when the cell changed and *nl_flag when the particle
// left its neighbour-list skin.  Returns false after raising an outside-grid
// error.
__device__ __forceinline__ bool integrate_values(const DevParams &P, const DevState &S, unsigned k,
                                                 const IntegrateIn &in, const StepClock &clk,
                                                 double4 *x_out, double4 *vel_out,
                                                 double4 *angvel_out, float4 *vel_f_out,
                                                 float4 *angvel_f_out, int *resort_flag,
                                                 int *nl_flag)
{
    const long long iter = clk.iter;
    const double t_current = clk.t_current;
    // rate-state velocity step (device.cu:2461-2469), decided from the
    // loop state before this step
    int change_velocity_state = 0;
    {
        int vs = clk.velocity_state;
        if (t_current >= 10.0 && t_current < 15.0 && vs == 1) change_velocity_state = 1;
        else if (t_current >= 15.0 && vs == 2) change_velocity_state = -1;
    }
    const double velocity_factor = 10.0;
    const double4 force = in.force, torque = in.torque;
    double4 angpos = in.angpos;
    double4 x = in.x, vel = in.vel, angvel = in.angvel;
    double4 xyzsum = in.xyzsum;
    int wall0mode = 0;
    double wall0mass = 0.0;
    if (P.nw > 0) {
        wall0mode = P.wmode[0];
        wall0mass = S.wmvfd[0].x;
    }
    double tau_eff_x = 0.0;
    if (P.nw > 0 && wall0mode == 3) tau_eff_x = clk.tau_eff_x;
    double4 acc0 = make_double4(0, 0, 0, 0), angacc0 = make_double4(0, 0, 0, 0);
    if (iter != 0) {
        acc0 = in.acc0;
        angacc0 = in.angacc0;
    }
    double radius = x.w;
    double dt = P.dt;
    double m = 4.0 / 3.0 * SPHB_PI * radius * radius * radius * P.rho;
    double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
    acc.x = force.x / m + P.g[0];
    acc.y = force.y / m + P.g[1];
    acc.z = force.z / m + P.g[2];
    double4 angacc = make_double4(0.0, 0.0, 0.0, 0.0);
    angacc.x = torque.x * 1.0 / (2.0 / 5.0 * m * radius * radius);
    angacc.y = torque.y * 1.0 / (2.0 / 5.0 * m * radius * radius);
    angacc.z = torque.z * 1.0 / (2.0 / 5.0 * m * radius * radius);
    const double4 zero4 = make_double4(0.0, 0.0, 0.0, 0.0);
    if (wall0mode == 3 && vel.w > 0.0001 && x.z > P.L[2] * 0.5) {
        double f_tau_x = (P.tau_x + tau_eff_x) * P.L[0] * P.L[1];
        acc.x = f_tau_x / wall0mass;
        acc.y = 0.0;
        acc.z -= P.g[2];
        angacc = zero4;
    } else if (vel.w > 0.0001 && vel.w < 10.0) {
        acc.x = 0.0;
        acc.y = 0.0;
        acc.z -= P.g[2];
        angacc = zero4;
    }
    if (vel.w >= 10.0) {
        acc.y = 0.0;
        angacc.x = 0.0;
        angacc.z = 0.0;
    }
    if (vel.w < -0.0001) {
        acc.x = 0.0;
        acc.y = 0.0;
        acc.z = 0.0;
        angacc = zero4;
    }
    double4 x_new, vel_new, angpos_new, angvel_new;
    if (P.integrator == 3) {
        double dax = (acc.x - acc0.x) / dt, day = (acc.y - acc0.y) / dt, daz = (acc.z - acc0.z) / dt;
        double dwx = (angacc.x - angacc0.x) / dt, dwy = (angacc.y - angacc0.y) / dt,
               dwz = (angacc.z - angacc0.z) / dt;
        x_new.x = x.x + vel.x * dt + 0.5 * acc.x * dt * dt + 1.0 / 6.0 * dax * dt * dt * dt;
        x_new.y = x.y + vel.y * dt + 0.5 * acc.y * dt * dt + 1.0 / 6.0 * day * dt * dt * dt;
        x_new.z = x.z + vel.z * dt + 0.5 * acc.z * dt * dt + 1.0 / 6.0 * daz * dt * dt * dt;
        x_new.w = x.w;
        vel_new.x = vel.x + acc.x * dt + 0.5 * dax * dt * dt;
        vel_new.y = vel.y + acc.y * dt + 0.5 * day * dt * dt;
        vel_new.z = vel.z + acc.z * dt + 0.5 * daz * dt * dt;
        vel_new.w = vel.w;
        angpos_new.x = angpos.x + angvel.x * dt + 0.5 * angacc.x * dt * dt + 1.0 / 6.0 * dwx * dt * dt * dt;
        angpos_new.y = angpos.y + angvel.y * dt + 0.5 * angacc.y * dt * dt + 1.0 / 6.0 * dwy * dt * dt * dt;
        angpos_new.z = angpos.z + angvel.z * dt + 0.5 * angacc.z * dt * dt + 1.0 / 6.0 * dwz * dt * dt * dt;
        angpos_new.w = angpos.w;
        angvel_new.x = angvel.x + angacc.x * dt + 0.5 * dwx * dt * dt;
        angvel_new.y = angvel.y + angacc.y * dt + 0.5 * dwy * dt * dt;
        angvel_new.z = angvel.z + angacc.z * dt + 0.5 * dwz * dt * dt;
        angvel_new.w = angvel.w;
        xyzsum.x += vel.x * dt + 0.5 * acc.x * dt * dt + 1.0 / 6.0 * dax * dt * dt * dt;
        xyzsum.y += vel.y * dt + 0.5 * acc.y * dt * dt + 1.0 / 6.0 * day * dt * dt * dt;
        xyzsum.z += vel.z * dt + 0.5 * acc.z * dt * dt + 1.0 / 6.0 * daz * dt * dt * dt;
    } else {
        x_new.x = x.x + vel.x * dt + 0.5 * acc.x * dt * dt;
        x_new.y = x.y + vel.y * dt + 0.5 * acc.y * dt * dt;
        x_new.z = x.z + vel.z * dt + 0.5 * acc.z * dt * dt;
        x_new.w = x.w;
        vel_new.x = vel.x + acc.x * dt;
        vel_new.y = vel.y + acc.y * dt;
        vel_new.z = vel.z + acc.z * dt;
        vel_new.w = vel.w;
        angpos_new.x = angpos.x + angvel.x * dt + 0.5 * angacc.x * dt * dt;
        angpos_new.y = angpos.y + angvel.y * dt + 0.5 * angacc.y * dt * dt;
        angpos_new.z = angpos.z + angvel.z * dt + 0.5 * angacc.z * dt * dt;
        angpos_new.w = angpos.w;
        angvel_new.x = angvel.x + angacc.x * dt;
        angvel_new.y = angvel.y + angacc.y * dt;
        angvel_new.z = angvel.z + angacc.z * dt;
        angvel_new.w = angvel.w;
        xyzsum.x += vel.x * dt + 0.5 * acc.x * dt * dt;
        xyzsum.y += vel.y * dt + 0.5 * acc.y * dt * dt;
        xyzsum.z += vel.z * dt + 0.5 * acc.z * dt * dt;
    }
    if (P.periodic == 1) {
        if (x_new.x < P.origo[0]) x_new.x += P.L[0];
        if (x_new.x > P.L[0]) x_new.x -= P.L[0];
        if (x_new.y < P.origo[1]) x_new.y += P.L[1];
        if (x_new.y > P.L[1]) x_new.y -= P.L[1];
    } else if (P.periodic == 2) {
        if (x_new.x < P.origo[0]) x_new.x += P.L[0];
        if (x_new.x > P.L[0]) x_new.x -= P.L[0];
    }
    if (vel.w > 5.0 && vel.w < 10.0) {
        if (change_velocity_state == 1) vel_new.x *= velocity_factor;
        else if (change_velocity_state == -1) vel_new.x /= velocity_factor;
    }
    S.xyzsum[k] = xyzsum;
    S.acc[k] = acc;
    S.angacc[k] = angacc;
    angvel_out[k] = angvel_new;
    vel_out[k] = vel_new;
    S.angpos[k] = angpos_new;
    x_out[k] = x_new;
    if (vel_f_out) {
        vel_f_out[k] = make_float4((float)vel_new.x, (float)vel_new.y, (float)vel_new.z, (float)vel_new.w);
        angvel_f_out[k] = make_float4((float)angvel_new.x, (float)angvel_new.y, (float)angvel_new.z, 0.0f);
    }
    // cell of the new position
    int ix, iy, iz;
    if (!cell_coord(P, x_new.x, 0, ix) || !cell_coord(P, x_new.y, 1, iy) ||
        !cell_coord(P, x_new.z, 2, iz)) {
        raise_err(S.ctl, DERR_OUTSIDE, (int)S.orig_of[k]);
        return false;
    }
    unsigned c = ((unsigned)iz * P.num[1]) * P.num[0] + (unsigned)iy * P.num[0] + (unsigned)ix;
    S.cell_new[k] = c;
    if (c != in.cell) *resort_flag = 1;
    // neighbour lists stay exact while every particle is within 0.45 skin
    // of its position at the build
    const float4 xr = in.x_ref;
    double ddx = x_new.x - (double)xr.x, ddy = x_new.y - (double)xr.y, ddz = x_new.z - (double)xr.z;
    double lim = 0.45 * P.skin;
    if (ddx * ddx + ddy * ddy + ddz * ddz > lim * lim) *nl_flag = 1;
    return true;
}

// integrate_values for sorted particle k with its state read from S and the
// given force and torque.
__device__ __forceinline__ bool integrate_particle(const DevParams &P, const DevState &S, unsigned k,
                                                   double4 force, double4 torque, const StepClock &clk,
                                                   double4 *x_out, double4 *vel_out,
                                                   double4 *angvel_out, float4 *vel_f_out,
                                                   float4 *angvel_f_out, int *resort_flag,
                                                   int *nl_flag)
{
    IntegrateIn in;
    in.force = force;
    in.torque = torque;
    in.angpos = S.angpos[k];
    in.x = S.x[k];
    in.vel = S.vel[k];
    in.angvel = S.angvel[k];
    in.xyzsum = S.xyzsum[k];
    in.acc0 = make_double4(0, 0, 0, 0);
    in.angacc0 = make_double4(0, 0, 0, 0);
    if (clk.iter != 0) {
        in.acc0 = S.acc[k];
        in.angacc0 = S.angacc[k];
    }
    in.cell = S.cell_of[k];
    in.x_ref = S.x_ref[k];
    return integrate_values(P, S, k, in, clk, x_out, vel_out, angvel_out, vel_f_out, angvel_f_out,
                            resort_flag, nl_flag);
}

// Copies sorted particle k's x / vel / angvel (and their FP32 copies) into
// the other buffer of the ping-pong pair unchanged: a step that does not
// integrate k still hands its state on to the next buffer.
__device__ __forceinline__ void carry_particle(const DevState &S, unsigned k)
{
    S.x_nx[k] = S.x[k];
    S.vel_nx[k] = S.vel[k];
    S.angvel_nx[k] = S.angvel[k];
    if (S.vel_f_nx) {
        S.vel_f_nx[k] = S.vel_f[k];
        S.angvel_f_nx[k] = S.angvel_f[k];
    }
}

// The 256-element tree sum of the wall-0 forces of chunk j (ORIGINAL
// indices [256 j, 256 j + 256)) in the reference's summation order
// (src/integration.cuh:309-341: cache[e] += cache[e + i] for i = 128, 64,
// ..., 1), formed by one warp: lane l holds e = l + 32 q, q = 0..7, so the
// levels 128, 64 and 32 pair values within a lane and the levels 16..1 are
// shuffles.  The result is valid in lane 0.
__device__ __forceinline__ double warp_chunk_tree_sum(const double *in, unsigned np, unsigned j)
{
    const unsigned lane = threadIdx.x & 31u;
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const unsigned idx = (j << 8) + lane + 32u * q;
        double t = 0.0f;
        if (idx < np) t += __ldcg(in + idx);
        v[q] = t;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] += v[q + 4];
    v[0] += v[2];
    v[1] += v[3];
    v[0] += v[1];
#pragma unroll
    for (unsigned i = 16; i != 0; i /= 2) v[0] += __shfl_down_sync(0xffffffffu, v[0], i);
    return v[0];
}

// The end of a step whose particles k_contacts_integrate advanced, by one
// warp once every chunk partial is written: the partials added in chunk
// order (the reference's serial loop, integration.cuh:67-68, 376-378;
// every lane forms the same sum), then in lane 0 the wall update, the loop
// counters and the next step's flags.
__device__ __forceinline__ void finish_step(const DevParams &P, const DevState &S)
{
    const unsigned lane = threadIdx.x & 31u;
    DevCtl *ctl = S.ctl;
    double wforce = 0.0;
    if (P.nw > 0) {
        // 32 partials per pass, the next 32 already in flight; past
        // the last partial the lanes hold +0.0, which leaves the sum
        // unchanged (it starts at +0.0, so it is never -0.0)
        const unsigned n = P.nblocks256;
        double v = lane < n ? __ldcg(S.partials + lane) : 0.0;
        for (unsigned base = 0; base < n; base += 32) {
            const unsigned nx = base + 32 + lane;
            const double vn = nx < n ? __ldcg(S.partials + nx) : 0.0;
#pragma unroll
            for (int i = 0; i < 32; ++i) wforce += __shfl_sync(0xffffffffu, v, i);
            v = vn;
        }
    }
    if (lane != 0) return;
    ctl->ticket = 0;
    // the flags the integration raised in the contact launch
    if (__ldcg(&ctl->resort_next)) ctl->resort = 1;
    // lists rebuilt at the start of this step are current unless a particle
    // has since left its skin
    ctl->nl_rebuild = __ldcg(&ctl->nl_next);
    ctl->resort_next = 0;
    ctl->nl_next = 0;
    if (*(volatile int *)&ctl->err) return;
    const long long iter = ctl->iter;
    const double t_current = ctl->t_current;
    walls_integrate(P, S, wforce, iter, t_current);
    ctl->velocity_state = next_velocity_state(ctl->velocity_state, t_current);
    ctl->t_current = t_current + P.dt;
    ctl->iter = iter + 1;
}

// Contacts, forces and integration of sorted particle k (the particle work
// of k_contacts_integrate).  After a device error (raised by an earlier
// step, or by this particle's contact search) the particle's state is
// carried to the other buffer unchanged.
template <int PREC, int MODEL>
__device__ __forceinline__ void contacts_integrate_particle(const DevParams &P, const DevState &S,
                                                            unsigned k, uint32_t *srow)
{
    DevCtl *ctl = S.ctl;
    if (ctl->err) {
        carry_particle(S, k);
        return;
    }
    StepClock clk;
    clk.iter = ctl->iter;
    clk.t_current = ctl->t_current;
    clk.velocity_state = ctl->velocity_state;
    clk.tau_eff_x = ctl->tau_eff_x;
    ContactOut c;
    if (!contact_particle<PREC, MODEL>(P, S, k, srow, blockDim.x, threadIdx.x, c)) {
        carry_particle(S, k);
        return;
    }
    contact_writeback(P, S, k, c);
    integrate_particle(P, S, k, make_double4(c.F.x, c.F.y, c.F.z, 0.0f),
                       make_double4(c.T.x, c.T.y, c.T.z, 0.0f), clk, S.x_nx, S.vel_nx,
                       S.angvel_nx, S.vel_f_nx, S.angvel_f_nx, &ctl->resort_next, &ctl->nl_next);
}

// The contact stage and the particle integration of one DEM step in one
// launch, for dry boxes without bonds, fluid or a shear-stress wall (their
// forces would have to join before the integration).  Thread k runs sorted
// particle k's contact search and forces, writes them back, then integrates
// it into the other buffer of the x / vel / angvel ping-pong pair
// (S.x_nx, ...).  Every partner is read from the current buffer, which no
// thread of this launch writes, so the particles advance exactly as with
// k_contacts followed by k_integrate.  The cell and list flags of the next
// step go to DevCtl::resort_next / nl_next; the wall reduction, the wall
// update and the loop counters follow in k_walls_step.
template <int PREC, int MODEL>
__global__ void __launch_bounds__(SPHB_CONTACT_B, SPHB_CONTACT_MINB)
k_contacts_integrate(DevParams P, DevState S)
{
    extern __shared__ uint32_t srow[];   // blockDim * nc slot partners
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < P.np) contacts_integrate_particle<PREC, MODEL>(P, S, k, srow);
}

}  // namespace sphb
