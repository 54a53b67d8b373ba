// DEM step kernels, FP64 (faithful and true-FP64 lengths).
//
// Compiled with -fmad=false: every expression keeps the reference's
// operation order and rounding (the reference is built with --fmad=false,
// src/CMakeLists.txt:25).  One thread per particle in sorted order.
#include "dem_state.h"
#include "dem_launch.h"

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

// Neighbour list build: runs every step, works only when DevCtl::nl_rebuild.
__global__ void __launch_bounds__(128) k_nl_build(DevParams P, DevState S)
{
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (S.ctl->err || !S.ctl->nl_rebuild || k >= P.np) return;
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
    if (k == 0) S.ctl->nl_builds += 1;
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

template <int PREC, int MODEL>
__global__ void __launch_bounds__(128) k_contacts(DevParams P, DevState S)
{
    extern __shared__ uint32_t srow[];
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0 && S.ctl->nl_rebuild) S.ctl->nl_rebuild = 0;  // k_nl_build has run
    if (S.ctl->err || k >= P.np) return;
    const unsigned B = blockDim.x, t = threadIdx.x;
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
            double len = vlen<PREC>(xab);
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
        if (!ok) return;
        // --- interact, history contacts in slot order ---
        uint64_t m = mask;
        while (m) {
            const int i = __ffsll((long long)m) - 1;
            m &= m - 1;
            const unsigned b_orig = srow[i * B + t];
            if (b_orig >= P.np) { raise_err(S.ctl, DERR_CAPACITY, (int)o); return; }
            const size_t mempos = rowbase + i;
            V3 dm = dm_decode(P, S.dmcode[mempos]);
            unsigned kb = S.pos_of[b_orig];
            double4 xb = S.x[kb];
            double rb = xb.w;
            V3 x_ab = mk3(xa.x - xb.x + dm.x, xa.y - xb.y + dm.y, xa.z - xb.z + dm.z);
            double len = vlen<PREC>(x_ab);
            double delta_n = len - (ra + rb);
            if (delta_n < 0.0) {
                V3 dt_new = contact_linear<PREC>(P, F, T, es_dot, ev_dot, p, vel_a, angvel_a,
                                                 S.vel[kb], xyz(S.angvel[kb]),
                                                 S.delta_t[mempos], ra, rb, x_ab, len, delta_n);
                S.delta_t[mempos] = make_double4(dt_new.x, dt_new.y, dt_new.z, 0.0);
            } else {
                mask &= ~(1ull << i);
                written |= 1ull << i;
                S.delta_t[mempos] = make_double4(0.0, 0.0, 0.0, 0.0);
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
            double len = vlen<PREC>(x_ab);
            double delta_ab = len - (ra + rb);
            if (delta_ab < 0.0f)
                contact_linear_viscous<PREC>(P, F, T, p, vel_a, angvel_a, S.vel[b],
                                             xyz(S.angvel[b]), ra, rb, x_ab, len, delta_ab,
                                             P.kappa);
            else if (delta_ab < P.db)
                capillary_exp<PREC>(P, F, ra, rb, delta_ab, x_ab, len, P.kappa);
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

    // --- walls (contactsearch.cuh:602-701) ---
    double4 wnx[5] = {make_double4(0.0f, 0.0f, -1.0f, P.L[2]), make_double4(-1.0f, 0.0f, 0.0f, P.L[0]),
                      make_double4(1.0f, 0.0f, 0.0f, 0.0f), make_double4(0.0f, -1.0f, 0.0f, P.L[1]),
                      make_double4(0.0f, 1.0f, 0.0f, 0.0f)};
    double wvel[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (unsigned w = 0; w < P.nw && w < 5; ++w) {
        wnx[w] = S.wnx[w];
        wvel[w] = S.wmvfd[w].y;
    }
    double wf[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    V3 vlin = xyz(vel_a);
    double dw = wnx[0].w - (xa.z + ra);
    if (dw < 0.0f)
        wf[0] = contact_wall<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a, xyz(wnx[0]), dw, wvel[0]);
    dw = xa.z - ra - P.origo[2];
    if (dw < 0.0f)
        (void)contact_wall<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a,
                                 mk3(0.0f, 0.0f, 1.0f), dw, 0.0);
    if (P.periodic == 0) {
        dw = wnx[1].w - (xa.x + ra);
        if (dw < 0.0f)
            wf[1] = contact_wall<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a, xyz(wnx[1]), dw, wvel[1]);
        dw = xa.x - ra - wnx[2].w;
        if (dw < 0.0f)
            wf[2] = contact_wall<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a, xyz(wnx[2]), dw, wvel[2]);
    }
    if (P.periodic == 0 || P.periodic == 2) {
        dw = wnx[3].w - (xa.y + ra);
        if (dw < 0.0f)
            wf[3] = contact_wall<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a, xyz(wnx[3]), dw, wvel[3]);
        dw = xa.y - ra - wnx[4].w;
        if (dw < 0.0f)
            wf[4] = contact_wall<PREC>(P, F, T, es_dot, ev_dot, p, ra, vlin, angvel_a, xyz(wnx[4]), dw, wvel[4]);
    }
    // --- write-back (contactsearch.cuh:706-724) ---
    S.force[k] = make_double4(F.x, F.y, F.z, 0.0f);
    S.torque[k] = make_double4(T.x, T.y, T.z, 0.0f);
    S.es_dot[k] = es_dot;
    S.ev_dot[k] = ev_dot;
    S.es[k] += es_dot * P.dt;
    S.ev[k] += ev_dot * P.dt;
    S.p[k] = p;
    for (unsigned w = 0; w < P.nw && w < 5; ++w) S.walls_force_pp[o + (size_t)P.np * w] = wf[w];
}

// Occupancy masks of the slot rows (after the rows were set from the host).
__global__ void k_occ_from_rows(DevParams P, DevState S)
{
    unsigned o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= P.np) return;
    uint64_t m = 0;
    for (unsigned i = 0; i < P.nc; ++i)
        if (S.contacts[(size_t)o * P.nc + i] != P.np) m |= 1ull << i;
    S.occ[o] = m;
}
// ---------------------------------------------------------------------
// bondsLinear, src/cohesion.cuh:8-233: one thread per bond computes the
// bond state; forces are added per particle in bond order (k_bond_gather)
// instead of the reference's unsynchronised `+=`.
// ---------------------------------------------------------------------
template <int PREC>
__global__ void k_bonds(DevParams P, DevState S, double4 *bond_f, double4 *bond_t)
{
    unsigned idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (S.ctl->err || idx >= P.nb0) return;
    const double dt = P.dt;
    uint2 bond = S.bonds[idx];
    bond_f[idx] = make_double4(0.0, 0.0, 0.0, 0.0);
    bond_t[idx] = make_double4(0.0, 0.0, 0.0, -1.0);  // w < 0: no contribution
    if (!(bond.x < P.np)) return;
    if (bond.y >= P.np) { raise_err(S.ctl, DERR_BOND, (int)idx); return; }
    double4 d0 = S.bonds_delta[idx], w0 = S.bonds_omega[idx];
    V3 delta0_t = xyz(d0);
    double delta0_n = d0.w;
    V3 omega0_t = xyz(w0);
    double omega0_n = w0.w;
    unsigned ki = S.pos_of[bond.x], kj = S.pos_of[bond.y];
    double4 x_i = S.x[ki], x_j = S.x[kj], vel_i = S.vel[ki], vel_j = S.vel[kj];
    V3 angvel_i = xyz(S.angvel[ki]), angvel_j = xyz(S.angvel[kj]);
    double R_bar = P.lambda_bar * fmin(x_i.w, x_j.w);
    double A = SPHB_PI * R_bar * R_bar;
    double I = 0.25 * SPHB_PI * R_bar * R_bar * R_bar * R_bar;
    double J = I * 2.0;
    V3 x = mk3(x_i.x - x_j.x, x_i.y - x_j.y, x_i.z - x_j.z);
    double x_length = vlen<PREC>(x);
    double overlap = fmin(0.0, x_length - (x_i.w + x_j.w));
    V3 n = divs3(x, x_length);
    delta0_t = sub3(delta0_t, muls3(n, dot3(n, delta0_t)));
    V3 ddelta = muls3(add3(add3(mk3(vel_i.x - vel_j.x, vel_i.y - vel_j.y, vel_i.z - vel_j.z),
                                smul3(x_i.w + overlap / 2.0, cross3(n, angvel_i))),
                           smul3(x_j.w + overlap / 2.0, cross3(n, angvel_j))),
                      dt);
    double ddelta_n = -dot3(ddelta, n);
    double delta_n = delta0_n + ddelta_n;
    V3 ddelta_t = sub3(ddelta, muls3(n, dot3(n, ddelta)));
    V3 delta_t = add3(delta0_t, ddelta_t);
    V3 f_n = smul3(P.k_n * A * delta_n + P.gamma_n * ddelta_n / dt, n);
    V3 f_t = sub3(smul3(-P.k_t * A, delta_t), divs3(smul3(P.gamma_t, ddelta_t), dt));
    V3 f = add3(f_n, f_t);
    V3 nn = neg3(n);
    omega0_t = sub3(omega0_t, muls3(nn, dot3(omega0_t, nn)));
    V3 domega = muls3(mk3(angvel_j.x - angvel_i.x, angvel_j.y - angvel_i.y,
                          angvel_j.z - angvel_i.z), dt);
    double domega_n = dot3(domega, nn);
    double omega_n = omega0_n + domega_n;
    V3 domega_t = sub3(domega, smul3(domega_n, nn));
    V3 omega_t = add3(omega0_t, domega_t);
    V3 t_n = smul3(-P.k_t * J * omega_n, nn);
    V3 t_t = smul3(-P.k_n * I, omega_t);
    V3 t_j = add3(t_n, t_t);
    double sigma_max = vlen<PREC>(f_n) / A + vlen<PREC>(t_t) * R_bar / I;
    double tau_max = vlen<PREC>(f_t) / A + vlen<PREC>(t_n) * R_bar / J;
    if (sigma_max >= P.sigma_b || tau_max >= P.tau_b) {
        S.bonds[idx].x = P.nb0;  // cohesion.cuh:205
        return;
    }
    S.bonds_delta[idx] = make_double4(delta_t.x, delta_t.y, delta_t.z, delta_n);
    S.bonds_omega[idx] = make_double4(omega_t.x, omega_t.y, omega_t.z, omega_n);
    bond_f[idx] = make_double4(f.x, f.y, f.z, 0.0);
    bond_t[idx] = make_double4(t_j.x, t_j.y, t_j.z, 1.0);
}

// Adds each particle's bond forces in increasing bond order.  bond_list
// entries are (bond index << 1) | (1 if the particle is bond.y).
__global__ void k_bond_gather(DevParams P, DevState S, const double4 *bond_f,
                              const double4 *bond_t)
{
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (S.ctl->err || k >= P.np) return;
    unsigned o = S.orig_of[k];
    unsigned b0 = S.bond_ptr[o], b1 = S.bond_ptr[o + 1];
    if (b0 == b1) return;
    double4 f = S.force[k], tq = S.torque[k];
    for (unsigned j = b0; j < b1; ++j) {
        unsigned e = S.bond_list[j];
        unsigned b = e >> 1;
        double4 bt = bond_t[b];
        if (bt.w < 0.0) continue;
        double4 bf = bond_f[b];
        if ((e & 1) == 0) {
            f.x += bf.x; f.y += bf.y; f.z += bf.z; f.w += 0.0;
            tq.x -= bt.x; tq.y -= bt.y; tq.z -= bt.z; tq.w -= 0.0;
        } else {
            f.x -= bf.x; f.y -= bf.y; f.z -= bf.z; f.w -= 0.0;
            tq.x += bt.x; tq.y += bt.y; tq.z += bt.z; tq.w += 0.0;
        }
    }
    S.force[k] = f;
    S.torque[k] = tq;
}

// findShearStressOnFixedMovingParticles, src/integration.cuh:457-484
__global__ void k_shear_stress(DevParams P, DevState S)
{
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (S.ctl->err || k >= P.np) return;
    double z = S.x[k].z, fixvel = S.vel[k].w, force_x = S.force[k].x;
    double f_x = 0.0;
    if (fixvel > 0.0 && z > P.L[2] * 0.5) f_x = force_x;
    S.tau_pp[S.orig_of[k]] = f_x / (P.L[0] * P.L[1]);
}

// summation, src/integration.cuh:309-341: per-block partial sums over
// 256 consecutive ORIGINAL indices with the same tree as the reference.
// The block that finishes last also adds the partials in block order,
// as integrate/integrateWalls do (integration.cuh:67-68, 376-378).
__device__ double block_tree_sum(const double *in, unsigned np, unsigned nblocks, double *cache)
{
    unsigned t = threadIdx.x;
    unsigned idx = t + blockIdx.x * 256;
    double temp = 0.0f;
    while (idx < np) {
        temp += in[idx];
        idx += 256 * nblocks;
    }
    cache[t] = temp;
    __syncthreads();
    for (unsigned i = 128; i != 0; i /= 2) {
        if (t < i) cache[t] += cache[t + i];
        __syncthreads();
    }
    return cache[0];
}

__global__ void __launch_bounds__(256) k_tau_partials(DevParams P, DevState S)
{
    __shared__ double cache[256];
    __shared__ bool last;
    if (S.ctl->err) return;
    double s = block_tree_sum(S.tau_pp, P.np, P.nblocks256, cache);
    if (threadIdx.x == 0) {
        S.tau_partials[blockIdx.x] = s;
        __threadfence();
        last = atomicAdd(&S.ctl->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double tau = 0.0;
        for (unsigned i = 0; i < P.nblocks256; ++i) tau += ((volatile double *)S.tau_partials)[i];
        S.ctl->tau_eff_x = tau;
        S.ctl->ticket = 0;
    }
}

// ---------------------------------------------------------------------
// integrate, src/integration.cuh:14-305 (TY3 default, TY2 selectable),
// then the cell hash of the new position (src/sorting.cuh:7-51) so the
// next step knows whether the sort changes.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_integrate(DevParams P, DevState S)
{
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (S.ctl->err || k >= P.np) return;
    const long long iter = S.ctl->iter;
    const double t_current = S.ctl->t_current;
    // rate-state velocity step (device.cu:2461-2469), decided from the
    // loop state before this step
    int change_velocity_state = 0;
    {
        int vs = S.ctl->velocity_state;
        if (t_current >= 10.0 && t_current < 15.0 && vs == 1) change_velocity_state = 1;
        else if (t_current >= 15.0 && vs == 2) change_velocity_state = -1;
    }
    const double velocity_factor = 10.0;
    double4 force = S.force[k], torque = S.torque[k], angpos = S.angpos[k];
    double4 x = S.x[k], vel = S.vel[k], angvel = S.angvel[k];
    double4 xyzsum = S.xyzsum[k];
    int wall0mode = 0;
    double wall0mass = 0.0;
    if (P.nw > 0) {
        wall0mode = P.wmode[0];
        wall0mass = S.wmvfd[0].x;
    }
    double tau_eff_x = 0.0;
    if (P.nw > 0 && wall0mode == 3) tau_eff_x = S.ctl->tau_eff_x;
    double4 acc0 = make_double4(0, 0, 0, 0), angacc0 = make_double4(0, 0, 0, 0);
    if (iter != 0) {
        acc0 = S.acc[k];
        angacc0 = S.angacc[k];
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
    S.angvel[k] = angvel_new;
    S.vel[k] = vel_new;
    S.angpos[k] = angpos_new;
    S.x[k] = x_new;
    // cell of the new position
    int ix, iy, iz;
    if (!cell_coord(P, x_new.x, 0, ix) || !cell_coord(P, x_new.y, 1, iy) ||
        !cell_coord(P, x_new.z, 2, iz)) {
        raise_err(S.ctl, DERR_OUTSIDE, (int)S.orig_of[k]);
        return;
    }
    unsigned c = ((unsigned)iz * P.num[1]) * P.num[0] + (unsigned)iy * P.num[0] + (unsigned)ix;
    S.cell_new[k] = c;
    if (c != S.cell_of[k]) S.ctl->resort = 1;
    // neighbour lists stay exact while every particle is within 0.45 skin
    // of its position at the build
    float4 xr = S.x_ref[k];
    double ddx = x_new.x - (double)xr.x, ddy = x_new.y - (double)xr.y, ddz = x_new.z - (double)xr.z;
    double lim = 0.45 * P.skin;
    if (ddx * ddx + ddy * ddy + ddz * ddz > lim * lim) S.ctl->nl_rebuild = 1;
}

// Cell hash of the current positions (first step, after sph_set).
__global__ void k_hash(DevParams P, DevState S)
{
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P.np) return;
    double4 x = S.x[k];
    int ix, iy, iz;
    if (!cell_coord(P, x.x, 0, ix) || !cell_coord(P, x.y, 1, iy) || !cell_coord(P, x.z, 2, iz)) {
        raise_err(S.ctl, DERR_OUTSIDE, (int)S.orig_of[k]);
        return;
    }
    S.cell_new[k] = ((unsigned)iz * P.num[1]) * P.num[0] + (unsigned)iy * P.num[0] + (unsigned)ix;
}

// Wall-force partial sums + integrateWalls (integration.cuh:344-450) in
// the block that finishes last, then the loop counters
// (device.cu:2543-2545).  With nw == 0 it runs as one block and only
// advances the counters.
__global__ void __launch_bounds__(256) k_walls_and_clock(DevParams P, DevState S)
{
    __shared__ double cache[256];
    __shared__ bool last;
    DevCtl *ctl = S.ctl;
    if (ctl->err) return;
    if (P.nw > 0) {
        double s = block_tree_sum(S.walls_force_pp, P.np, P.nblocks256, cache);
        if (threadIdx.x == 0) {
            S.partials[blockIdx.x] = s;
            __threadfence();
            last = atomicAdd(&ctl->ticket, 1u) == gridDim.x - 1;
        }
        __syncthreads();
    } else {
        if (threadIdx.x == 0) last = true;
        __syncthreads();
    }
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    const long long iter = ctl->iter;
    const double t_current = ctl->t_current;
    const double dt = P.dt;
    for (unsigned w = 0; w < P.nw; ++w) {
        double4 w_nx = S.wnx[w], w_mvfd = S.wmvfd[w];
        int wmode = P.wmode[w];
        if (wmode == 0) continue;
        double acc0 = iter == 0 ? 0.0 : S.wacc[w];
        w_mvfd.z = 0.0;
        for (unsigned b = 0; b < P.nblocks256; ++b) w_mvfd.z += ((volatile double *)S.partials)[b];
        double sigma_0 = w_mvfd.w + P.sigma0_A * sin(2.0 * SPHB_PI * P.sigma0_f * t_current);
        double N = -sigma_0 * P.L[0] * P.L[1];
        double acc = (w_mvfd.z + N) / w_mvfd.x;
        if (wmode == 2) acc = 0.0;
        if (P.integrator == 3) {
            double dacc_dt = (acc - acc0) / dt;
            w_nx.w += w_mvfd.y * dt + 0.5 * acc * dt * dt + 1.0 / 6.0 * dacc_dt * dt * dt * dt;
            w_mvfd.y += acc * dt + 0.5 * dacc_dt * dt * dt;
        } else {
            w_nx.w += w_mvfd.y * dt + 0.5 * acc * dt * dt;
            w_mvfd.y += acc * dt;
        }
        S.wnx[w] = w_nx;
        S.wmvfd[w] = w_mvfd;
        S.wacc[w] = acc;
    }
    // rate-state bookkeeping (device.cu:2461-2469)
    int vs = ctl->velocity_state;
    if (t_current >= 10.0 && t_current < 15.0 && vs == 1) ctl->velocity_state = 2;
    else if (t_current >= 15.0 && vs == 2) ctl->velocity_state = 1;
    ctl->t_current = t_current + dt;
    ctl->iter = iter + 1;
    ctl->ticket = 0;
}

// ---------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------
static inline unsigned blocks_for(unsigned n, unsigned b) { return (n + b - 1) / b; }

cudaError_t launch_contacts(const DevParams &P, const DevState &S, int prec, cudaStream_t st)
{
    if (P.np == 0) return cudaSuccess;
    const unsigned B = 128;
    k_nl_build<<<blocks_for(P.np, B), B, 0, st>>>(P, S);
    size_t smem = (P.contactmodel == 2) ? (size_t)B * P.nc * sizeof(uint32_t) : 0;
    dim3 grid(blocks_for(P.np, B));
    if (P.contactmodel == 2) {
        if (prec == 0) {
            cudaFuncSetAttribute(k_contacts<0, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_contacts<0, 2><<<grid, B, smem, st>>>(P, S);
        } else {
            cudaFuncSetAttribute(k_contacts<1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_contacts<1, 2><<<grid, B, smem, st>>>(P, S);
        }
    } else {
        if (prec == 0) k_contacts<0, 1><<<grid, B, 0, st>>>(P, S);
        else k_contacts<1, 1><<<grid, B, 0, st>>>(P, S);
    }
    return cudaGetLastError();
}

cudaError_t launch_bonds(const DevParams &P, const DevState &S, int prec, double4 *bf,
                         double4 *bt, cudaStream_t st)
{
    if (P.nb0 == 0) return cudaSuccess;
    if (prec == 0) k_bonds<0><<<blocks_for(P.nb0, 256), 256, 0, st>>>(P, S, bf, bt);
    else k_bonds<1><<<blocks_for(P.nb0, 256), 256, 0, st>>>(P, S, bf, bt);
    k_bond_gather<<<blocks_for(P.np, 256), 256, 0, st>>>(P, S, bf, bt);
    return cudaGetLastError();
}

cudaError_t launch_integrate(const DevParams &P, const DevState &S, cudaStream_t st)
{
    if (P.np > 0) {
        if (P.nw > 0 && P.wmode[0] == 3) {
            k_shear_stress<<<blocks_for(P.np, 256), 256, 0, st>>>(P, S);
            k_tau_partials<<<P.nblocks256, 256, 0, st>>>(P, S);
        }
        k_integrate<<<blocks_for(P.np, 256), 256, 0, st>>>(P, S);
    }
    unsigned g = (P.nw > 0 && P.np > 0) ? P.nblocks256 : 1;
    k_walls_and_clock<<<g, 256, 0, st>>>(P, S);
    return cudaGetLastError();
}

cudaError_t launch_occ_from_rows(const DevParams &P, const DevState &S, cudaStream_t st)
{
    if (P.np == 0) return cudaSuccess;
    k_occ_from_rows<<<blocks_for(P.np, 256), 256, 0, st>>>(P, S);
    return cudaGetLastError();
}

cudaError_t launch_hash(const DevParams &P, const DevState &S, cudaStream_t st)
{
    if (P.np == 0) return cudaSuccess;
    k_hash<<<blocks_for(P.np, 256), 256, 0, st>>>(P, S);
    return cudaGetLastError();
}

}  // namespace sphb
