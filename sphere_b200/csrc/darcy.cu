// Darcy porosity-coupled pressure solver (cfd_solver 1) on the device.
//
// Follows the cfd_solver == 1 block of DEM::startTime
// (src/device.cu:1901-2426) and the kernels of src/darcy.cuh, compiled with
// -fmad=false like the reference.  Fields are ghost-padded
// (nx+2)(ny+2)(nz+2) doubles (src/darcy.cpp:36-40).  The Jacobi fixed point
// (firstDarcySolution + updateDarcySolution + copyValues, repeated) runs as
// one cooperative kernel: ping-pong pressure buffers, each cell writes the
// ghost faces that depend on it right after its update, the residual
// maximum is reduced on the device every iteration, and the reference's
// stopping rule (checked after iteration 0 and every 10th iteration) is
// applied on the device -- no host round trip per check.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "dem_device.cuh"
#include "warmstart.h"
#include "../../include/sphere_b200.h"

namespace sphb {

struct DarcyParams {
    int nx, ny, nz;
    double dx, dy, dz;
    double mu, rho_f, beta_f, k_c, c_phi, tolerance;
    double p_mod_A, p_mod_f, p_mod_phi, p_top_orig;
    double bc_bot_flux, bc_top_flux;
    int bc_xn, bc_xp, bc_yn, bc_yp, bc_bot, bc_top;
    unsigned maxiter, ndem;
    unsigned inject;               // 1: the Jacobi waits never succeed (a test knob)
};

struct DarcyCtl {
    unsigned wall0_iz;             // from the host copy of the wall (file outputs)
    long long nijac_last;          // the reference's nijac at the end of the solve
    long long nijac_total;         // iterations performed since open
    long long converged_at;        // first iteration whose residual met the tolerance
    int converged;                 // 1: the last solve stopped at a residual check
    unsigned long long res_bits[3];  // |residual| maxima as ordered bit patterns, 3-slot ring
    int final_buf;                 // buffer holding the final pressure (0: p, 1: p2)
    unsigned barrier_count, barrier_gen;
    int err;
    // learned warm start: first-iteration residuals of the previous-step
    // guess (0) and of the network's guess (1); solves that used the latter
    unsigned long long guess_res[3];
    long long ws_picked;
};

// Synchronisation of the cooperative Jacobi kernel (zeroed before each
// launch).  Block b owns a contiguous range of cells and publishes in
// done[b] how many iterations it has completed; an iteration only needs the
// previous iterate of the cells within one z layer, so a block waits for
// the few blocks around it instead of the whole grid.  The residual maxima
// go to a ring of per-iteration slots; the check iterations of the stop rule
// count their arrivals so every block can read a complete maximum.  Each
// counter has its own 128-byte line.
constexpr unsigned kJacobiMaxBlocks = 1024;
constexpr unsigned kJacobiRing = 64;     // residual slots (iterations mod 64)
constexpr unsigned kJacobiChecks = 8;    // arrival counters (check index mod 8)
struct JacobiSync {
    unsigned long long ring[kJacobiRing];
    unsigned arrive[kJacobiChecks][32];
    unsigned done[kJacobiMaxBlocks][32];
};

// Constants of one solve's Jacobi update, independent of the iterate and
// formed once per fluid step with the reference's operation order, so the
// iteration reproduces updateDarcySolution's arithmetic bit for bit while
// reading 9 values per cell instead of 24 and dividing 9 times fewer.
struct JacobiCoef {
    const double *cf;      // 6 x ng: face factors 2 k_nb k / (k_nb + k): xp, xn, yp, yn, zp, zn
    const double *a;       // ndt / (beta_f phi mu)
    const double *src;     // ndt / (beta_f phi (1 - phi)) * (dphi / ndt + v_p . grad phi)
    const double *base;    // p_old + (1 - epsilon) dp_expl
    const unsigned char *fixed;  // 1 where the pressure change is forced to 0
    unsigned long long ng;
};

struct DarcyDev {
    DarcyParams D;
    size_t ng;
    double *cf = nullptr, *ca = nullptr, *csrc = nullptr, *cbase = nullptr;
    unsigned char *cfixed = nullptr;
    double *p, *p2, *p_old, *dp_expl, *phi, *dphi, *k, *div_v_p;
    double *v, *vp_avg, *grad_p, *grad_k;  // 3 doubles per cell
    int *p_constant;
    double4 *f_p;                          // original particle order
    double *gather;                        // nx*ny*nz*3 doubles for field reads
    DarcyCtl *ctl;
    JacobiSync *jsync;
    double host_wall0_w;
    long long conv_iters_last;
    // learned warm start (null when off)
    WarmStart *ws = nullptr;
    unsigned char *freec = nullptr;        // cells the solve may change
    double *guess = nullptr;               // padded guess (extrapolation + network)
    double *guess_base = nullptr;          // padded extrapolation alone (learned mode)
};

__device__ __forceinline__ unsigned didx(const DarcyParams &D, int x, int y, int z)
{
    return (unsigned)(x + 1) + ((unsigned)D.nx + 2u) * (unsigned)(y + 1) +
           ((unsigned)D.nx + 2u) * ((unsigned)D.ny + 2u) * (unsigned)(z + 1);
}

__device__ __forceinline__ bool cell_of_thread(const DarcyParams &D, int &x, int &y, int &z)
{
    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned n = (unsigned)D.nx * D.ny * D.nz;
    if (i >= n) return false;
    x = (int)(i % D.nx);
    y = (int)((i / D.nx) % D.ny);
    z = (int)(i / ((unsigned)D.nx * D.ny));
    return true;
}

// setDarcyGhostNodes<T>, darcy.cuh:194-264 (comps doubles per cell)
template <int C>
__device__ __forceinline__ void ghost_from(const DarcyParams &D, double *f, int x, int y, int z,
                                           const double *val)
{
    const int nx = D.nx, ny = D.ny, nz = D.nz;
    auto put = [&](int X, int Y, int Z) {
        double *d = &f[(size_t)C * didx(D, X, Y, Z)];
        for (int c = 0; c < C; ++c) d[c] = val[c];
    };
    if (x == 0 && D.bc_xn == 0) put(-1, y, z);
    if (x == 1 && D.bc_xn == 1) put(-1, y, z);
    if (x == 0 && D.bc_xn == 2) put(nx, y, z);
    if (x == nx - 1 && D.bc_xp == 0) put(nx, y, z);
    if (x == nx - 2 && D.bc_xp == 1) put(nx, y, z);
    if (x == nx - 1 && D.bc_xp == 2) put(-1, y, z);
    if (y == 0 && D.bc_yn == 0) put(x, -1, z);
    if (y == 1 && D.bc_yn == 1) put(x, -1, z);
    if (y == 0 && D.bc_yn == 2) put(x, ny, z);
    if (y == ny - 1 && D.bc_yp == 0) put(x, ny, z);
    if (y == ny - 2 && D.bc_yp == 1) put(x, ny, z);
    if (y == ny - 1 && D.bc_yp == 2) put(x, -1, z);
    if (z == 0 && D.bc_bot == 0) put(x, y, -1);
    if (z == 1 && D.bc_bot == 1) put(x, y, -1);
    if (z == 0 && D.bc_bot == 2) put(x, y, nz);
    if (z == nz - 1 && D.bc_top == 0) put(x, y, nz);
    if (z == nz - 2 && D.bc_top == 1) put(x, y, nz);
    if (z == nz - 1 && D.bc_top == 2) put(x, y, -1);
}

template <int C>
__global__ void k_ghost(DarcyParams D, double *f)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    double val[C];
    const double *s = &f[(size_t)C * didx(D, x, y, z)];
    for (int c = 0; c < C; ++c) val[c] = s[c];
    ghost_from<C>(D, f, x, y, z, val);
}

// flux ghost value below/above cell (x,y,z) from its pressure p
// (setDarcyGhostNodesFlux, darcy.cuh:270-312)
__device__ __forceinline__ void flux_ghost(const DarcyParams &D, const double *k, double *dst,
                                           int x, int y, int z, double p)
{
    const double kk = k[didx(D, x, y, z)];
    const double dz = D.dz;
    double q_z = 0.;
    if (z == 0) q_z = D.bc_bot_flux;
    else if (z == D.nz - 1) q_z = D.bc_top_flux;
    const double p_ghost = -D.mu / kk * q_z * dz + p;
    if (z == 0 && D.bc_bot == 4) dst[didx(D, x, y, -1)] = p_ghost;
    if (z == D.nz - 1 && D.bc_top == 4) dst[didx(D, x, y, D.nz)] = p_ghost;
}

// Inside the fused Jacobi loop the flux ghosts and the ordinary ghosts of
// the next iterate are written in the same pass; the reference writes the
// ordinary ghosts later (at the start of the next iteration), so where both
// target one face (a periodic partner face) the ordinary ghost wins.
__device__ __forceinline__ void flux_ghost_next(const DarcyParams &D, const double *k, double *dst,
                                                int x, int y, int z, double p)
{
    const double kk = k[didx(D, x, y, z)];
    double q_z = 0.;
    if (z == 0) q_z = D.bc_bot_flux;
    else if (z == D.nz - 1) q_z = D.bc_top_flux;
    const double p_ghost = -D.mu / kk * q_z * D.dz + p;
    if (z == 0 && D.bc_bot == 4 && D.bc_top != 2) dst[didx(D, x, y, -1)] = p_ghost;
    if (z == D.nz - 1 && D.bc_top == 4 && D.bc_bot != 2) dst[didx(D, x, y, D.nz)] = p_ghost;
}

__global__ void k_flux_ghost(DarcyParams D, double *p, const double *k)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    flux_ghost(D, k, p, x, y, z, p[didx(D, x, y, z)]);
}

__global__ void k_copy_interior(DarcyParams D, const double *src, double *dst)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    unsigned c = didx(D, x, y, z);
    dst[c] = src[c];
}

__global__ void k_zero_interior(DarcyParams D, double *f)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    f[didx(D, x, y, z)] = 0.0;
}

// findDarcyPressureGradient, darcy.cuh:889-943
__global__ void k_pressure_gradient(DarcyParams D, const double *p, double *grad_p)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    double *g = &grad_p[3 * (size_t)didx(D, x, y, z)];
    g[0] = (p[didx(D, x + 1, y, z)] - p[didx(D, x - 1, y, z)]) / (D.dx + D.dx);
    g[1] = (p[didx(D, x, y + 1, z)] - p[didx(D, x, y - 1, z)]) / (D.dy + D.dy);
    g[2] = (p[didx(D, x, y, z + 1)] - p[didx(D, x, y, z - 1)]) / (D.dz + D.dz);
}

__device__ __forceinline__ double sphere_volume(double r)
{
    // 4/3 pi r^3 with the reference's M_PI and pow (darcy.cuh:318-321)
    return 4.0 / 3.0 * 3.14159265358979323846 * pow(r, 3.0);
}

__device__ __forceinline__ double weight_dist(V3 d, double dx, double dy, double dz)
{
    V3 a = mk3(fabs(d.x), fabs(d.y), fabs(d.z));
    if (a.x < dx && a.y < dy && a.z < dz)
        return (1.0 - a.x / dx) * (1.0 - a.y / dy) * (1.0 - a.z / dz);
    return 0.0;
}

// findDarcyPressureForceLinear, darcy.cuh:948-1102 (one thread per particle
// in sorted order; force[k] += f_p; f_p kept at the original index)
__global__ void k_pressure_force(DevParams P, DevState S, DarcyParams D, const double *grad_p,
                                 const DarcyCtl *dctl, double4 *f_p_out)
{
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (S.ctl->err || k >= P.np) return;
    const unsigned nx = (unsigned)D.nx, ny = (unsigned)D.ny, nz = (unsigned)D.nz;
    const double dx = D.dx, dy = D.dy, dz = D.dz;
    const unsigned wall0_iz = dctl->wall0_iz;
    double4 x = S.x[k];
    unsigned i_x = (unsigned)floor((x.x - P.origo[0]) / (P.L[0] / P.num[0]));
    unsigned i_y = (unsigned)floor((x.y - P.origo[1]) / (P.L[1] / P.num[1]));
    unsigned i_z = (unsigned)floor((x.z - P.origo[2]) / (P.L[2] / P.num[2]));
    if (i_x >= nx || i_y >= ny || i_z >= nz) {
        // the 27 reads below would leave the padded grid
        raise_err(S.ctl, DERR_OUTSIDE, (int)S.orig_of[k]);
        return;
    }
    V3 X = mk3(i_x * dx + 0.5 * dx, i_y * dy + 0.5 * dy, i_z * dz + 0.5 * dz);
    V3 gp = mk3(0., 0., 0.);
    for (int d_iz = -1; d_iz < 2; d_iz++)
        for (int d_iy = -1; d_iy < 2; d_iy++)
            for (int d_ix = -1; d_ix < 2; d_ix++) {
                int ix_n = (int)i_x + d_ix, iy_n = (int)i_y + d_iy, iz_n = (int)i_z + d_iz;
                const double *gs = &grad_p[3 * (size_t)didx(D, ix_n, iy_n, iz_n)];
                V3 g = mk3(gs[0], gs[1], gs[2]);
                if ((ix_n == -1 && iy_n == -1) || (ix_n == -1 && iz_n == -1) ||
                    (iy_n == -1 && iz_n == -1) || (ix_n == (int)nx && iy_n == (int)ny) ||
                    (ix_n == (int)nx && iz_n == (int)nz) || (iy_n == (int)ny && iz_n == (int)nz) ||
                    (ix_n == (int)nx && iy_n == -1) || (ix_n == (int)nx && iz_n == -1) ||
                    (iy_n == (int)ny && ix_n == -1) || (iy_n == (int)ny && iz_n == -1) ||
                    (iz_n == (int)nz && ix_n == -1) || (iz_n == (int)nz && iy_n == -1))
                    g = mk3(0., 0., 0.);
                // unsigned comparison, as in the reference
                if (D.bc_top == 0 && i_z + (unsigned)d_iz >= wall0_iz - 1u) g.z = 0.0;
                V3 n = mk3(dx * d_ix, dy * d_iy, dz * d_iz);
                V3 xf = mk3(X.x + n.x, X.y + n.y, X.z + n.z);
                double w = weight_dist(mk3(x.x - xf.x, x.y - xf.y, x.z - xf.z), dx, dy, dz);
                gp = add3(gp, smul3(w, g));
            }
    const double v = sphere_volume(x.w);
    const double rv = D.rho_f * v;
    V3 f_p = mk3((-1.0 * gp.x) * v - rv * P.g[0], (-1.0 * gp.y) * v - rv * P.g[1],
                 (-1.0 * gp.z) * v - rv * P.g[2]);
    if (D.bc_top == 0 && i_z >= wall0_iz) f_p.z = 0.0;
    double4 f = S.force[k];
    f.x += f_p.x; f.y += f_p.y; f.z += f_p.z; f.w += 0.0;
    S.force[k] = f;
    f_p_out[S.orig_of[k]] = make_double4(f_p.x, f_p.y, f_p.z, 0.0);
}

// findDarcyPorositiesLinear, darcy.cuh:359-550
__global__ void k_porosities(DevParams P, DevState S, DarcyParams D, double *phi_a, double *dphi_a,
                             double *vp_avg)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    const unsigned cellidx = didx(D, x, y, z);
    if (P.np == 0) {
        phi_a[cellidx] = 0.9;
        dphi_a[cellidx] = 0.0;
        return;
    }
    const long long iter = S.ctl->iter;
    const double dx = D.dx, dy = D.dy, dz = D.dz;
    const V3 X = mk3(x * dx + 0.5 * dx, y * dy + 0.5 * dy, z * dz + 0.5 * dz);
    double solid = 0.0, solid_new = 0.0, den = 0.0;
    V3 num = mk3(0.0, 0.0, 0.0);
    const double phi_0 = phi_a[cellidx];
    for (int dzc = -1; dzc < 2; ++dzc)
        for (int dyc = -1; dyc < 2; ++dyc)
            for (int dxc = -1; dxc < 2; ++dxc) {
                int cx = x + dxc, cy = y + dyc, cz = z + dzc, sx, sy;
                if (cz == -1) cz = 1;
                if (P.periodic == 2) {
                    if (cy == -1) cy = 1;
                    if (cy == (int)P.num[1]) cy = (int)P.num[1] - 2;
                }
                if (!wrap_cell(P, cx, cy, cz, sx, sy)) continue;
                V3 dm = shift_vec(P, sx, sy);
                unsigned cell = (unsigned)cx + (unsigned)cy * P.num[0] +
                                (P.num[0] * P.num[1]) * (unsigned)cz;
                unsigned start = S.cell_start[cell];
                if (start == 0xffffffffu) continue;
                unsigned end = S.cell_end[cell];
                for (unsigned i = start; i < end; ++i) {
                    double4 xr = S.x[i], v = S.vel[i];
                    V3 dist = add3(mk3(X.x - xr.x, X.y - xr.y, X.z - xr.z), dm);
                    double sw = weight_dist(dist, dx, dy, dz);
                    double vol_p = sphere_volume(xr.w);
                    solid += sw * vol_p;
                    double sv = sw * vol_p;
                    num = add3(num, mk3(sv * v.x, sv * v.y, sv * v.z));
                    den += sw * vol_p;
                    xr.x += v.x * P.dt; xr.y += v.y * P.dt; xr.z += v.z * P.dt;
                    V3 d2 = add3(mk3(X.x - xr.x, X.y - xr.y, X.z - xr.z), dm);
                    solid_new += weight_dist(d2, dx, dy, dz) * vol_p;
                }
            }
    double cell_volume = dx * dy * dz;
    if (z == D.nz - 1) cell_volume *= 0.875;
    const double phi = fmin(0.9, fmax(0.1, 1.0 - solid / cell_volume));
    const double phi_new = fmin(0.9, fmax(0.1, 1.0 - solid_new / cell_volume));
    double dphi;
    V3 vp = mk3(0.0, 0.0, 0.0);
    if (iter == 0) {
        dphi = 0.0;
    } else {
        dphi = 0.5 * (phi_new - phi_0);
        vp = divs3(num, fmax(1.0e-16, den));
    }
    phi_a[cellidx] = phi * D.c_phi;
    dphi_a[cellidx] = dphi * D.c_phi;
    vp_avg[3 * (size_t)cellidx] = vp.x;
    vp_avg[3 * (size_t)cellidx + 1] = vp.y;
    vp_avg[3 * (size_t)cellidx + 2] = vp.z;
}

// copyDarcyPorositiesToEdges + ToBottom, darcy.cuh:556-628 (periodic == 2)
__global__ void k_copy_edges(DarcyParams D, double *phi, double *dphi, double *div_v_p, double *vp)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    if (y == 0 || y == D.ny - 1) {
        int yr = y == 0 ? 1 : D.ny - 2;
        unsigned r = didx(D, x, yr, z), w = didx(D, x, y, z);
        phi[w] = phi[r]; dphi[w] = dphi[r]; div_v_p[w] = div_v_p[r];
        for (int c = 0; c < 3; ++c) vp[3 * (size_t)w + c] = vp[3 * (size_t)r + c];
    }
}

__global__ void k_copy_bottom(DarcyParams D, double *phi, double *dphi, double *div_v_p, double *vp)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z) || z != 0) return;
    unsigned r = didx(D, x, y, 1), w = didx(D, x, y, 0);
    phi[w] = phi[r]; dphi[w] = dphi[r]; div_v_p[w] = div_v_p[r];
    for (int c = 0; c < 3; ++c) vp[3 * (size_t)w + c] = vp[3 * (size_t)r + c];
}

// setDarcyTopPressure + setDarcyTopWallPressure (darcy.cuh:1195-1240) for
// cells inside the grid
__global__ void k_top_pressure(DarcyParams D, const DarcyCtl *dctl, double *p, double t)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    double np_ = D.p_top_orig + D.p_mod_A * sin(2.0 * 3.14159265358979323846 * D.p_mod_f * t + D.p_mod_phi);
    if (z == D.nz - 1 || (unsigned)z == dctl->wall0_iz) p[didx(D, x, y, z)] = np_;
    if (z == D.nz - 1 && dctl->wall0_iz == (unsigned)D.nz) p[didx(D, x, y, D.nz)] = np_;
}

// findDarcyPermeabilities, darcy.cuh:1266-1313
__global__ void k_permeabilities(DarcyParams D, const double *phi, double *k)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    unsigned c = didx(D, x, y, z);
    double ph = phi[c];
    if (ph > 0.9999) ph = 0.9999;
    double kk = D.k_c * pow(ph, 3.0) / pow(1.0 - ph, 2.0);
    k[c] = fmin(2.7e-10, kk);
}

// findDarcyPermeabilityGradients, darcy.cuh:1316-1374
__global__ void k_permeability_gradients(DarcyParams D, const double *k, double *grad_k)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    double *g = &grad_k[3 * (size_t)didx(D, x, y, z)];
    g[0] = (k[didx(D, x + 1, y, z)] - k[didx(D, x - 1, y, z)]) / (D.dx + D.dx);
    g[1] = (k[didx(D, x, y + 1, z)] - k[didx(D, x, y - 1, z)]) / (D.dy + D.dy);
    g[2] = (k[didx(D, x, y, z + 1)] - k[didx(D, x, y, z - 1)]) / (D.dz + D.dz);
}

struct DarcyFields {
    const double *phi, *dphi, *k, *vp_avg, *p_old, *dp_expl;
    const int *p_constant;
};

// The pressure change of firstDarcySolution / updateDarcySolution
// (darcy.cuh:1425-1598, 1602-1799) from the pressure field pf.
__device__ __forceinline__ double dp_of(const DarcyParams &D, const DarcyFields &F, const double *pf,
                                        unsigned wall0_iz, double dt, int x, int y, int z)
{
    const int nx = D.nx, ny = D.ny, nz = D.nz;
    const double dx = D.dx, dy = D.dy, dz = D.dz;
    const unsigned c = didx(D, x, y, z);
    const double phi_xn = F.phi[didx(D, x - 1, y, z)], phi = F.phi[c];
    const double phi_xp = F.phi[didx(D, x + 1, y, z)], phi_yn = F.phi[didx(D, x, y - 1, z)];
    const double phi_yp = F.phi[didx(D, x, y + 1, z)], phi_zn = F.phi[didx(D, x, y, z - 1)];
    const double phi_zp = F.phi[didx(D, x, y, z + 1)];
    const double dphi = F.dphi[c];
    const double *vp = &F.vp_avg[3 * (size_t)c];
    const int p_constant = F.p_constant[c];
    double p_xn = pf[didx(D, x - 1, y, z)];
    const double p = pf[c];
    double p_xp = pf[didx(D, x + 1, y, z)], p_yn = pf[didx(D, x, y - 1, z)];
    double p_yp = pf[didx(D, x, y + 1, z)], p_zn = pf[didx(D, x, y, z - 1)];
    double p_zp = pf[didx(D, x, y, z + 1)];
    const double k_xn = F.k[didx(D, x - 1, y, z)], k = F.k[c], k_xp = F.k[didx(D, x + 1, y, z)];
    const double k_yn = F.k[didx(D, x, y - 1, z)], k_yp = F.k[didx(D, x, y + 1, z)];
    const double k_zn = F.k[didx(D, x, y, z - 1)], k_zp = F.k[didx(D, x, y, z + 1)];
    if (x == 0 && D.bc_xn == 1) p_xn = p;
    if (x == nx - 1 && D.bc_xp == 1) p_xp = p;
    if (y == 0 && D.bc_yn == 1) p_yn = p;
    if (y == ny - 1 && D.bc_yp == 1) p_yp = p;
    if (z == 0 && D.bc_bot == 1) p_zn = p;
    if (z == nz - 1 && D.bc_top == 1) p_zp = p;
    const double gx = (phi_xp - phi_xn) / (dx + dx), gy = (phi_yp - phi_yn) / (dy + dy),
                 gz = (phi_zp - phi_zn) / (dz + dz);
    const double div_k_grad_p =
        (2. * k_xp * k / (k_xp + k) * (p_xp - p) / dx - 2. * k_xn * k / (k_xn + k) * (p - p_xn) / dx) / dx +
        (2. * k_yp * k / (k_yp + k) * (p_yp - p) / dy - 2. * k_yn * k / (k_yn + k) * (p - p_yn) / dy) / dy +
        (2. * k_zp * k / (k_zp + k) * (p_zp - p) / dz - 2. * k_zn * k / (k_zn + k) * (p - p_zn) / dz) / dz;
    const double ndt = D.ndem * dt;
    double dp = ndt / (D.beta_f * phi * D.mu) * div_k_grad_p -
                (ndt / (D.beta_f * phi * (1.0 - phi))) *
                    (dphi / ndt + (vp[0] * gx + vp[1] * gy + vp[2] * gz));
    if ((D.bc_bot == 0 && z == 0) || (D.bc_top == 0 && z == nz - 1) ||
        ((unsigned)z >= wall0_iz && D.bc_top == 0) || (D.bc_xn == 0 && x == 0) ||
        (D.bc_xp == 0 && x == nx - 1) || (D.bc_yn == 0 && y == 0) ||
        (D.bc_yp == 0 && y == nx - 1) || p_constant == 1)
        dp = 0.0;
    return dp;
}

// firstDarcySolution: dp_expl from the current pressure
__global__ void k_first_solution(DarcyParams D, DarcyFields F, const double *p, double *dp_expl,
                                 const DarcyCtl *dctl, double dt)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    dp_expl[didx(D, x, y, z)] = dp_of(D, F, p, dctl->wall0_iz, dt, x, y, z);
}

// The iterate-independent parts of dp_of for every interior cell
// (darcy.cuh:1602-1799), written for k_jacobi.
__global__ void k_jacobi_coef(DarcyParams D, DarcyFields F, const DarcyCtl *dctl, double dt,
                              double *cf, double *ca, double *csrc, double *cbase,
                              unsigned char *cfixed, unsigned long long ng)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    const int nx = D.nx, ny = D.ny, nz = D.nz;
    const double dx = D.dx, dy = D.dy, dz = D.dz;
    const unsigned c = didx(D, x, y, z);
    const unsigned wall0_iz = dctl->wall0_iz;
    const double phi_xn = F.phi[didx(D, x - 1, y, z)], phi = F.phi[c];
    const double phi_xp = F.phi[didx(D, x + 1, y, z)], phi_yn = F.phi[didx(D, x, y - 1, z)];
    const double phi_yp = F.phi[didx(D, x, y + 1, z)], phi_zn = F.phi[didx(D, x, y, z - 1)];
    const double phi_zp = F.phi[didx(D, x, y, z + 1)];
    const double dphi = F.dphi[c];
    const double *vp = &F.vp_avg[3 * (size_t)c];
    const double k_xn = F.k[didx(D, x - 1, y, z)], k = F.k[c], k_xp = F.k[didx(D, x + 1, y, z)];
    const double k_yn = F.k[didx(D, x, y - 1, z)], k_yp = F.k[didx(D, x, y + 1, z)];
    const double k_zn = F.k[didx(D, x, y, z - 1)], k_zp = F.k[didx(D, x, y, z + 1)];
    const double gx = (phi_xp - phi_xn) / (dx + dx), gy = (phi_yp - phi_yn) / (dy + dy),
                 gz = (phi_zp - phi_zn) / (dz + dz);
    cf[c] = 2. * k_xp * k / (k_xp + k);
    cf[ng + c] = 2. * k_xn * k / (k_xn + k);
    cf[2 * ng + c] = 2. * k_yp * k / (k_yp + k);
    cf[3 * ng + c] = 2. * k_yn * k / (k_yn + k);
    cf[4 * ng + c] = 2. * k_zp * k / (k_zp + k);
    cf[5 * ng + c] = 2. * k_zn * k / (k_zn + k);
    const double ndt = D.ndem * dt;
    ca[c] = ndt / (D.beta_f * phi * D.mu);
    csrc[c] = (ndt / (D.beta_f * phi * (1.0 - phi))) * (dphi / ndt + (vp[0] * gx + vp[1] * gy + vp[2] * gz));
    const double epsilon = 0.5;
    cbase[c] = F.p_old[c] + (1.0 - epsilon) * F.dp_expl[c];
    cfixed[c] = ((D.bc_bot == 0 && z == 0) || (D.bc_top == 0 && z == nz - 1) ||
                 ((unsigned)z >= wall0_iz && D.bc_top == 0) || (D.bc_xn == 0 && x == 0) ||
                 (D.bc_xp == 0 && x == nx - 1) || (D.bc_yn == 0 && y == 0) ||
                 (D.bc_yp == 0 && y == nx - 1) || F.p_constant[c] == 1) ? 1 : 0;
    (void)ny;
}

// dp_of from the per-solve constants: the same operations in the same
// order on the same values.
__device__ __forceinline__ double dp_fast(const DarcyParams &D, const JacobiCoef &C, const double *pf,
                                          unsigned c, int x, int y, int z)
{
    if (C.fixed[c]) return 0.0;
    const unsigned sx = (unsigned)D.nx + 2u, sxy = sx * ((unsigned)D.ny + 2u);
    const double dx = D.dx, dy = D.dy, dz = D.dz;
    const double p = pf[c];
    double p_xn = pf[c - 1], p_xp = pf[c + 1], p_yn = pf[c - sx], p_yp = pf[c + sx];
    double p_zn = pf[c - sxy], p_zp = pf[c + sxy];
    if (x == 0 && D.bc_xn == 1) p_xn = p;
    if (x == D.nx - 1 && D.bc_xp == 1) p_xp = p;
    if (y == 0 && D.bc_yn == 1) p_yn = p;
    if (y == D.ny - 1 && D.bc_yp == 1) p_yp = p;
    if (z == 0 && D.bc_bot == 1) p_zn = p;
    if (z == D.nz - 1 && D.bc_top == 1) p_zp = p;
    const size_t ng = C.ng;
    const double div_k_grad_p =
        (C.cf[c] * (p_xp - p) / dx - C.cf[ng + c] * (p - p_xn) / dx) / dx +
        (C.cf[2 * ng + c] * (p_yp - p) / dy - C.cf[3 * ng + c] * (p - p_yn) / dy) / dy +
        (C.cf[4 * ng + c] * (p_zp - p) / dz - C.cf[5 * ng + c] * (p - p_zn) / dz) / dz;
    return C.a[c] * div_k_grad_p - C.src[c];
}

// Bounded wait of thread 0 until *p >= target; false (and DERR_TIMEOUT in
// the engine's error flag) after ~2^22 polls, or as soon as another block
// has flagged an error.  With `inject` the wait never succeeds and gives up
// after kInjectPolls polls.
__device__ __forceinline__ bool jacobi_wait_ge(const unsigned *p, unsigned target, DarcyCtl *ctl,
                                               unsigned inject)
{
    unsigned spins = 0, nap = 16;
    const unsigned limit = inject ? kInjectPolls : (1u << 22);
    for (;;) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        if (v >= target && !inject) return true;
        if (++spins > limit) {
            atomicCAS(&ctl->err, 0, DERR_TIMEOUT);
            return false;
        }
        if (*(volatile int *)&ctl->err != 0) return false;
        __nanosleep(nap);
        if (nap < 128) nap <<= 1;
    }
}

__device__ __forceinline__ bool jacobi_is_check(unsigned it, unsigned maxiter, int exact_stop)
{
    return exact_stop || it % 10u == 0u || it + 1u == maxiter;
}

// The Jacobi iterations of the reference (device.cu:2184-2386):
// p_new = p_old + 0.5 dp_expl + 0.5 dp_impl(p); p_new <- 0.95 p + 0.05 p_new;
// residual (p_new - p)/(p + 1e-16); stop when the maximum |residual| is at
// most the tolerance at an iteration divisible by 10 (every iteration with
// exact_stop).
//
// Block b updates the cells [b*chunk, (b+1)*chunk).  Before iteration i it
// waits until the blocks whose cells lie within reach (one z layer, one row
// and one cell: the stencil and the periodic ghost faces the cells write)
// have completed iteration i-1, which makes their part of iterate i-1
// visible and frees the buffer iteration i overwrites.  The stop decision of
// a check iteration c needs every block's residual; it is taken at the start
// of iteration c+2, so iteration c+1 is computed while the last blocks
// arrive (iteration c+1 writes the other buffer: iterate c stays intact and
// is the result if the solve stops at c).
__global__ void __launch_bounds__(256) k_jacobi(DarcyParams D, DarcyFields F, JacobiCoef C, double *pa,
                                                double *pb, DarcyCtl *ctl, JacobiSync *js, int exact_stop)
{
    __shared__ double wmax[8];
    __shared__ int s_state;          // 0 continue, 1 stop, 2 abort
    __shared__ long long s_final;    // iterate the solve ends with
    __shared__ long long s_conv_at;
    const unsigned G = gridDim.x, b = blockIdx.x;
    const unsigned n = (unsigned)D.nx * D.ny * D.nz;
    const unsigned maxiter = D.maxiter;
    const unsigned chunk = (n + G - 1) / G;
    const unsigned lo = min(n, b * chunk), hi = min(n, lo + chunk);
    const unsigned reach = (unsigned)D.nx * D.ny + (unsigned)D.nx + 1u;
    const unsigned nb_lo = lo > reach ? (lo - reach) / chunk : 0u;
    const unsigned nb_hi = min(G - 1u, (hi + reach) / chunk);
    // thread 0's view of the decisions
    unsigned next_dec = 0, dec_count = 0, scanned = 0;
    if (threadIdx.x == 0) {
        s_state = 0;
        s_final = -1;
        s_conv_at = -1;
    }
    __syncthreads();

    // Decides check iteration c (thread 0): waits for every block's arrival,
    // scans the residual maxima up to c, sets s_state / s_final.
    auto decide = [&](unsigned c) {
        const unsigned k = dec_count;
        // acquire: every block's residual (ordered before its release-add)
        if (!jacobi_wait_ge(&js->arrive[k % kJacobiChecks][0], G, ctl, D.inject)) {
            s_state = 2;
            return;
        }
        bool nan = false;
        double mc = 0.0;
        for (unsigned j = scanned; j <= c; ++j) {
            const unsigned long long bits = __ldcg(&js->ring[j % kJacobiRing]);
            if (bits == ~0ull) { nan = true; break; }
            const double m = __longlong_as_double((long long)bits);
            if (m <= D.tolerance && s_conv_at < 0) s_conv_at = j;
            if (j == c) mc = m;
        }
        scanned = c + 1;
        // every block has waited on the counter of the check decided two
        // decisions ago (it arrived here after deciding it)
        if (b == 0 && k >= 2) js->arrive[(k - 2) % kJacobiChecks][0] = 0u;
        if (nan) {
            atomicCAS(&ctl->err, 0, DERR_NAN);
            s_state = 2;
            s_final = c;
        } else if (mc <= D.tolerance && (exact_stop || c % 10u == 0u)) {
            s_state = 1;
            s_final = c;
        }
        ++dec_count;
        // the next check iteration
        unsigned nx = c + 1;
        while (nx < maxiter && !jacobi_is_check(nx, maxiter, exact_stop)) ++nx;
        next_dec = nx;
    };

    unsigned it = 0;
    for (; it < maxiter; ++it) {
        if (threadIdx.x < 32) {
            if (threadIdx.x == 0)
                while (s_state == 0 && next_dec < maxiter && next_dec + 2u <= it) decide(next_dec);
            __syncwarp();
            if (s_state == 0 && it > 0) {
                // the lanes of warp 0 watch the neighbours in parallel
                bool ok = true;
                for (unsigned q = nb_lo + threadIdx.x; q <= nb_hi; q += 32)
                    if (q != b && !jacobi_wait_ge(&js->done[q][0], it, ctl, D.inject)) ok = false;
                if (!__all_sync(0xffffffffu, ok) && threadIdx.x == 0) s_state = 2;
            }
        }
        // the acquire loads above and this barrier make the neighbours'
        // cells visible to the whole block
        __syncthreads();
        if (s_state != 0) break;
        const bool even = (it & 1u) == 0u;
        const double *cur = even ? pa : pb;
        double *nxt = even ? pb : pa;
        double lmax = 0.0;
        bool nan = false;
        for (unsigned i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const int x = (int)(i % D.nx), y = (int)((i / D.nx) % D.ny),
                      z = (int)(i / ((unsigned)D.nx * D.ny));
            const unsigned c = didx(D, x, y, z);
            const double dp_impl = dp_fast(D, C, cur, c, x, y, z);
            const double epsilon = 0.5, theta = 0.05;
            const double p = cur[c];
            double p_new = C.base[c] + epsilon * dp_impl;
            p_new = p * (1.0 - theta) + p_new * theta;
            const double res = (p_new - p) / (p + 1.0e-16);
            const double a = fabs(res);
            if (a != a) nan = true;
            else lmax = fmax(lmax, a);
            nxt[c] = p_new;
            // ghost faces of the next iterate that this cell determines
            // (setDarcyGhostNodes at the start of the next iteration), and
            // the flux ghosts, which the reference derives from the
            // pressure before the copy
            ghost_from<1>(D, nxt, x, y, z, &p_new);
            if (D.bc_bot == 4 || D.bc_top == 4) flux_ghost_next(D, F.k, nxt, x, y, z, p);
        }
        // block maximum, one atomic per block into this iteration's slot
        for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
        if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = lmax;
        // the barrier orders every thread's cell stores before thread 0's
        // release (cumulative at GPU scope), so the neighbours may go on
        const bool any_nan = __syncthreads_or(nan);
        if (threadIdx.x == 0) {
            asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(&js->done[b][0]), "r"(it + 1u) : "memory");
            double bm = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) bm = fmax(bm, wmax[w]);
            unsigned long long *slot = &js->ring[it % kJacobiRing];
            if (any_nan) atomicExch(slot, ~0ull);
            else atomicMax(slot, (unsigned long long)__double_as_longlong(bm));
            // the slot of iteration it + kJacobiRing / 2 was last used by
            // iteration it - kJacobiRing / 2, scanned by every block long ago
            if (b == 0) js->ring[(it + kJacobiRing / 2) % kJacobiRing] = 0ull;
            if (jacobi_is_check(it, maxiter, exact_stop)) {
                // index of this check among the checks: iterations 0, 10,
                // 20, ... (every iteration with exact_stop), plus maxiter - 1;
                // the release orders the residual above before the arrival
                const unsigned k = exact_stop ? it : it / 10u + ((it % 10u) ? 1u : 0u);
                asm volatile("red.release.gpu.global.add.u32 [%0], 1;"
                             :: "l"(&js->arrive[k % kJacobiChecks][0]) : "memory");
            }
        }
    }
    // decide the checks still open (the last one or two iterations)
    if (threadIdx.x == 0) {
        while (s_state == 0 && next_dec < it) decide(next_dec);
    }
    __syncthreads();
    if (b == 0 && threadIdx.x == 0) {
        if (s_state == 2 && s_final < 0) return;      // timeout: ctl->err is set
        long long fin = s_final >= 0 ? s_final : (maxiter > 0 ? (long long)maxiter - 1 : 0);
        ctl->nijac_last = fin;
        ctl->nijac_total += fin + 1;
        ctl->converged_at = s_conv_at;
        ctl->converged = s_state == 1 ? 1 : 0;
        ctl->final_buf = maxiter == 0 ? 0 : ((fin & 1) == 0 ? 1 : 0);
    }
}

// Cells whose pressure the solve may change: dp_of's zeroing conditions
// (Dirichlet faces, cells at or above the top wall, fixed-pressure cells)
// are false.
__global__ void k_free_cells(DarcyParams D, const DarcyCtl *ctl, const int *p_constant,
                             unsigned char *freec)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    const unsigned wall0_iz = ctl->wall0_iz;
    const bool fixed = (D.bc_bot == 0 && z == 0) || (D.bc_top == 0 && z == D.nz - 1) ||
                       ((unsigned)z >= wall0_iz && D.bc_top == 0) || (D.bc_xn == 0 && x == 0) ||
                       (D.bc_xp == 0 && x == D.nx - 1) || (D.bc_yn == 0 && y == 0) ||
                       (D.bc_yp == 0 && y == D.nx - 1) || p_constant[didx(D, x, y, z)] == 1;
    freec[(size_t)(z * D.ny + y) * D.nx + x] = fixed ? 0 : 1;
}

// max |residual| of the first Jacobi iteration started from pg
__global__ void k_guess_residual(DarcyParams D, DarcyFields F, const double *pg, DarcyCtl *ctl,
                                 double dt, int slot)
{
    int x, y, z;
    double a = 0.0;
    if (cell_of_thread(D, x, y, z)) {
        const unsigned c = didx(D, x, y, z);
        const double dp_impl = dp_of(D, F, pg, ctl->wall0_iz, dt, x, y, z);
        const double p = pg[c];
        double p_new = F.p_old[c] + 0.5 * F.dp_expl[c] + 0.5 * dp_impl;
        p_new = p * 0.95 + p_new * 0.05;
        a = fabs((p_new - p) / (p + 1.0e-16));
        if (a != a) a = 1.0e300;
    }
    for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(&ctl->guess_res[slot], (unsigned long long)__double_as_longlong(a));
}

// The solve starts from the candidate with the smallest first residual:
// the previous solution (slot 0, kept on ties), the guess (slot 1) or the
// extrapolation alone (slot 2, when guess_base is given).
__global__ void k_take_guess(DarcyCtl *ctl, double *p, const double *guess, const double *guess_base,
                             size_t ng)
{
    int pick = 0;
    unsigned long long best = ctl->guess_res[0];
    if (ctl->guess_res[1] < best) { pick = 1; best = ctl->guess_res[1]; }
    if (guess_base && ctl->guess_res[2] < best) pick = 2;
    if (pick == 0) return;
    const double *src = pick == 1 ? guess : guess_base;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < ng;
         i += (size_t)gridDim.x * blockDim.x)
        p[i] = src[i];
    if (blockIdx.x == 0 && threadIdx.x == 0 && pick == 1) ctl->ws_picked += 1;
}

__global__ void k_clear_guess_res(DarcyCtl *ctl)
{
    ctl->guess_res[0] = 0ull;
    ctl->guess_res[1] = 0ull;
    ctl->guess_res[2] = 0ull;
}

// findDarcyVelocities, darcy.cuh:1839-1897
__global__ void k_velocities(DarcyParams D, const double *p, const double *phi, const double *k,
                             double *v)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    unsigned c = didx(D, x, y, z);
    double gx = (p[didx(D, x + 1, y, z)] - p[didx(D, x - 1, y, z)]) / (D.dx + D.dx);
    double gy = (p[didx(D, x, y + 1, z)] - p[didx(D, x, y - 1, z)]) / (D.dy + D.dy);
    double gz = (p[didx(D, x, y, z + 1)] - p[didx(D, x, y, z - 1)]) / (D.dz + D.dz);
    double a = -k[c] / D.mu;
    v[3 * (size_t)c] = (a * gx) / phi[c];
    v[3 * (size_t)c + 1] = (a * gy) / phi[c];
    v[3 * (size_t)c + 2] = (a * gz) / phi[c];
}

// Gathers interior cells (x fastest) of a padded field into dst.
__global__ void k_gather_interior(DarcyParams D, const double *src, double *dst, int comps)
{
    int x, y, z;
    if (!cell_of_thread(D, x, y, z)) return;
    size_t o = ((size_t)(z * D.ny + y) * D.nx + x) * comps;
    for (int c = 0; c < comps; ++c) dst[o + c] = src[(size_t)didx(D, x, y, z) * comps + c];
}

// Copies the buffer holding the final pressure into p when it is the other one.
__global__ void k_final_pressure(DarcyParams D, const DarcyCtl *ctl, double *p, const double *p2,
                                 size_t ng)
{
    if (ctl->final_buf != 1) return;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < ng;
         i += (size_t)gridDim.x * blockDim.x)
        p[i] = p2[i];
}

// ---------------------------------------------------------------------
// engine glue
// ---------------------------------------------------------------------
static unsigned cells_blocks(const DarcyParams &D) { return ((unsigned)D.nx * D.ny * D.nz + 255) / 256; }

int Engine::darcy_init()
{
    if (!hs.fluid) return ST_OK;
    if (hs.cfd_solver == 0) return ns_init();
    if (hs.ndem == 0) return fail(ST_INPUT, "ndem must be positive");
    darcy = new DarcyDev();
    DarcyDev &Dd = *darcy;
    DarcyParams &D = Dd.D;
    D.nx = (int)hs.num[0]; D.ny = (int)hs.num[1]; D.nz = (int)hs.num[2];
    D.dx = hs.L[0] / hs.num[0]; D.dy = hs.L[1] / hs.num[1]; D.dz = hs.L[2] / hs.num[2];
    D.mu = hs.mu; D.rho_f = hs.rho_f; D.beta_f = hs.beta_f; D.k_c = hs.k_c; D.c_phi = hs.c_phi;
    D.tolerance = hs.tolerance;
    D.p_mod_A = hs.p_mod_A; D.p_mod_f = hs.p_mod_f; D.p_mod_phi = hs.p_mod_phi;
    D.bc_bot_flux = hs.bc_bot_flux; D.bc_top_flux = hs.bc_top_flux;
    D.bc_xn = hs.bc_xn; D.bc_xp = hs.bc_xp; D.bc_yn = hs.bc_yn; D.bc_yp = hs.bc_yp;
    D.bc_bot = hs.bc_bot; D.bc_top = hs.bc_top;
    D.maxiter = hs.maxiter; D.ndem = hs.ndem;
    D.inject = (inject & kInjectDarcy) ? 1u : 0u;
    const size_t nx = D.nx, ny = D.ny, nz = D.nz;
    const size_t ng = (nx + 2) * (ny + 2) * (nz + 2);
    Dd.ng = ng;
    auto didx_h = [&](size_t x, size_t y, size_t z) { return (x + 1) + (nx + 2) * (y + 1) + (nx + 2) * (ny + 2) * (z + 1); };
    // device.cu:1017-1020
    D.p_top_orig = hs.p_f[(nz - 1) * nx * ny] -
                   hs.p_mod_A * sin(2.0 * 3.14159265358979323846 * hs.p_mod_f * hs.t_current + hs.p_mod_phi);
    Dd.p = dalloc<double>(ng); Dd.p2 = dalloc<double>(ng); Dd.p_old = dalloc<double>(ng);
    Dd.dp_expl = dalloc<double>(ng); Dd.phi = dalloc<double>(ng); Dd.dphi = dalloc<double>(ng);
    Dd.k = dalloc<double>(ng); Dd.div_v_p = dalloc<double>(ng);
    Dd.v = dalloc<double>(3 * ng); Dd.vp_avg = dalloc<double>(3 * ng);
    Dd.grad_p = dalloc<double>(3 * ng); Dd.grad_k = dalloc<double>(3 * ng);
    Dd.p_constant = dalloc<int>(ng);
    Dd.f_p = dalloc<double4>(hs.np);
    Dd.gather = dalloc<double>(3 * nx * ny * nz);
    Dd.ctl = dalloc<DarcyCtl>(1);
    Dd.jsync = dalloc<JacobiSync>(1);
    Dd.cf = dalloc<double>(6 * ng); Dd.ca = dalloc<double>(ng); Dd.csrc = dalloc<double>(ng);
    Dd.cbase = dalloc<double>(ng); Dd.cfixed = dalloc<unsigned char>(ng);
    if (!Dd.p || !Dd.p2 || !Dd.p_old || !Dd.dp_expl || !Dd.phi || !Dd.dphi || !Dd.k ||
        !Dd.div_v_p || !Dd.v || !Dd.vp_avg || !Dd.grad_p || !Dd.grad_k || !Dd.p_constant ||
        !Dd.f_p || !Dd.gather || !Dd.ctl || !Dd.jsync || !Dd.cf || !Dd.ca || !Dd.csrc ||
        !Dd.cbase || !Dd.cfixed) return fail(ST_CUDA, "device allocation failed (Darcy)");
    std::vector<double> p(ng, 0.0), phi(ng, 0.0), dphi(ng, 0.0), v(3 * ng, 0.0);
    std::vector<int> pc(ng, 0);
    for (size_t z = 0; z < nz; ++z)
        for (size_t y = 0; y < ny; ++y)
            for (size_t x = 0; x < nx; ++x) {
                size_t f = (z * ny + y) * nx + x, g = didx_h(x, y, z);
                p[g] = hs.p_f[f]; phi[g] = hs.phi[f]; dphi[g] = hs.dphi[f];
                pc[g] = hs.p_constant[f];
                for (int c = 0; c < 3; ++c) v[3 * g + c] = hs.v_f[3 * f + c];
            }
    std::vector<double4> fp(hs.np);
    for (uint32_t i = 0; i < hs.np; ++i) fp[i] = make_double4(hs.f_p[i].x, hs.f_p[i].y, hs.f_p[i].z, 0.0);
    cudaMemcpyAsync(Dd.p, p.data(), ng * 8, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(Dd.phi, phi.data(), ng * 8, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(Dd.dphi, dphi.data(), ng * 8, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(Dd.v, v.data(), 3 * ng * 8, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(Dd.p_constant, pc.data(), ng * 4, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(Dd.f_p, fp.data(), hs.np * 32, cudaMemcpyHostToDevice, stream);
    DarcyCtl c;
    std::memset(&c, 0, sizeof c);
    c.wall0_iz = 10000000u;
    cudaMemcpyAsync(Dd.ctl, &c, sizeof c, cudaMemcpyHostToDevice, stream);
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "Darcy upload");
    Dd.host_wall0_w = hs.nw > 0 ? hs.wnx[0].w : 0.0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jacobi, 256, 0);
    if (per_sm < 1) return fail(ST_CUDA, "Jacobi kernel cannot be resident");
    // resident blocks per SM of the Jacobi launch (four by default: about
    // one cell per thread on the 40 x 40 x 80 benchmark grid, measured
    // fastest among 1..4; the variable SPHB_JACOBI_BLOCKS_PER_SM overrides
    // it for tuning runs)
    int bps = 4;
    if (const char *env = std::getenv("SPHB_JACOBI_BLOCKS_PER_SM")) bps = std::max(1, std::atoi(env));
    jacobi_grid = sms * (per_sm < bps ? per_sm : bps);
    unsigned need = cells_blocks(D);
    if ((unsigned)jacobi_grid > need) jacobi_grid = (int)need;
    if ((unsigned)jacobi_grid > kJacobiMaxBlocks) jacobi_grid = (int)kJacobiMaxBlocks;
    if (warm_start) {
        Dd.freec = dalloc<unsigned char>(nx * ny * nz);
        Dd.guess = dalloc<double>(ng);
        if (warm_start == 1) Dd.guess_base = dalloc<double>(ng);
        Dd.ws = ws_create(D.nx, D.ny, D.nz, 0x5eed5eedull, warm_start_train, warm_start == 1);
        if (!Dd.ws || !Dd.freec || !Dd.guess)
            return fail(ST_CUDA, "could not set up the learned warm start");
    }
    return darcy_sync_wall();
}

// wall0_iz comes from the host's copy of wall 0, refreshed at file output
// (device.cu:1908-1911 reads walls.nx->w on the host); it keeps its initial
// value unless wall 0 moves under wmode 1 or 3.
int Engine::darcy_sync_wall()
{
    if (!darcy) return ST_OK;
    if (hs.nw > 0 && (hs.wmode[0] == 1 || hs.wmode[0] == 3))
        darcy_wall0_iz = (unsigned)(darcy->host_wall0_w / (hs.L[2] / hs.num[2]));
    cudaError_t e = cudaMemcpyAsync(&darcy->ctl->wall0_iz, &darcy_wall0_iz, 4, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e == cudaSuccess ? ST_OK : cuda_fail(e, "Darcy wall");
}

void Engine::darcy_set_host_wall()
{
    if (darcy) darcy->host_wall0_w = hs.nw > 0 ? hs.wnx[0].w : 0.0;
}

void Engine::darcy_free()
{
    if (darcy && darcy->ws) ws_destroy(darcy->ws);
    delete darcy;   // device arrays are released with the engine's allocations
    darcy = nullptr;
}

cudaError_t Engine::enqueue_fluid()
{
    if (ns) return enqueue_ns();
    if (!darcy) return cudaSuccess;
    DarcyDev &Dd = *darcy;
    const DarcyParams &D = Dd.D;
    const unsigned cb = cells_blocks(D);
    cudaError_t e;
    if (hs.np > 0) {
        k_ghost<1><<<cb, 256, 0, stream>>>(D, Dd.p);
        k_pressure_gradient<<<cb, 256, 0, stream>>>(D, Dd.p, Dd.grad_p);
        k_ghost<3><<<cb, 256, 0, stream>>>(D, Dd.grad_p);
        k_pressure_force<<<(hs.np + 127) / 128, 128, 0, stream>>>(P, S, D, Dd.grad_p, Dd.ctl, Dd.f_p);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // iter % ndem == 0, decided from the host's mirror of the step counter
    if ((host_iter % (int64_t)D.ndem) != 0) return cudaSuccess;
    k_porosities<<<cb, 256, 0, stream>>>(P, S, D, Dd.phi, Dd.dphi, Dd.vp_avg);
    if (hs.periodic == 2) {
        k_copy_edges<<<cb, 256, 0, stream>>>(D, Dd.phi, Dd.dphi, Dd.div_v_p, Dd.vp_avg);
        k_copy_bottom<<<cb, 256, 0, stream>>>(D, Dd.phi, Dd.dphi, Dd.div_v_p, Dd.vp_avg);
    }
    if ((D.p_mod_A > 1.0e-5 || D.p_mod_A < -1.0e-5) && D.p_mod_f > 1.0e-7)
        k_top_pressure<<<cb, 256, 0, stream>>>(D, Dd.ctl, Dd.p, host_t);
    k_permeabilities<<<cb, 256, 0, stream>>>(D, Dd.phi, Dd.k);
    k_ghost<1><<<cb, 256, 0, stream>>>(D, Dd.phi);
    k_ghost<1><<<cb, 256, 0, stream>>>(D, Dd.k);
    k_permeability_gradients<<<cb, 256, 0, stream>>>(D, Dd.k, Dd.grad_k);
    const bool flux = D.bc_bot == 4 || D.bc_top == 4;
    if (flux) k_flux_ghost<<<cb, 256, 0, stream>>>(D, Dd.p, Dd.k);
    // nijac == 0: p -> p_old, ghosts, dp_expl
    k_copy_interior<<<cb, 256, 0, stream>>>(D, Dd.p, Dd.p_old);
    k_ghost<1><<<cb, 256, 0, stream>>>(D, Dd.p);
    DarcyFields F{Dd.phi, Dd.dphi, Dd.k, Dd.vp_avg, Dd.p_old, Dd.dp_expl, Dd.p_constant};
    k_first_solution<<<cb, 256, 0, stream>>>(D, F, Dd.p, Dd.dp_expl, Dd.ctl, P.dt);
    k_jacobi_coef<<<cb, 256, 0, stream>>>(D, F, Dd.ctl, P.dt, Dd.cf, Dd.ca, Dd.csrc, Dd.cbase, Dd.cfixed,
                                          (unsigned long long)Dd.ng);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (Dd.ws) {
        // predicted initial iterate; the previous solution stays unless a
        // candidate has the smaller first residual
        k_free_cells<<<cb, 256, 0, stream>>>(D, Dd.ctl, Dd.p_constant, Dd.freec);
        if ((e = cudaMemcpyAsync(Dd.guess, Dd.p, Dd.ng * 8, cudaMemcpyDeviceToDevice, stream)) != cudaSuccess)
            return e;
        if (Dd.guess_base &&
            (e = cudaMemcpyAsync(Dd.guess_base, Dd.p, Dd.ng * 8, cudaMemcpyDeviceToDevice, stream)) != cudaSuccess)
            return e;
        WSDarcyInputs in{Dd.p, Dd.phi, Dd.dphi, Dd.freec};
        if ((e = ws_predict(Dd.ws, in, Dd.guess, Dd.guess_base, stream)) != cudaSuccess) return e;
        k_ghost<1><<<cb, 256, 0, stream>>>(D, Dd.guess);
        if (Dd.guess_base) k_ghost<1><<<cb, 256, 0, stream>>>(D, Dd.guess_base);
        k_clear_guess_res<<<1, 1, 0, stream>>>(Dd.ctl);
        k_guess_residual<<<cb, 256, 0, stream>>>(D, F, Dd.p, Dd.ctl, P.dt, 0);
        k_guess_residual<<<cb, 256, 0, stream>>>(D, F, Dd.guess, Dd.ctl, P.dt, 1);
        if (Dd.guess_base) k_guess_residual<<<cb, 256, 0, stream>>>(D, F, Dd.guess_base, Dd.ctl, P.dt, 2);
        k_take_guess<<<(unsigned)std::min<size_t>((Dd.ng + 255) / 256, 1024), 256, 0, stream>>>(
            Dd.ctl, Dd.p, Dd.guess, Dd.guess_base, Dd.ng);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // the second buffer starts as a copy (its ghost faces are read too)
    if ((e = cudaMemcpyAsync(Dd.p2, Dd.p, Dd.ng * 8, cudaMemcpyDeviceToDevice, stream)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(Dd.jsync, 0, sizeof(JacobiSync), stream)) != cudaSuccess) return e;
    int exact = darcy_exact_stop;
    JacobiCoef C{Dd.cf, Dd.ca, Dd.csrc, Dd.cbase, Dd.cfixed, (unsigned long long)Dd.ng};
    void *args[] = {(void *)&D, (void *)&F, (void *)&C, (void *)&Dd.p, (void *)&Dd.p2, (void *)&Dd.ctl,
                    (void *)&Dd.jsync, (void *)&exact};
    e = cudaLaunchCooperativeKernel((void *)k_jacobi, dim3(jacobi_grid), dim3(256), args, 0, stream);
    if (e != cudaSuccess) return e;
    k_final_pressure<<<cb, 256, 0, stream>>>(D, Dd.ctl, Dd.p, Dd.p2, Dd.ng);
    if (Dd.ws && (e = ws_train(Dd.ws, Dd.p_old, Dd.p, stream)) != cudaSuccess) return e;
    if (!darcy_keep_dphi) k_zero_interior<<<cb, 256, 0, stream>>>(D, Dd.dphi);
    k_ghost<1><<<cb, 256, 0, stream>>>(D, Dd.p);
    k_velocities<<<cb, 256, 0, stream>>>(D, Dd.p, Dd.phi, Dd.k, Dd.v);
    return cudaGetLastError();
}

int64_t Engine::darcy_field_bytes(int f) const
{
    if (ns) return ns_field_bytes(f);
    if (!darcy) return -1;
    const size_t nc = (size_t)hs.num[0] * hs.num[1] * hs.num[2];
    switch (f) {
    case SPH_F_DARCY_P: case SPH_F_DARCY_PHI: case SPH_F_DARCY_DPHI: case SPH_F_DARCY_K:
        return (int64_t)nc * 8;
    case SPH_F_DARCY_V: return (int64_t)nc * 24;
    case SPH_F_DARCY_F_P: return (int64_t)hs.np * 32;
    case SPH_F_DARCY_ITERS: case SPH_F_DARCY_ITERS_TOTAL: case SPH_F_DARCY_ITERS_EXACT:
        return 8;
    case SPH_F_DARCY_WARM: return 32;
    default: return -1;
    }
}

int Engine::darcy_get(int f, void *dst, size_t bytes)
{
    if (ns) return ns_get(f, dst, bytes);
    if (!darcy) return fail(ST_ARG, "no fluid in this run");
    int64_t need = darcy_field_bytes(f);
    if (need < 0) return fail(ST_ARG, "unknown field");
    if ((!dst && need > 0) || bytes < (size_t)need) return fail(ST_ARG, "destination buffer too small");
    DarcyDev &Dd = *darcy;
    const unsigned cb = cells_blocks(Dd.D);
    cudaError_t e = cudaSuccess;
    const double *src = nullptr;
    int comps = 1;
    switch (f) {
    case SPH_F_DARCY_P: src = Dd.p; break;
    case SPH_F_DARCY_PHI: src = Dd.phi; break;
    case SPH_F_DARCY_DPHI: src = Dd.dphi; break;
    case SPH_F_DARCY_K: src = Dd.k; break;
    case SPH_F_DARCY_V: src = Dd.v; comps = 3; break;
    case SPH_F_DARCY_F_P:
        e = cudaMemcpyAsync(dst, Dd.f_p, (size_t)need, cudaMemcpyDeviceToHost, stream);
        break;
    case SPH_F_DARCY_WARM: {
        // predictions, training steps, solves that used the network's guess,
        // last training loss (as double bits)
        DarcyCtl c;
        e = cudaMemcpyAsync(&c, Dd.ctl, sizeof c, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "get");
        long long v[4] = {0, 0, 0, 0};
        if (Dd.ws) {
            v[0] = ws_predictions(Dd.ws);
            v[1] = ws_trained(Dd.ws);
            v[2] = c.ws_picked;
            double loss = ws_last_loss(Dd.ws, stream);
            std::memcpy(&v[3], &loss, 8);
        }
        std::memcpy(dst, v, 32);
        return ST_OK;
    }
    default: {
        DarcyCtl c;
        e = cudaMemcpyAsync(&c, Dd.ctl, sizeof c, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "get");
        long long v = f == SPH_F_DARCY_ITERS ? c.nijac_last
                      : f == SPH_F_DARCY_ITERS_TOTAL ? c.nijac_total : c.converged_at;
        std::memcpy(dst, &v, 8);
        return ST_OK;
    }
    }
    if (src) {
        e = cudaSuccess;
        k_gather_interior<<<cb, 256, 0, stream>>>(Dd.D, src, Dd.gather, comps);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst, Dd.gather, (size_t)need, cudaMemcpyDeviceToHost, stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e == cudaSuccess ? ST_OK : cuda_fail(e, "get");
}

int Engine::darcy_download()
{
    if (ns) return ns_download();
    if (!darcy) return ST_OK;
    const size_t nc = hs.ncells();
    int rc;
    if ((rc = darcy_get(SPH_F_DARCY_P, hs.p_f.data(), nc * 8))) return rc;
    if ((rc = darcy_get(SPH_F_DARCY_PHI, hs.phi.data(), nc * 8))) return rc;
    if ((rc = darcy_get(SPH_F_DARCY_DPHI, hs.dphi.data(), nc * 8))) return rc;
    if ((rc = darcy_get(SPH_F_DARCY_V, hs.v_f.data(), nc * 24))) return rc;
    std::vector<double4> fp(hs.np);
    if ((rc = darcy_get(SPH_F_DARCY_F_P, fp.data(), hs.np * 32))) return rc;
    for (uint32_t i = 0; i < hs.np; ++i) hs.f_p[i] = d4{fp[i].x, fp[i].y, fp[i].z, 0.0};
    return ST_OK;
}

void Engine::conv_open()
{
    if (!darcy && !ns) return;
    std::string f = outdir + "/" + sid + "-conv.log";
    convlog = std::fopen(f.c_str(), "w");
}

void Engine::conv_close()
{
    if (convlog) std::fclose(convlog);
    convlog = nullptr;
}

// Dry runs step through the captured graphs; with fluid every step runs
// eagerly because the Jacobi loop length is data dependent, and the
// iteration count is read back for the conv log and the stopping check.
int Engine::step_with_fluid_log(uint64_t n)
{
    if (ns) return ns_step_with_log(n);
    if (!darcy) return step(n);
    int warn = ST_OK;
    for (uint64_t i = 0; i < n; ++i) {
        const int64_t it = host_iter;
        // dphi survives only the step that ends at a file output
        // (device.cu:2400-2410)
        darcy_keep_dphi = !(filetimeclock + hs.dt < hs.file_dt);
        cudaError_t e = enqueue_step();
        if (e != cudaSuccess) return cuda_fail(e, "step");
        advance_host_clock(1);
        warmed = true;
        // steps without a solve (ndem > 1) need no read-back; device errors
        // stop the kernels and are reported at the next solve or at the end
        if ((it % (int64_t)darcy->D.ndem) != 0 && i + 1 < n) continue;
        DarcyCtl c;
        e = cudaMemcpyAsync(&c, darcy->ctl, sizeof c, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "step");
        if (c.err == DERR_TIMEOUT) return fail(ST_TIMEOUT, "Darcy solver: a bounded device wait timed out");
        if (c.err == DERR_NAN) return fail(ST_OUTSIDE, "Darcy solver: normalized residual is NaN");
        const bool solved = (it % (int64_t)darcy->D.ndem) == 0;
        // conv log lines as device.cu:2356-2372 (conv_log_interval 10)
        if (solved) {
            if (c.converged) {
                if (convlog && it % 10 == 0)
                    std::fprintf(convlog, "%lld\t%lld\n", (long long)it + 1, c.nijac_last);
            } else {
                warn = SPH_WARN_NOCONV;
                if (convlog) std::fprintf(convlog, "%lld\t%lld\n", (long long)it + 1, c.nijac_last);
            }
        }
        int rc = poll_errors("step");
        if (rc) return rc;
    }
    return warn;
}

}  // namespace sphb
