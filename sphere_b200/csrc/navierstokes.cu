// Navier-Stokes porous flow coupled to the particles (cfd_solver 0) on the
// device.
//
// Follows the cfd_solver == 0 block of DEM::startTime (src/device.cu:1213-
// 1898, with CFD_DEM_COUPLING and SET_2 as src/debug.h defines them) and the
// kernels of src/navierstokes.cuh, compiled with -fmad=false like the
// reference.  Cell fields are ghost-padded (nx+2)(ny+2)(nz+2) doubles and the
// staggered face velocities (nx+3)(ny+3)(nz+3) doubles
// (src/navierstokes.cpp:53-61).  One thread handles one cell (or one face);
// the projection's Jacobi loop (findNSforcing, ghost nodes,
// jacobiIterationNS, copyValues, repeated) runs as one cooperative kernel:
// rotating iterate buffers replace the reference's four kernels per
// iteration, blocks wait (bounded) only for the blocks whose cells they
// read, and the reference's stopping rule (the maximum normalised residual,
// checked at every 10th iteration) is decided on the device.
//
// Where two threads of a reference kernel write one ghost node (a periodic
// bottom with a Dirichlet or Neumann top), the reference's result depends on
// thread scheduling; this file keeps the value of the thread with the larger
// z, the order of the reference's host build.  The reference's smoothing
// kernel updates the pressure change in place while its neighbours read it;
// here it reads the whole field before writing (gamma > 0 only; the default
// gamma is 0, which skips it).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "dem_device.cuh"
#include "../../include/sphere_b200.h"

namespace sphb {

struct NSParams {
    int nx, ny, nz;
    double dx, dy, dz;
    double mu, rho_f, beta, theta, gamma, tolerance, c_phi, c_v, dt, dp_dz;
    double g[3];
    int bc_bot, bc_top;
    unsigned maxiter, ndem, np;
    unsigned inject;                // 1: the Jacobi waits never succeed (a test knob)
};

struct NSCtl {
    long long nijac_last;           // the reference's nijac at the end of the last solve
    long long nijac_total;          // iterations performed since open
    int converged;                  // 1: the last solve met the tolerance
    int err;                        // DERR_TIMEOUT or DERR_NAN
    unsigned barrier_count, barrier_gen;
};

// Synchronisation of the cooperative Jacobi kernel (zeroed before each
// launch).  Block b owns a contiguous range of cells and publishes in
// done[b] how many iterations it has completed; an iteration reads the
// previous iterates of the cells within one z layer only (and, with a
// periodic z boundary, of the far end), so a block waits for the blocks
// around it instead of the whole grid.  The residual maxima of the check
// iterations go to a ring of slots and their arrivals are counted, so every
// block can read a complete maximum.  Each counter has its own 128-byte line.
constexpr unsigned kNSMaxBlocks = 1024;
constexpr unsigned kNSChecks = 8;
struct NSSync {
    unsigned long long ring[kNSChecks];
    unsigned arrive[kNSChecks][32];
    unsigned done[kNSMaxBlocks][32];
};

// The fields the Jacobi kernel reads and writes.
struct NSJacobi {
    double *eps, *b1, *b2;          // the eps field and two rotating iterate buffers
    const double *eps_new;          // values of the rows the update skips
    double *norm, *tmp;
    const double *f1, *f2;
};

struct NSDev {
    NSParams N;
    size_t ng, ngf;                 // padded cell and face counts
    double *p, *v, *v_p, *vp_avg, *d_avg, *F_pf, *phi, *dphi;
    double *eps, *eps_new, *norm, *f1, *f2, *div_phi_vi_v, *tmp, *b1, *b2;
    double *v_x, *v_y, *v_z, *v_p_x, *v_p_y, *v_p_z, *tau_x, *tau_y, *tau_z;
    double *f_pf;                   // 3 doubles per particle, sorted order (the drag force)
    double4 *f_d, *f_p, *f_v, *f_sum;   // original particle order
    double *gather;
    NSCtl *ctl;
    NSSync *sync;
    double host_wall0_w;
    unsigned wall0_iz = 10000000u;
    int jgrid = 0, jthreads = 256;
};

namespace {

constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ unsigned cix(const NSParams &N, int x, int y, int z)
{
    return (unsigned)(x + 1) + (unsigned)(N.nx + 2) * (unsigned)(y + 1) +
           (unsigned)(N.nx + 2) * (unsigned)(N.ny + 2) * (unsigned)(z + 1);
}

__device__ __forceinline__ unsigned fix(const NSParams &N, int x, int y, int z)
{
    return (unsigned)(x + 1) + (unsigned)(N.nx + 3) * (unsigned)(y + 1) +
           (unsigned)(N.nx + 3) * (unsigned)(N.ny + 3) * (unsigned)(z + 1);
}

__device__ __forceinline__ double amean(double a, double b) { return (a + b) * 0.5; }

__device__ __forceinline__ bool cell_of(const NSParams &N, unsigned i, int &x, int &y, int &z)
{
    const unsigned n = (unsigned)N.nx * N.ny * N.nz;
    if (i >= n) return false;
    x = (int)(i % N.nx);
    y = (int)((i / N.nx) % N.ny);
    z = (int)(i / ((unsigned)N.nx * N.ny));
    return true;
}

__device__ __forceinline__ V3 ld3(const double *f, unsigned c) { return mk3(f[3 * c], f[3 * c + 1], f[3 * c + 2]); }
__device__ __forceinline__ void st3(double *f, unsigned c, V3 v)
{
    f[3 * c] = v.x;
    f[3 * c + 1] = v.y;
    f[3 * c + 2] = v.z;
}

// setNSghostNodes<T>(field, bc_bot, bc_top), navierstokes.cuh:660-713, from
// the value of interior cell (x,y,z); C doubles per cell.
template <int C>
__device__ __forceinline__ void ghost_cell(const NSParams &N, double *f, int x, int y, int z, const double *val)
{
    const int nx = N.nx, ny = N.ny, nz = N.nz;
    auto put = [&](int X, int Y, int Z) {
        double *d = &f[(size_t)C * cix(N, X, Y, Z)];
        for (int c = 0; c < C; ++c) d[c] = val[c];
    };
    if (x == 0) put(nx, y, z);
    if (x == nx - 1) put(-1, y, z);
    if (y == 0) put(x, ny, z);
    if (y == ny - 1) put(x, -1, z);
    // a bottom rule yields where a top rule writes the same node
    if (z == 0 && (N.bc_bot == 0 || N.bc_bot == 1) && N.bc_top != 2) put(x, y, -1);
    if (z == 0 && N.bc_bot == 2 && N.bc_top != 0 && N.bc_top != 1) put(x, y, nz);
    if (z == nz - 1 && N.bc_top == 0) put(x, y, nz);
    if (z == nz - 2 && N.bc_top == 1) put(x, y, nz);
    if (z == nz - 1 && N.bc_top == 2) put(x, y, -1);
}

template <int C>
__global__ void k_ghost(NSParams N, double *f)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    double val[C];
    const double *s = &f[(size_t)C * cix(N, x, y, z)];
    for (int c = 0; c < C; ++c) val[c] = s[c];
    ghost_cell<C>(N, f, x, y, z, val);
}

// setNSghostNodesFace<Float>, navierstokes.cuh:715-911
__global__ void k_ghost_face(NSParams N, double *X, double *Y, double *Z)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const int nx = N.nx, ny = N.ny, nz = N.nz, bb = N.bc_bot, bt = N.bc_top;
    const unsigned c = fix(N, x, y, z);
    const double vx = X[c], vy = Y[c], vz = Z[c];
    auto F = [&](int a, int b, int d) { return fix(N, a, b, d); };
    if (x == 0) { X[F(nx, y, z)] = vx; Y[F(nx, y, z)] = vy; Z[F(nx, y, z)] = vz; }
    if (x == 1) X[F(nx + 1, y, z)] = vx;
    if (x == nx - 1) { X[F(-1, y, z)] = vx; Y[F(-1, y, z)] = vy; Z[F(-1, y, z)] = vz; }
    if (z == nz - 1 && x == nx - 1 && bt == 0) Z[F(-1, y, nz)] = vz;
    if (z == nz - 1 && x == nx - 1 && (bt == 1 || bt == 2)) Z[F(-1, y, nz)] = 0.0;
    if (z == 0 && x == nx - 1 && bt == 3) Z[F(-1, y, nz)] = vz;
    if (z == nz - 1 && y == ny - 1 && bt == 0) Z[F(x, -1, nz)] = vz;
    if (z == nz - 1 && y == ny - 1 && (bt == 1 || bt == 2)) Z[F(x, -1, nz)] = 0.0;
    if (z == 0 && y == ny - 1 && bt == 3) Z[F(x, -1, nz)] = vz;
    if (z == 0 && x == 0 && (bb == 0 || bb == 1 || bb == 3)) X[F(nx, y, -1)] = vx;
    if (z == 0 && x == 0 && bb == 2) X[F(nx, y, -1)] = -vx;
    if (z == 0 && y == 0 && (bb == 0 || bb == 1 || bb == 3)) Y[F(x, ny, -1)] = vy;
    if (z == 0 && y == 0 && bb == 2) Y[F(x, ny, -1)] = -vy;
    if (z == nz - 1 && x == 0 && (bt == 0 || bt == 3)) Z[F(nx, y, nz)] = vz;
    if (z == nz - 1 && x == 0 && (bt == 1 || bt == 2)) Z[F(nx, y, nz)] = 0.0;
    if (z == nz - 1 && y == 0 && (bt == 0 || bt == 3)) Z[F(x, ny, nz)] = vz;
    if (z == nz - 1 && y == 0 && (bt == 1 || bt == 2)) Z[F(x, ny, nz)] = 0.0;
    if (z == nz - 1 && x == 0 && (bb == 0 || bb == 1 || bb == 3)) X[F(nx, y, nz)] = vx;
    if (z == nz - 1 && x == 0 && bb == 2) X[F(nx, y, nz)] = -vx;
    if (z == nz - 1 && y == 0 && (bb == 0 || bb == 1 || bb == 3)) Y[F(x, ny, nz)] = vy;
    if (z == nz - 1 && y == 0 && bb == 2) Y[F(x, ny, nz)] = -vy;
    if (y == 0) { X[F(x, ny, z)] = vx; Y[F(x, ny, z)] = vy; Z[F(x, ny, z)] = vz; }
    if (y == 1) Y[F(x, ny + 1, z)] = vy;
    if (y == ny - 1) { X[F(x, -1, z)] = vx; Y[F(x, -1, z)] = vy; Z[F(x, -1, z)] = vz; }
    // bottom rules yield where a top rule of a higher thread writes the node
    if (bt != 3) {
        // the Dirichlet bottom swaps the x and y values, as the reference
        if (z == 0 && bb == 0) { X[F(x, y, -1)] = vy; Y[F(x, y, -1)] = vx; Z[F(x, y, -1)] = vz; }
        if (z == 0 && bb == 1) { X[F(x, y, -1)] = vx; Y[F(x, y, -1)] = vy; Z[F(x, y, -1)] = 0.0; }
        if (z == 0 && bb == 2) { X[F(x, y, -1)] = -vx; Y[F(x, y, -1)] = -vy; Z[F(x, y, -1)] = 0.0; }
    }
    if (z == 0 && bb == 3) {
        if (bt != 1 && bt != 2) { X[F(x, y, nz)] = vx; Y[F(x, y, nz)] = vy; }
        if (bt != 0 && bt != 1 && bt != 2) Z[F(x, y, nz)] = vz;
    }
    if (z == 1 && bb == 3 && bt != 1 && bt != 2) Z[F(x, y, nz + 1)] = vz;
    if (z == nz - 1 && bt == 0) Z[F(x, y, nz)] = vz;
    if (z == nz - 1 && bt == 1) {
        X[F(x, y, nz)] = vx; Y[F(x, y, nz)] = vy; Z[F(x, y, nz)] = 0.0; Z[F(x, y, nz + 1)] = 0.0;
    }
    if (z == nz - 1 && bt == 2) {
        X[F(x, y, nz)] = -vx; Y[F(x, y, nz)] = -vy; Z[F(x, y, nz)] = 0.0; Z[F(x, y, nz + 1)] = 0.0;
    }
    if (z == nz - 1 && bt == 3) { X[F(x, y, -1)] = vx; Y[F(x, y, -1)] = vy; Z[F(x, y, -1)] = vz; }
}

// gradient() and divergence(), navierstokes.cuh:1585-1626
template <class LD>
__device__ __forceinline__ V3 gradient(const NSParams &N, LD ld, int x, int y, int z)
{
    const double xn = ld(cix(N, x - 1, y, z)), xp = ld(cix(N, x + 1, y, z));
    const double yn = ld(cix(N, x, y - 1, z)), yp = ld(cix(N, x, y + 1, z));
    const double zn = ld(cix(N, x, y, z - 1)), zp = ld(cix(N, x, y, z + 1));
    return mk3((xp - xn) / (2.0 * N.dx), (yp - yn) / (2.0 * N.dy), (zp - zn) / (2.0 * N.dz));
}

__device__ __forceinline__ double divergence(const NSParams &N, const double *X, const double *Y,
                                             const double *Z, int x, int y, int z)
{
    const double xn = X[fix(N, x, y, z)], xp = X[fix(N, x + 1, y, z)];
    const double yn = Y[fix(N, x, y, z)], yp = Y[fix(N, x, y + 1, z)];
    const double zn = Z[fix(N, x, y, z)], zp = Z[fix(N, x, y, z + 1)];
    return (xp - xn) / N.dx + (yp - yn) / N.dy + (zp - zn) / N.dz;
}

// findPorositiesVelocitiesDiametersSpherical, navierstokes.cuh:1136-1340:
// the void fraction of a sphere of radius min(dx,dy,dz) at the cell centre,
// from the particles of the 5 x 5 x 5 surrounding sort cells.  The
// reference's averaging branch is guarded by its own initial phi (1.00) and
// never runs, so the velocity and diameter sums are stored undivided.
__global__ void k_porosity(DevParams P, DevState S, NSParams N, double *phi_a, double *dphi_a,
                           double *vp_avg, double *d_avg, int first)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const unsigned cellidx = cix(N, x, y, z);
    if (N.np == 0) {
        phi_a[cellidx] = 1.0;
        dphi_a[cellidx] = 0.0;
        st3(vp_avg, cellidx, mk3(0.0, 0.0, 0.0));
        d_avg[cellidx] = 0.0;
        return;
    }
    const double dx = N.dx, dy = N.dy, dz = N.dz;
    const double R = fmin(dx, fmin(dy, dz));
    const double cell_volume = 4.0 / 3.0 * kPi * R * R * R;
    double void_volume = cell_volume;
    const V3 X = mk3(x * dx + 0.5 * dx, y * dy + 0.5 * dy, z * dz + 0.5 * dz);
    V3 v_avg = mk3(0.0, 0.0, 0.0);
    double davg = 0.0;
    const double phi_0 = phi_a[cellidx];
    for (int z_dim = -2; z_dim < 3; ++z_dim)
        for (int y_dim = -2; y_dim < 3; ++y_dim)
            for (int x_dim = -2; x_dim < 3; ++x_dim) {
                int cx = x + x_dim, cy = y + y_dim, cz = z + z_dim, sx, sy;
                if (!wrap_cell(P, cx, cy, cz, sx, sy)) continue;
                const V3 dm = shift_vec(P, sx, sy);
                const unsigned cell = (unsigned)cx + (unsigned)cy * P.num[0] +
                                      (P.num[0] * P.num[1]) * (unsigned)cz;
                const unsigned start = S.cell_start[cell];
                if (start == 0xffffffffu) continue;
                const unsigned end = S.cell_end[cell];
                for (unsigned i = start; i < end; ++i) {
                    const double4 xr = S.x[i], v = S.vel[i];
                    const double r = xr.w;
                    const V3 dist = add3(mk3(X.x - xr.x, X.y - xr.y, X.z - xr.z), dm);
                    const double d = vlen<0>(dist);
                    if ((R - r) < d && d < (R + r)) {
                        void_volume -= 1.0 / (12.0 * d) *
                                       (kPi * (R + r - d) * (R + r - d) *
                                        (d * d + 2.0 * d * r - 3.0 * r * r + 2.0 * d * R + 6.0 * r * R -
                                         3.0 * R * R));
                        v_avg = add3(v_avg, mk3(v.x, v.y, v.z));
                        davg += 2.0 * r;
                    }
                    if (d <= R - r) {
                        void_volume -= 4.0 / 3.0 * kPi * r * r * r;
                        v_avg = add3(v_avg, mk3(v.x, v.y, v.z));
                        davg += 2.0 * r;
                    }
                }
            }
    const double phi = fmin(1.00, fmax(0.00, void_volume / cell_volume));
    double dphi = phi - phi_0;
    if (first) dphi = 0.0;
    phi_a[cellidx] = phi * N.c_phi;
    dphi_a[cellidx] = dphi * N.c_phi;
    st3(vp_avg, cellidx, v_avg);
    d_avg[cellidx] = davg;
}

// interpolateCenterToFace, navierstokes.cuh:3347-3382 (faces 0..n per axis)
__global__ void k_center_to_face(NSParams N, const double *v, double *X, double *Y, double *Z)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned fx = N.nx + 1, fy = N.ny + 1, fz = N.nz + 1;
    if (i >= fx * fy * fz) return;
    const int x = (int)(i % fx), y = (int)((i / fx) % fy), z = (int)(i / (fx * fy));
    const V3 xn = ld3(v, cix(N, x - 1, y, z)), yn = ld3(v, cix(N, x, y - 1, z));
    const V3 zn = ld3(v, cix(N, x, y, z - 1)), c = ld3(v, cix(N, x, y, z));
    const unsigned f = fix(N, x, y, z);
    X[f] = amean(c.x, xn.x);
    Y[f] = amean(c.y, yn.y);
    Z[f] = amean(c.z, zn.z);
}

// interpolateFaceToCenter, navierstokes.cuh:3384-3425
__global__ void k_face_to_center(NSParams N, const double *X, const double *Y, const double *Z, double *v)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const double x_n = X[fix(N, x, y, z)], x_p = X[fix(N, x + 1, y, z)];
    const double y_n = Y[fix(N, x, y, z)], y_p = Y[fix(N, x, y + 1, z)];
    const double z_n = Z[fix(N, x, y, z)], z_p = Z[fix(N, x, y, z + 1)];
    st3(v, cix(N, x, y, z), mk3(amean(x_n, x_p), amean(y_n, y_p), amean(z_n, z_p)));
}

// findFaceDivTau, navierstokes.cuh:3427-3510
__global__ void k_face_div_tau(NSParams N, const double *X, const double *Y, const double *Z,
                               double *TX, double *TY, double *TZ)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const double dx = N.dx, dy = N.dy, dz = N.dz, mu = N.mu;
    const unsigned f = fix(N, x, y, z);
    auto lap = [&](const double *A) {
        const double c = A[f];
        const double xn = A[fix(N, x - 1, y, z)], xp = A[fix(N, x + 1, y, z)];
        const double yn = A[fix(N, x, y - 1, z)], yp = A[fix(N, x, y + 1, z)];
        const double zn = A[fix(N, x, y, z - 1)], zp = A[fix(N, x, y, z + 1)];
        return mu * ((xp - 2.0 * c + xn) / (dx * dx) + (yp - 2.0 * c + yn) / (dy * dy) +
                     (zp - 2.0 * c + zn) / (dz * dz));
    };
    const double tx = lap(X), ty = lap(Y), tz = lap(Z);
    TX[f] = tx;
    TY[f] = ty;
    TZ[f] = tz;
}

// findInteractionForce, navierstokes.cuh:3141-3282 (one thread per particle
// in sorted order): drag (Di Felice), pressure and viscous forces from the
// particle's cell; the total is added to the particle force, the drag kept
// for the fluid (SET_2) and the parts stored at the original index.
__global__ void k_interaction(DevParams P, DevState S, NSParams N, const double *phi, const double *p,
                              const double *X, const double *Y, const double *Z, const double *TX,
                              const double *TY, const double *TZ, double *f_pf, double4 *f_d_out,
                              double4 *f_p_out, double4 *f_v_out, double4 *f_sum_out)
{
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (S.ctl->err || k >= P.np) return;
    const double4 x = S.x[k], vel = S.vel[k];
    const V3 v_p = mk3(vel.x, vel.y, vel.z);
    const double d = x.w;   // the radius, used as the diameter, as the reference
    const unsigned i_x = (unsigned)floor((x.x - P.origo[0]) / (P.L[0] / P.num[0]));
    const unsigned i_y = (unsigned)floor((x.y - P.origo[1]) / (P.L[1] / P.num[1]));
    const unsigned i_z = (unsigned)floor((x.z - P.origo[2]) / (P.L[2] / P.num[2]));
    if (i_x >= (unsigned)N.nx || i_y >= (unsigned)N.ny || i_z >= (unsigned)N.nz) {
        raise_err(S.ctl, DERR_OUTSIDE, (int)S.orig_of[k]);
        return;
    }
    const int ix = (int)i_x, iy = (int)i_y, iz = (int)i_z;
    const double dx = N.dx, dy = N.dy, dz = N.dz;
    const double ph = phi[cix(N, ix, iy, iz)];
    const V3 v_f = mk3(amean(X[fix(N, ix, iy, iz)], X[fix(N, ix + 1, iy, iz)]),
                       amean(Y[fix(N, ix, iy, iz)], Y[fix(N, ix, iy + 1, iz)]),
                       amean(Z[fix(N, ix, iy, iz)], Z[fix(N, ix, iy, iz + 1)]));
    const V3 div_tau = mk3(amean(TX[fix(N, ix, iy, iz)], TX[fix(N, ix + 1, iy, iz)]),
                           amean(TY[fix(N, ix, iy, iz)], TY[fix(N, ix, iy + 1, iz)]),
                           amean(TZ[fix(N, ix, iy, iz)], TZ[fix(N, ix, iy, iz + 1)]));
    const V3 v_rel = sub3(v_f, v_p);
    const double v_rel_length = vlen<0>(v_rel);
    const double V_p = dx * dy * dz - ph * dx * dy * dz;
    const double Re = N.rho_f * d * ph * v_rel_length / N.mu;
    double Cd = pow(0.63 + 4.8 / pow(Re, 0.5), 2.0);
    double chi = 3.7 - 0.65 * exp(-pow(1.5 - log10(Re), 2.0) / 2.0);
    if (v_rel_length < 1.0e-6) {
        Cd = 0.0;
        chi = 0.0;
    }
    const double s = 0.125 * Cd * N.rho_f * kPi * d * d * ph * ph * v_rel_length;
    const double pw = pow(ph, -chi);
    const V3 f_d = muls3(smul3(s, v_rel), pw);
    const V3 g = gradient(N, [&](unsigned c) { return p[c]; }, ix, iy, iz);
    const V3 f_p = muls3(smul3(-1.0, g), V_p);
    const V3 f_v = muls3(smul3(-1.0, div_tau), V_p);
    const V3 f_pf_ = add3(add3(f_d, f_p), f_v);
    st3(f_pf, k, f_d);
    double4 fo = S.force[k];
    fo.x += f_pf_.x; fo.y += f_pf_.y; fo.z += f_pf_.z; fo.w += 0.0;
    S.force[k] = fo;
    const unsigned o = S.orig_of[k];
    f_d_out[o] = make_double4(f_d.x, f_d.y, f_d.z, 0.0);
    f_p_out[o] = make_double4(f_p.x, f_p.y, f_p.z, 0.0);
    f_v_out[o] = make_double4(f_v.x, f_v.y, f_v.z, 0.0);
    f_sum_out[o] = make_double4(f_d.x + f_p.x + f_v.x, f_d.y + f_p.y + f_v.y, f_d.z + f_p.z + f_v.z, 0.0);
}

// applyInteractionForceToFluid, navierstokes.cuh:3284-3345: the drag of the
// particles of a cell, summed in sorted order, per cell volume
__global__ void k_apply_to_fluid(DevParams P, DevState S, NSParams N, const double *f_pf, double *F_pf)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const unsigned cellID = (unsigned)x + (unsigned)y * P.num[0] + (P.num[0] * P.num[1]) * (unsigned)z;
    const unsigned start = S.cell_start[cellID];
    V3 fi = mk3(0.0, 0.0, 0.0);
    if (start != 0xffffffffu) {
        const unsigned end = S.cell_end[cellID];
        for (unsigned i = start; i < end; ++i) fi = add3(fi, ld3(f_pf, i));
    }
    st3(F_pf, cix(N, x, y, z), divs3(fi, N.dx * N.dy * N.dz));
}

// setNSepsilonTop / Bottom / Interior / AtTopWall, setUpperPressureNS and
// setNSnormZero (navierstokes.cuh:356-516, 1550-1582) in one kernel
// selected by `what`.
enum { EPS_TOP = 0, EPS_AT_WALL, EPS_UPPER_PRESSURE, EPS_INTERIOR, EPS_NORM_ZERO, EPS_BOTTOM };

__global__ void k_eps_set(NSParams N, int what, double *eps, double *eps_new, double *p, double *norm,
                          double value, unsigned iz)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const unsigned c = cix(N, x, y, z);
    const int nz = N.nz;
    switch (what) {
    case EPS_TOP:
        if (z == nz - 1) { eps[c] = value; eps_new[c] = value; }
        break;
    case EPS_AT_WALL:
        if ((unsigned)z == iz) { eps[c] = value; eps_new[c] = value; }
        if ((unsigned)z == iz + 1) {
            const double pz = value - N.dp_dz;
            eps[c] = pz;
            eps_new[c] = pz;
        }
        break;
    case EPS_UPPER_PRESSURE:
        if (z == nz - 1) {
            const double e = value - N.beta * p[c];
            eps[c] = e;
            eps_new[c] = e;
            p[c] = value;
        }
        break;
    case EPS_INTERIOR:
        if (z > 0 && z < nz - 1) eps[c] = value;
        break;
    case EPS_NORM_ZERO:
        norm[c] = 0.0;
        break;
    case EPS_BOTTOM:
        if (z == 0) { eps[c] = value; eps_new[c] = value; }
        break;
    }
}

// findNSdivphiviv, navierstokes.cuh:1909-2043 (half upwind, half central)
__global__ void k_div_phi_vi_v(NSParams N, const double *phi, const double *v, double *out)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const double phi_xn = phi[cix(N, x - 1, y, z)], ph = phi[cix(N, x, y, z)];
    const double phi_xp = phi[cix(N, x + 1, y, z)], phi_yn = phi[cix(N, x, y - 1, z)];
    const double phi_yp = phi[cix(N, x, y + 1, z)], phi_zn = phi[cix(N, x, y, z - 1)];
    const double phi_zp = phi[cix(N, x, y, z + 1)];
    const V3 v_xn = ld3(v, cix(N, x - 1, y, z)), vc = ld3(v, cix(N, x, y, z));
    const V3 v_xp = ld3(v, cix(N, x + 1, y, z)), v_yn = ld3(v, cix(N, x, y - 1, z));
    const V3 v_yp = ld3(v, cix(N, x, y + 1, z)), v_zn = ld3(v, cix(N, x, y, z - 1));
    const V3 v_zp = ld3(v, cix(N, x, y, z + 1));
    const double a[3] = {copysign(1.0, vc.x), copysign(1.0, vc.y), copysign(1.0, vc.z)};
    const double vv[3] = {vc.x, vc.y, vc.z};
    const double vxn[3] = {v_xn.x, v_xn.y, v_xn.z}, vxp[3] = {v_xp.x, v_xp.y, v_xp.z};
    const double vyn[3] = {v_yn.x, v_yn.y, v_yn.z}, vyp[3] = {v_yp.x, v_yp.y, v_yp.z};
    const double vzn[3] = {v_zn.x, v_zn.y, v_zn.z}, vzp[3] = {v_zp.x, v_zp.y, v_zp.z};
    const double two_dx = 2.0 * N.dx, two_dy = 2.0 * N.dy, two_dz = 2.0 * N.dz;
    double res[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        // component i: d(phi v_i v_j)/dx_j summed over j = x, y, z
        const double uw =
            ((1.0 + a[0]) * (ph * vv[i] * vv[0] - phi_xn * vxn[i] * vxn[0]) +
             (1.0 - a[0]) * (phi_xp * vxp[i] * vxp[0] - ph * vv[i] * vv[0])) / two_dx +
            ((1.0 + a[1]) * (ph * vv[i] * vv[1] - phi_yn * vyn[i] * vyn[1]) +
             (1.0 - a[1]) * (phi_yp * vyp[i] * vyp[1] - ph * vv[i] * vv[1])) / two_dy +
            ((1.0 + a[2]) * (ph * vv[i] * vv[2] - phi_zn * vzn[i] * vzn[2]) +
             (1.0 - a[2]) * (phi_zp * vzp[i] * vzp[2] - ph * vv[i] * vv[2])) / two_dz;
        const double cd = (phi_xp * vxp[i] * vxp[0] - phi_xn * vxn[i] * vxn[0]) / two_dx +
                          (phi_yp * vyp[i] * vyp[1] - phi_yn * vyn[i] * vyn[1]) / two_dy +
                          (phi_zp * vzp[i] * vzp[2] - phi_zn * vzn[i] * vzn[2]) / two_dz;
        const double tau = 0.5;
        res[i] = tau * uw + (1.0 - tau) * cd;
    }
    st3(out, cix(N, x, y, z), mk3(res[0], res[1], res[2]));
}

// findPredNSvelocities, navierstokes.cuh:2276-2495 (SET_2)
__global__ void k_pred_velocity(NSParams N, const double *p, const double *X, const double *Y,
                                const double *Z, const double *phi_a, const double *dphi_a,
                                const double *TX, const double *TY, const double *TZ, const double *dpvv,
                                const double *F_pf, unsigned wall0_iz, double *PX, double *PY, double *PZ)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const unsigned fidx = fix(N, x, y, z), c = cix(N, x, y, z);
    const unsigned cxn = cix(N, x - 1, y, z), cyn = cix(N, x, y - 1, z), czn = cix(N, x, y, z - 1);
    const V3 v = mk3(X[fidx], Y[fidx], Z[fidx]);
    V3 div_tau = mk3(0.0, 0.0, 0.0);
    if (N.mu > 0.0) div_tau = mk3(TX[fidx], TY[fidx], TZ[fidx]);
    const V3 phi = mk3(amean(phi_a[c], phi_a[cxn]), amean(phi_a[c], phi_a[cyn]), amean(phi_a[c], phi_a[czn]));
    const V3 dphi = mk3(amean(dphi_a[c], dphi_a[cxn]), amean(dphi_a[c], dphi_a[cyn]),
                        amean(dphi_a[c], dphi_a[czn]));
    V3 f_i = mk3(0.0, 0.0, 0.0);
    if (N.mu > 0.0 && N.np > 0) {
        const V3 fc = ld3(F_pf, c), fxn = ld3(F_pf, cxn), fyn = ld3(F_pf, cyn), fzn = ld3(F_pf, czn);
        f_i = mk3(amean(fc.x, fxn.x), amean(fc.y, fyn.y), amean(fc.z, fzn.z));
    }
    const double dt = N.ndem * N.dt;
    V3 pressure_term = mk3(0.0, 0.0, 0.0);
    if (N.beta > 0.0) {
        const double pc = p[c];
        const V3 grad_p = mk3((pc - p[cxn]) / N.dx, (pc - p[cyn]) / N.dy, (pc - p[czn]) / N.dz);
        pressure_term = smul3(-N.beta * dt / N.rho_f, grad_p);
    }
    // the reference pairs the neighbours' x components with the centre's
    // y and z components
    const V3 dc = ld3(dpvv, c), dxn = ld3(dpvv, cxn), dyn = ld3(dpvv, cyn), dzn = ld3(dpvv, czn);
    const V3 div_phi_vi_v = mk3(amean(dxn.x, dc.x), amean(dyn.x, dc.y), amean(dzn.x, dc.z));
    const V3 interaction_term = mk3(-dt / (N.rho_f * phi.x) * f_i.x, -dt / (N.rho_f * phi.y) * f_i.y,
                                    -dt / (N.rho_f * phi.z) * f_i.z);
    const V3 gravity_term = mk3(N.g[0] * dt, N.g[1] * dt, N.g[2] * dt);
    const V3 advection_term = mk3(-1.0 * div_phi_vi_v.x * dt / phi.x, -1.0 * div_phi_vi_v.y * dt / phi.y,
                                  -1.0 * div_phi_vi_v.z * dt / phi.z);
    const V3 porosity_term = mk3(-1.0 * v.x * dphi.x / phi.x, -1.0 * v.y * dphi.y / phi.y,
                                 -1.0 * v.z * dphi.z / phi.z);
    const V3 diffusion_term = smul3(dt / N.rho_f, div_tau);
    const V3 sum = add3(add3(add3(add3(add3(pressure_term, interaction_term), diffusion_term), gravity_term),
                             porosity_term),
                        advection_term);
    V3 v_p = add3(v, smul3(N.c_v, sum));
    if (z == 0 && N.bc_bot == 1) v_p.z = 0.0;
    if (z == 0 && N.bc_bot == 2) v_p = mk3(0.0, 0.0, 0.0);
    if ((unsigned)z >= wall0_iz) v_p = mk3(0.0, 0.0, 0.0);
    PX[fidx] = v_p.x;
    PY[fidx] = v_p.y;
    PZ[fidx] = v_p.z;
}

// The iteration-independent part of findNSforcing (nijac == 0,
// navierstokes.cuh:2530-2575, SET_2): f1 and f2 = grad(phi)/phi
__global__ void k_forcing_const(NSParams N, const double *phi_a, const double *dphi_a, const double *v_p,
                                const double *PX, const double *PY, const double *PZ, double *f1,
                                double *f2)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const unsigned c = cix(N, x, y, z);
    const V3 vp = ld3(v_p, c);
    const double phi = phi_a[c], dphi = dphi_a[c];
    const double div_v_p = divergence(N, PX, PY, PZ, x, y, z);
    const V3 grad_phi = gradient(N, [&](unsigned i) { return phi_a[i]; }, x, y, z);
    const double dt = N.dt * N.ndem;
    const double t1 = N.rho_f * div_v_p / (N.c_v * dt);
    const double t2 = N.rho_f * dot3(grad_phi, vp) / (N.c_v * dt * phi);
    const double t4 = N.rho_f * dphi / (dt * dt * phi * N.c_v);
    f1[c] = t1 + t2 + t4;
    st3(f2, c, divs3(grad_phi, phi));
}

// Bounded grid barrier of the cooperative Jacobi kernel: after ~2^24 polls
// it records DERR_TIMEOUT and returns false instead of spinning forever.
// With `inject` no block releases it and every block gives up after
// kInjectPolls polls.
__device__ bool ns_barrier(NSCtl *ctl, unsigned nblocks, unsigned inject)
{
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        volatile unsigned *gen = &ctl->barrier_gen;
        const unsigned g = *gen;
        __threadfence();
        const unsigned arrived = atomicAdd(&ctl->barrier_count, 1u);
        ok = 1;
        if (arrived == nblocks - 1 && !inject) {
            ctl->barrier_count = 0;
            __threadfence();
            atomicAdd(&ctl->barrier_gen, 1u);
        } else {
            unsigned spins = 0;
            const unsigned limit = inject ? kInjectPolls : (1u << 24);
            while (inject || *gen == g) {
                if (++spins > limit) {
                    atomicCAS(&ctl->err, 0, (int)DERR_TIMEOUT);
                    ok = 0;
                    break;
                }
                if (((volatile int *)&ctl->err)[0] != 0) { ok = 0; break; }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

__device__ __forceinline__ double ldg(const double *p) { return __ldcg(p); }

// The Jacobi loop of the projection step (device.cu:1631-1822) in one
// cooperative launch.
//
// The reference's iteration n is four kernels: the forcing from the current
// interior E_n and the ghost nodes of the previous iterate g(E_n-1) (its
// ghosts are refreshed after the forcing), the ghost nodes g(E_n), the
// relaxed Jacobi update from E_n and g(E_n), and the copy back.  Here three
// padded buffers rotate: iteration n reads E_n with its fresh ghosts from
// P[n%3] and the previous ghosts from P[(n+2)%3], and writes E_n+1 and its
// ghost images to P[(n+1)%3].  Rows the update skips (Dirichlet boundaries)
// take E_n+1 from eps_new, as the reference's copy does.
//
// Block b updates the cells [b*chunk, (b+1)*chunk).  Before iteration n it
// waits until the blocks whose cells lie within reach (one z layer, one row
// and one cell: the stencil and the ghost nodes the cells write; the whole
// grid with a periodic z boundary) have completed iteration n-1.  That makes
// their part of E_n visible, and since those are the only blocks that read
// this block's cells, none of them still reads the buffer iteration n
// overwrites.  At every 10th iteration each block adds its maximum
// |residual| to a slot and its arrival to a counter; the stop is decided at
// the start of the next iteration from the complete maximum.  At the end
// P[0] (the eps field) receives the final interior and the ghosts the
// reference leaves: those of the final iterate after convergence, those of
// the last input iterate when maxiter is reached.

// Waits (thread-wise, bounded) until *p >= target with acquire semantics;
// records DERR_TIMEOUT after ~2^22 polls or stops when another block has
// flagged an error.
__device__ __forceinline__ bool ns_wait_ge(const unsigned *p, unsigned target, NSCtl *ctl,
                                           unsigned inject)
{
    unsigned spins = 0, nap = 16;
    const unsigned limit = inject ? kInjectPolls : (1u << 22);
    for (;;) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        if (v >= target && !inject) return true;
        if (++spins > limit) {
            atomicCAS(&ctl->err, 0, (int)DERR_TIMEOUT);
            return false;
        }
        if (*(volatile int *)&ctl->err != 0) return false;
        __nanosleep(nap);
        if (nap < 128) nap <<= 1;
    }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_jacobi(NSParams N, NSJacobi J, NSCtl *ctl, NSSync *S, unsigned wall0_iz)
{
    const unsigned nc = (unsigned)N.nx * N.ny * N.nz;
    const unsigned ng = (unsigned)(N.nx + 2) * (N.ny + 2) * (N.nz + 2);
    const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    const int nx = N.nx, ny = N.ny, nz = N.nz;
    const int zmin = N.bc_bot == 0 ? 1 : 0;
    const int zmax = N.bc_top == 0 ? nz - 2 : nz - 1;
    const double dxdx = N.dx * N.dx, dydy = N.dy * N.dy, dzdz = N.dz * N.dz;
    const double den = 2.0 * (dxdx * dydy + dxdx * dzdz + dydy * dzdz);
    // the rotating buffers, selected without a local-memory array
    auto P = [&](unsigned k) { return k == 0 ? J.eps : k == 1 ? J.b1 : J.b2; };
    __shared__ unsigned long long wmax[NT / 32];
    bool ok = true, conv = false;
    long long last = -1;
    if (N.maxiter > 0) {
        // P[2] carries the loop's incoming ghost nodes (read by the first
        // forcing); P[0] gets the fresh ghosts of E_0
        for (unsigned q = tid; q < ng; q += stride) J.b2[q] = J.eps[q];
        ok = ns_barrier(ctl, gridDim.x, N.inject);
        if (ok) {
            for (unsigned i = tid; i < nc; i += stride) {
                int x, y, z;
                cell_of(N, i, x, y, z);
                const double val = J.eps[cix(N, x, y, z)];
                ghost_cell<1>(N, J.eps, x, y, z, &val);
            }
            ok = ns_barrier(ctl, gridDim.x, N.inject);
        }
    }
    // this block's cells and the blocks whose cells its iteration reads
    const unsigned G = gridDim.x, b = blockIdx.x;
    const unsigned chunk = (nc + G - 1) / G;
    const unsigned lo = min(nc, b * chunk), hi = min(nc, lo + chunk);
    const bool zwrap = N.bc_bot == 2 || N.bc_top == 2;
    const unsigned reach = zwrap ? nc : (unsigned)nx * ny + (unsigned)nx + 1u;
    const unsigned nb_lo = lo > reach ? (lo - reach) / chunk : 0u;
    const unsigned nb_hi = min(G - 1u, (hi + reach) / chunk);
    __shared__ int s_state;   // 0 continue, 1 converged, 2 stop (error)
    if (threadIdx.x == 0) s_state = 0;
    __syncthreads();
    // the stop rule of check iteration c (thread 0): every block's maximum
    auto decide = [&](unsigned c) {
        const unsigned k = c / 10u;
        if (!ns_wait_ge(&S->arrive[k % kNSChecks][0], G, ctl, N.inject)) {
            s_state = 2;
            return;
        }
        const unsigned long long mb = __ldcg(&S->ring[k % kNSChecks]);
        if (b == 0) {
            // every block has decided the checks before k
            S->ring[(k + kNSChecks / 2) % kNSChecks] = 0ull;
            if (k >= 2) S->arrive[(k - 2) % kNSChecks][0] = 0u;
        }
        if (mb > 0x7ff0000000000000ull) {
            // a NaN residual: maxNormResNS stops the run (navierstokes.cpp:283-300)
            atomicCAS(&ctl->err, 0, (int)DERR_NAN);
            s_state = 2;
        } else if (__longlong_as_double((long long)mb) < N.tolerance) {
            s_state = 1;
        }
    };
    for (unsigned nijac = 0; ok && nijac < N.maxiter; ++nijac) {
        if (threadIdx.x < 32 && nijac > 0) {
            if (threadIdx.x == 0 && (nijac - 1u) % 10u == 0u) decide(nijac - 1u);
            __syncwarp();
            if (s_state == 0) {
                // the lanes of warp 0 watch the neighbours in parallel
                bool okw = true;
                for (unsigned q = nb_lo + threadIdx.x; q <= nb_hi; q += 32)
                    if (q != b && !ns_wait_ge(&S->done[q][0], nijac, ctl, N.inject)) okw = false;
                if (!__all_sync(0xffffffffu, okw) && threadIdx.x == 0) s_state = 2;
            }
        }
        // the acquire loads above and this barrier make the neighbours'
        // cells visible to the whole block
        __syncthreads();
        if (s_state != 0) break;
        const double *cur = P(nijac % 3), *prev = P((nijac + 2) % 3);
        double *next = P((nijac + 1) % 3);
        const bool check = nijac % 10 == 0;
        unsigned long long m = 0;
        for (unsigned i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            int x, y, z;
            cell_of(N, i, x, y, z);
            const unsigned c = cix(N, x, y, z);
            double val, res_norm;
            if (z >= zmin && z <= zmax) {
                // findNSforcing: interior from E_n, ghost nodes from g(E_n-1)
                auto ef = [&](int X, int Y, int Z) {
                    const bool ghost = X < 0 || X >= nx || Y < 0 || Y >= ny || Z < 0 || Z >= nz;
                    const unsigned q = cix(N, X, Y, Z);
                    return ldg(ghost ? &prev[q] : &cur[q]);
                };
                const V3 ge = mk3((ef(x + 1, y, z) - ef(x - 1, y, z)) / (2.0 * N.dx),
                                  (ef(x, y + 1, z) - ef(x, y - 1, z)) / (2.0 * N.dy),
                                  (ef(x, y, z + 1) - ef(x, y, z - 1)) / (2.0 * N.dz));
                const double f = J.f1[c] - dot3(ge, ld3(J.f2, c));
                // jacobiIterationNS from E_n and g(E_n)
                const double e_xn = ldg(&cur[cix(N, x - 1, y, z)]), e = ldg(&cur[c]);
                const double e_xp = ldg(&cur[cix(N, x + 1, y, z)]), e_yn = ldg(&cur[cix(N, x, y - 1, z)]);
                const double e_yp = ldg(&cur[cix(N, x, y + 1, z)]), e_zn = ldg(&cur[cix(N, x, y, z - 1)]);
                const double e_zp = ldg(&cur[cix(N, x, y, z + 1)]);
                double e_new = (-dxdx * dydy * dzdz * f + dydy * dzdz * (e_xn + e_xp) +
                                dxdx * dzdz * (e_yn + e_yp) + dxdx * dydy * (e_zn + e_zp)) /
                               den;
                if ((unsigned)z == wall0_iz) e_new = e;
                if ((unsigned)z == wall0_iz + 1) e_new = e_zn + N.dp_dz;
                res_norm = (e_new - e) * (e_new - e) / (e_new * e_new + 1.0e-16);
                val = e * (1.0 - N.theta) + e_new * N.theta;
                J.norm[c] = res_norm;
            } else {
                val = J.eps_new[c];
                res_norm = J.norm[c];
            }
            next[c] = val;
            ghost_cell<1>(N, next, x, y, z, &val);
            if (check) {
                const unsigned long long bits = (unsigned long long)__double_as_longlong(fabs(res_norm));
                m = bits > m ? bits : m;
            }
        }
        if (check) {
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long q = __shfl_down_sync(0xffffffffu, m, o);
                m = q > m ? q : m;
            }
            if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
        }
        // the barrier orders every thread's cell stores before thread 0's
        // release (cumulative at GPU scope), so the neighbours may go on
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(&S->done[b][0]), "r"(nijac + 1u) : "memory");
            if (check) {
                unsigned long long bm = 0;
                for (unsigned w = 0; w < NT / 32; ++w) bm = wmax[w] > bm ? wmax[w] : bm;
                const unsigned k = nijac / 10u;
                atomicMax(&S->ring[k % kNSChecks], bm);
                asm volatile("red.release.gpu.global.add.u32 [%0], 1;" :: "l"(&S->arrive[k % kNSChecks][0]) : "memory");
            }
        }
        last = nijac;
    }
    // the last iteration's check, when the loop ran to maxiter
    if (threadIdx.x == 0 && s_state == 0 && last >= 0 && last + 1 == (long long)N.maxiter &&
        (unsigned)last % 10u == 0u)
        decide((unsigned)last);
    __syncthreads();
    if (s_state == 2) ok = false;
    conv = s_state == 1;
    // every block's cells before the final copy
    if (ok && last >= 0) ok = ns_barrier(ctl, gridDim.x, N.inject);
    if (ok && last >= 0) {
        const double *fin = P((unsigned)((last + 1) % 3));
        const double *gsrc = conv ? fin : P((unsigned)(last % 3));
        for (unsigned q = tid; q < ng; q += stride) {
            const int x = (int)(q % (unsigned)(nx + 2)) - 1;
            const int y = (int)((q / (unsigned)(nx + 2)) % (unsigned)(ny + 2)) - 1;
            const int z = (int)(q / ((unsigned)(nx + 2) * (unsigned)(ny + 2))) - 1;
            const bool interior = x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz;
            const double *src = interior ? fin : gsrc;
            if (src != J.eps) J.eps[q] = ldg(&src[q]);
        }
    }
    if (ok && conv && N.gamma > 0.0) {
        // smoothing<Float>, navierstokes.cuh:2619-2677, reading the whole
        // field before writing, then the ghost nodes again
        ok = ns_barrier(ctl, gridDim.x, N.inject);
        if (ok) {
            for (unsigned i = tid; i < nc; i += stride) {
                int x, y, z;
                cell_of(N, i, x, y, z);
                if (z < zmin || z > zmax) continue;
                const unsigned c = cix(N, x, y, z);
                const double e_xn = ldg(&J.eps[cix(N, x - 1, y, z)]), e = ldg(&J.eps[c]);
                const double e_xp = ldg(&J.eps[cix(N, x + 1, y, z)]);
                const double e_yn = ldg(&J.eps[cix(N, x, y - 1, z)]);
                const double e_yp = ldg(&J.eps[cix(N, x, y + 1, z)]);
                const double e_zn = ldg(&J.eps[cix(N, x, y, z - 1)]);
                const double e_zp = ldg(&J.eps[cix(N, x, y, z + 1)]);
                const double e_avg = 1.0 / 6.0 * (e_xn + e_xp + e_yn + e_yp + e_zn + e_zp);
                J.tmp[c] = (1.0 - N.gamma) * e + N.gamma * e_avg;
            }
            ok = ns_barrier(ctl, gridDim.x, N.inject);
        }
        if (ok) {
            for (unsigned i = tid; i < nc; i += stride) {
                int x, y, z;
                cell_of(N, i, x, y, z);
                if (z < zmin || z > zmax) continue;
                const unsigned c = cix(N, x, y, z);
                J.eps[c] = ldg(&J.tmp[c]);
            }
            ok = ns_barrier(ctl, gridDim.x, N.inject);
        }
        if (ok) {
            for (unsigned i = tid; i < nc; i += stride) {
                int x, y, z;
                cell_of(N, i, x, y, z);
                const double val = ldg(&J.eps[cix(N, x, y, z)]);
                ghost_cell<1>(N, J.eps, x, y, z, &val);
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->nijac_last = last;
        ctl->converged = conv ? 1 : 0;
        ctl->nijac_total += last + 1;
    }
}

// updateNSpressure, navierstokes.cuh:2881-2913
__global__ void k_update_pressure(NSParams N, const double *eps, double *p)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const unsigned c = cix(N, x, y, z);
    p[c] = N.beta * p[c] + eps[c];
}

// updateNSvelocity, navierstokes.cuh:2915-3057 (SET_2)
__global__ void k_update_velocity(NSParams N, const double *PX, const double *PY, const double *PZ,
                                  const double *eps, unsigned wall0_iz, double *X, double *Y, double *Z)
{
    int x, y, z;
    if (!cell_of(N, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const unsigned f = fix(N, x, y, z);
    const V3 v_p = mk3(PX[f], PY[f], PZ[f]);
    const double ec = eps[cix(N, x, y, z)];
    const V3 grad_epsilon = mk3((ec - eps[cix(N, x - 1, y, z)]) / N.dx, (ec - eps[cix(N, x, y - 1, z)]) / N.dy,
                                (ec - eps[cix(N, x, y, z - 1)]) / N.dz);
    V3 v = sub3(v_p, smul3(N.c_v * N.ndem * N.dt / N.rho_f, grad_epsilon));
    if (z == 0 && N.bc_bot == 1) v.z = 0.0;
    if (z == 0 && N.bc_bot == 2) v = mk3(0.0, 0.0, 0.0);
    if ((unsigned)z >= wall0_iz) v = mk3(0.0, 0.0, 0.0);
    X[f] = v.x;
    Y[f] = v.y;
    Z[f] = v.z;
}

// interior cells (x fastest) of a padded field, comps doubles per cell
__global__ void k_gather(NSParams N, const double *src, double *dst, int comps)
{
    int x, y, z;
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (!cell_of(N, i, x, y, z)) return;
    const unsigned c = cix(N, x, y, z);
    for (int k = 0; k < comps; ++k) dst[(size_t)comps * i + k] = src[(size_t)comps * c + k];
}

// faces 0..n per axis of the three staggered arrays, (x, y, z) per face
__global__ void k_gather_face(NSParams N, const double *X, const double *Y, const double *Z, double *dst)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned fx = N.nx + 1, fy = N.ny + 1, fz = N.nz + 1;
    if (i >= fx * fy * fz) return;
    const int x = (int)(i % fx), y = (int)((i / fx) % fy), z = (int)(i / (fx * fy));
    const unsigned f = fix(N, x, y, z);
    dst[3 * (size_t)i] = X[f];
    dst[3 * (size_t)i + 1] = Y[f];
    dst[3 * (size_t)i + 2] = Z[f];
}

unsigned blocks_for(size_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace

// ---------------------------------------------------------------------
// engine glue
// ---------------------------------------------------------------------
int Engine::ns_init()
{
    ns = new NSDev();
    NSDev &D = *ns;
    NSParams &N = D.N;
    N.nx = (int)hs.num[0]; N.ny = (int)hs.num[1]; N.nz = (int)hs.num[2];
    N.dx = hs.L[0] / hs.num[0]; N.dy = hs.L[1] / hs.num[1]; N.dz = hs.L[2] / hs.num[2];
    N.mu = hs.mu; N.rho_f = hs.rho_f; N.beta = hs.ns_beta; N.theta = hs.ns_theta; N.gamma = hs.ns_gamma;
    N.tolerance = hs.tolerance; N.c_phi = hs.c_phi; N.c_v = hs.c_v; N.dt = hs.dt;
    // device.cu:1009-1011
    N.dp_dz = std::fabs(hs.rho_f * hs.g[2] * hs.L[2] / hs.num[2]);
    for (int k = 0; k < 3; ++k) N.g[k] = hs.g[k];
    N.bc_bot = hs.bc_bot; N.bc_top = hs.bc_top;
    N.maxiter = hs.maxiter; N.ndem = hs.ndem; N.np = hs.np;
    N.inject = (inject & kInjectNS) ? 1u : 0u;
    const size_t nx = N.nx, ny = N.ny, nz = N.nz;
    D.ng = (nx + 2) * (ny + 2) * (nz + 2);
    D.ngf = (nx + 3) * (ny + 3) * (nz + 3);
    const size_t ng = D.ng, ngf = D.ngf;
    for (double **a : {&D.p, &D.d_avg, &D.phi, &D.dphi, &D.eps, &D.eps_new, &D.norm, &D.f1, &D.tmp, &D.b1,
                       &D.b2})
        *a = dalloc<double>(ng);
    for (double **a : {&D.v, &D.v_p, &D.vp_avg, &D.F_pf, &D.f2, &D.div_phi_vi_v}) *a = dalloc<double>(3 * ng);
    for (double **a : {&D.v_x, &D.v_y, &D.v_z, &D.v_p_x, &D.v_p_y, &D.v_p_z, &D.tau_x, &D.tau_y, &D.tau_z})
        *a = dalloc<double>(ngf);
    D.f_pf = dalloc<double>(3 * (size_t)hs.np);
    for (double4 **a : {&D.f_d, &D.f_p, &D.f_v, &D.f_sum}) *a = dalloc<double4>(hs.np);
    D.gather = dalloc<double>(3 * (nx + 1) * (ny + 1) * (nz + 1));
    D.ctl = dalloc<NSCtl>(1);
    D.sync = dalloc<NSSync>(1);
    if (alloc_failed) return fail(ST_CUDA, "device allocation failed (Navier-Stokes)");
    // interior cells from the file; the ghost nodes start at zero
    auto cidx_h = [&](size_t x, size_t y, size_t z) {
        return (x + 1) + (nx + 2) * (y + 1) + (nx + 2) * (ny + 2) * (z + 1);
    };
    std::vector<double> p(ng, 0.0), phi(ng, 0.0), dphi(ng, 0.0), v(3 * ng, 0.0);
    for (size_t z = 0; z < nz; ++z)
        for (size_t y = 0; y < ny; ++y)
            for (size_t x = 0; x < nx; ++x) {
                const size_t f = (z * ny + y) * nx + x, g = cidx_h(x, y, z);
                p[g] = hs.p_f[f]; phi[g] = hs.phi[f]; dphi[g] = hs.dphi[f];
                for (int c = 0; c < 3; ++c) v[3 * g + c] = hs.v_f[3 * f + c];
            }
    cudaMemcpyAsync(D.p, p.data(), ng * 8, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(D.phi, phi.data(), ng * 8, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(D.dphi, dphi.data(), ng * 8, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(D.v, v.data(), 3 * ng * 8, cudaMemcpyHostToDevice, stream);
    if (hs.np) {
        std::vector<double4> a(hs.np);
        const std::vector<d4> *src[4] = {&hs.f_d, &hs.f_p, &hs.f_v, &hs.f_sum};
        double4 *dst[4] = {D.f_d, D.f_p, D.f_v, D.f_sum};
        for (int q = 0; q < 4; ++q) {
            for (uint32_t i = 0; i < hs.np; ++i) {
                const d4 s = i < src[q]->size() ? (*src[q])[i] : d4{};
                a[i] = make_double4(s.x, s.y, s.z, 0.0);
            }
            cudaMemcpyAsync(dst[q], a.data(), hs.np * 32, cudaMemcpyHostToDevice, stream);
            cudaStreamSynchronize(stream);
        }
    }
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "Navier-Stokes upload");
    D.host_wall0_w = hs.nw > 0 ? hs.wnx[0].w : 0.0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // threads per block of the Jacobi launch: 256, up to four blocks per SM
    // and one cell per thread (500 blocks on the 40 x 40 x 80 grid; measured
    // 2.5 ms per DEM step against 2.7 with 250 blocks of 512 and 3.2 with 296
    // of 256);
    // SPHB_NS_THREADS=512 and SPHB_NS_BLOCKS_PER_SM override them for tuning
    D.jthreads = 256;
    if (const char *env = std::getenv("SPHB_NS_THREADS")) D.jthreads = std::atoi(env) == 512 ? 512 : 256;
    if (D.jthreads == 512)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jacobi<512>, 512, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jacobi<256>, 256, 0);
    if (per_sm < 1) return fail(ST_CUDA, "Navier-Stokes Jacobi kernel cannot be resident");
    int bps = 4;
    if (const char *env = std::getenv("SPHB_NS_BLOCKS_PER_SM")) bps = std::max(1, std::atoi(env));
    D.jgrid = std::min<int>(sms * std::min(per_sm, bps),
                            (int)((nx * ny * nz + D.jthreads - 1) / D.jthreads));
    D.jgrid = std::min<int>(D.jgrid, (int)kNSMaxBlocks);
    return ST_OK;
}

void Engine::ns_free()
{
    delete ns;   // device arrays are released with the engine's allocations
    ns = nullptr;
}

void Engine::ns_set_host_wall()
{
    if (ns) ns->host_wall0_w = hs.nw > 0 ? hs.wnx[0].w : 0.0;
}

// The cfd_solver == 0 block of one DEM step (device.cu:1213-1898).
cudaError_t Engine::enqueue_ns()
{
    NSDev &D = *ns;
    const NSParams &N = D.N;
    const size_t nc = (size_t)N.nx * N.ny * N.nz;
    const unsigned cb = blocks_for(nc);
    const unsigned fb = blocks_for((size_t)(N.nx + 1) * (N.ny + 1) * (N.nz + 1));
    const int64_t it = host_iter;
    cudaError_t e;
    k_porosity<<<cb, 256, 0, stream>>>(P, S, N, D.phi, D.dphi, D.vp_avg, D.d_avg, it == 0 ? 1 : 0);
    if (it == 0) {
        k_ghost<3><<<cb, 256, 0, stream>>>(N, D.v);
        k_center_to_face<<<fb, 256, 0, stream>>>(N, D.v, D.v_x, D.v_y, D.v_z);
    }
    k_ghost_face<<<cb, 256, 0, stream>>>(N, D.v_x, D.v_y, D.v_z);
    k_face_div_tau<<<cb, 256, 0, stream>>>(N, D.v_x, D.v_y, D.v_z, D.tau_x, D.tau_y, D.tau_z);
    k_ghost_face<<<cb, 256, 0, stream>>>(N, D.tau_x, D.tau_y, D.tau_z);
    k_ghost<1><<<cb, 256, 0, stream>>>(N, D.p);
    k_ghost<1><<<cb, 256, 0, stream>>>(N, D.phi);
    if (hs.np > 0) {
        k_interaction<<<blocks_for(hs.np), 256, 0, stream>>>(P, S, N, D.phi, D.p, D.v_x, D.v_y, D.v_z, D.tau_x,
                                                               D.tau_y, D.tau_z, D.f_pf, D.f_d, D.f_p, D.f_v,
                                                               D.f_sum);
        k_ghost<1><<<cb, 256, 0, stream>>>(N, D.p);
        k_apply_to_fluid<<<cb, 256, 0, stream>>>(P, S, N, D.f_pf, D.F_pf);
        k_ghost<3><<<cb, 256, 0, stream>>>(N, D.F_pf);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((it % (int64_t)N.ndem) != 0) return cudaSuccess;
    // boundary values of the pressure change from the host's copy of the
    // pressure, refreshed at file output as in the reference
    const size_t nx = N.nx, ny = N.ny;
    auto host_p = [&](size_t x, size_t y, size_t z) { return hs.p_f[(z * ny + y) * nx + x]; };
    const double p_top = host_p(0, 0, N.nz - 1);
    const double eps_top = p_top - N.beta * p_top;
    k_eps_set<<<cb, 256, 0, stream>>>(N, EPS_TOP, D.eps, D.eps_new, D.p, D.norm, eps_top, 0u);
    if (hs.nw > 0 && (hs.wmode[0] == 1 || hs.wmode[0] == 3)) {
        D.wall0_iz = (unsigned)(D.host_wall0_w / (hs.L[2] / hs.num[2]));
        k_eps_set<<<cb, 256, 0, stream>>>(N, EPS_AT_WALL, D.eps, D.eps_new, D.p, D.norm, eps_top, D.wall0_iz);
    }
    if ((hs.p_mod_A > 1.0e-5 || hs.p_mod_A < -1.0e-5) && hs.p_mod_f > 1.0e-7) {
        const double new_pressure = p_top + hs.p_mod_A * std::sin(2.0 * 3.14159265358979323846 * hs.p_mod_f * host_t +
                                                                  hs.p_mod_phi);
        k_eps_set<<<cb, 256, 0, stream>>>(N, EPS_UPPER_PRESSURE, D.eps, D.eps_new, D.p, D.norm, new_pressure, 0u);
    }
    k_ghost<1><<<cb, 256, 0, stream>>>(N, D.p);
    k_ghost_face<<<cb, 256, 0, stream>>>(N, D.v_p_x, D.v_p_y, D.v_p_z);
    k_ghost<1><<<cb, 256, 0, stream>>>(N, D.phi);
    k_ghost<1><<<cb, 256, 0, stream>>>(N, D.dphi);
    k_face_to_center<<<cb, 256, 0, stream>>>(N, D.v_x, D.v_y, D.v_z, D.v);
    k_ghost<3><<<cb, 256, 0, stream>>>(N, D.v);
    k_div_phi_vi_v<<<cb, 256, 0, stream>>>(N, D.phi, D.v, D.div_phi_vi_v);
    k_ghost<3><<<cb, 256, 0, stream>>>(N, D.div_phi_vi_v);
    k_pred_velocity<<<cb, 256, 0, stream>>>(N, D.p, D.v_x, D.v_y, D.v_z, D.phi, D.dphi, D.tau_x, D.tau_y, D.tau_z,
                                            D.div_phi_vi_v, D.F_pf, D.wall0_iz, D.v_p_x, D.v_p_y, D.v_p_z);
    k_ghost_face<<<cb, 256, 0, stream>>>(N, D.v_p_x, D.v_p_y, D.v_p_z);
    k_face_to_center<<<cb, 256, 0, stream>>>(N, D.v_p_x, D.v_p_y, D.v_p_z, D.v_p);
    if (it == 0) {
        const double p222 = host_p(2, 2, 2), p000 = host_p(0, 0, 0);
        k_eps_set<<<cb, 256, 0, stream>>>(N, EPS_INTERIOR, D.eps, D.eps_new, D.p, D.norm, p222 - N.beta * p222, 0u);
        k_eps_set<<<cb, 256, 0, stream>>>(N, EPS_NORM_ZERO, D.eps, D.eps_new, D.p, D.norm, 0.0, 0u);
        k_eps_set<<<cb, 256, 0, stream>>>(N, EPS_BOTTOM, D.eps, D.eps_new, D.p, D.norm, p000 - N.beta * p000, 0u);
        k_ghost<1><<<cb, 256, 0, stream>>>(N, D.eps);
    }
    k_forcing_const<<<cb, 256, 0, stream>>>(N, D.phi, D.dphi, D.v_p, D.v_p_x, D.v_p_y, D.v_p_z, D.f1, D.f2);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(D.sync, 0, sizeof(NSSync), stream)) != cudaSuccess) return e;
    NSJacobi J{D.eps, D.b1, D.b2, D.eps_new, D.norm, D.tmp, D.f1, D.f2};
    NSParams Nc = N;
    unsigned wall = D.wall0_iz;
    NSCtl *ctl = D.ctl;
    NSSync *sync = D.sync;
    void *args[] = {(void *)&Nc, (void *)&J, (void *)&ctl, (void *)&sync, (void *)&wall};
    e = cudaLaunchCooperativeKernel(D.jthreads == 512 ? (void *)k_jacobi<512> : (void *)k_jacobi<256>,
                                    dim3(D.jgrid), dim3(D.jthreads), args, 0, stream);
    if (e != cudaSuccess) return e;
    k_update_pressure<<<cb, 256, 0, stream>>>(N, D.eps, D.p);
    k_update_velocity<<<cb, 256, 0, stream>>>(N, D.v_p_x, D.v_p_y, D.v_p_z, D.eps, D.wall0_iz, D.v_x, D.v_y,
                                              D.v_z);
    k_ghost_face<<<cb, 256, 0, stream>>>(N, D.v_p_x, D.v_p_y, D.v_p_z);
    k_face_to_center<<<cb, 256, 0, stream>>>(N, D.v_x, D.v_y, D.v_z, D.v);
    return cudaGetLastError();
}

int64_t Engine::ns_field_bytes(int f) const
{
    const size_t nc = hs.ncells();
    const size_t nf = (size_t)(hs.num[0] + 1) * (hs.num[1] + 1) * (hs.num[2] + 1);
    switch (f) {
    case SPH_F_DARCY_P: case SPH_F_DARCY_PHI: case SPH_F_DARCY_DPHI: case SPH_F_NS_EPSILON:
    case SPH_F_NS_NORM:
        return (int64_t)nc * 8;
    case SPH_F_DARCY_V: return (int64_t)nc * 24;
    case SPH_F_NS_V_FACE: return (int64_t)nf * 24;
    case SPH_F_DARCY_F_P: case SPH_F_NS_F_D: case SPH_F_NS_F_V: case SPH_F_NS_F_SUM:
        return (int64_t)hs.np * 32;
    case SPH_F_DARCY_ITERS: case SPH_F_DARCY_ITERS_TOTAL: return 8;
    default: return -1;
    }
}

int Engine::ns_get(int f, void *dst, size_t bytes)
{
    const int64_t need = ns_field_bytes(f);
    if (need < 0) return fail(ST_ARG, "field not available with the Navier-Stokes solver");
    if ((!dst && need > 0) || bytes < (size_t)need) return fail(ST_ARG, "destination buffer too small");
    NSDev &D = *ns;
    const NSParams &N = D.N;
    const size_t nc = hs.ncells();
    cudaError_t e = cudaSuccess;
    const double *src = nullptr;
    int comps = 1;
    const double4 *part = nullptr;
    switch (f) {
    case SPH_F_DARCY_P: src = D.p; break;
    case SPH_F_DARCY_PHI: src = D.phi; break;
    case SPH_F_DARCY_DPHI: src = D.dphi; break;
    case SPH_F_NS_EPSILON: src = D.eps; break;
    case SPH_F_NS_NORM: src = D.norm; break;
    case SPH_F_DARCY_V: src = D.v; comps = 3; break;
    case SPH_F_DARCY_F_P: part = D.f_p; break;
    case SPH_F_NS_F_D: part = D.f_d; break;
    case SPH_F_NS_F_V: part = D.f_v; break;
    case SPH_F_NS_F_SUM: part = D.f_sum; break;
    case SPH_F_NS_V_FACE:
        k_gather_face<<<blocks_for((size_t)need / 24), 256, 0, stream>>>(N, D.v_x, D.v_y, D.v_z, D.gather);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst, D.gather, (size_t)need, cudaMemcpyDeviceToHost, stream);
        break;
    default: {
        NSCtl c;
        e = cudaMemcpyAsync(&c, D.ctl, sizeof c, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "get");
        const long long v = f == SPH_F_DARCY_ITERS ? c.nijac_last : c.nijac_total;
        std::memcpy(dst, &v, 8);
        return ST_OK;
    }
    }
    if (part) e = cudaMemcpyAsync(dst, part, (size_t)need, cudaMemcpyDeviceToHost, stream);
    if (src) {
        k_gather<<<blocks_for(nc), 256, 0, stream>>>(N, src, D.gather, comps);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst, D.gather, (size_t)need, cudaMemcpyDeviceToHost, stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e == cudaSuccess ? ST_OK : cuda_fail(e, "get");
}

// Host copies for a file: the cell-centre velocities are interpolated from
// the faces first (device.cu:2586-2593).
int Engine::ns_download()
{
    NSDev &D = *ns;
    const NSParams &N = D.N;
    const size_t nc = hs.ncells();
    k_face_to_center<<<blocks_for(nc), 256, 0, stream>>>(N, D.v_x, D.v_y, D.v_z, D.v);
    int rc;
    if ((rc = ns_get(SPH_F_DARCY_P, hs.p_f.data(), nc * 8))) return rc;
    if ((rc = ns_get(SPH_F_DARCY_PHI, hs.phi.data(), nc * 8))) return rc;
    if ((rc = ns_get(SPH_F_DARCY_DPHI, hs.dphi.data(), nc * 8))) return rc;
    if ((rc = ns_get(SPH_F_DARCY_V, hs.v_f.data(), nc * 24))) return rc;
    const int fields[4] = {SPH_F_NS_F_D, SPH_F_DARCY_F_P, SPH_F_NS_F_V, SPH_F_NS_F_SUM};
    std::vector<d4> *dst[4] = {&hs.f_d, &hs.f_p, &hs.f_v, &hs.f_sum};
    std::vector<double4> a(hs.np);
    for (int q = 0; q < 4; ++q) {
        if (hs.np && (rc = ns_get(fields[q], a.data(), hs.np * 32))) return rc;
        dst[q]->assign(hs.np, d4{});
        for (uint32_t i = 0; i < hs.np; ++i) (*dst[q])[i] = d4{a[i].x, a[i].y, a[i].z, 0.0};
    }
    return ST_OK;
}

// DEM::checkNSstability (src/navierstokes.cpp:86-123) on the host copy of
// the cell-centre velocities, before a file is written.
int Engine::ns_check_stability()
{
    const double dx = hs.L[0] / hs.num[0], dy = hs.L[1] / hs.num[1], dz = hs.L[2] / hs.num[2];
    const double dmin = std::fmin(dx, std::fmin(dy, dz));
    if (hs.mu * hs.dt / (dmin * dmin) > 0.5)
        return fail(ST_INPUT, "The time step is too large to ensure stability in the diffusive term of the "
                              "fluid momentum equation");
    const size_t nx = hs.num[0], ny = hs.num[1], nz = hs.num[2];
    for (size_t x = 0; x < nx; ++x)
        for (size_t y = 0; y < ny; ++y)
            for (size_t z = 0; z < nz; ++z) {
                const double *v = &hs.v_f[3 * ((z * ny + y) * nx + x)];
                if (v[0] * hs.dt / dx + v[1] * hs.dt / dy + v[2] * hs.dt / dz > 1.0) {
                    char m[256];
                    std::snprintf(m, sizeof m,
                                  "The time step is too large to ensure stability in the advective term of "
                                  "the fluid momentum equation: v(%zu,%zu,%zu) = [%g,%g,%g] m/s",
                                  x, y, z, v[0], v[1], v[2]);
                    return fail(ST_INPUT, m);
                }
            }
    return ST_OK;
}

// Fluid steps run eagerly (the Jacobi loop length is data dependent); the
// iteration count of each projection is read back for the conv log
// (device.cu:1782-1835, conv_log_interval 10).
int Engine::ns_step_with_log(uint64_t n)
{
    int warn = ST_OK;
    for (uint64_t i = 0; i < n; ++i) {
        const int64_t it = host_iter;
        cudaError_t e = enqueue_step();
        if (e != cudaSuccess) return cuda_fail(e, "step");
        advance_host_clock(1);
        warmed = true;
        // steps without a projection (ndem > 1) need no read-back; device
        // errors stop the kernels and are reported at the next projection
        // or at the end of the call
        if ((it % (int64_t)ns->N.ndem) != 0 && i + 1 < n) continue;
        NSCtl c;
        e = cudaMemcpyAsync(&c, ns->ctl, sizeof c, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "step");
        if (c.err == DERR_TIMEOUT) return fail(ST_TIMEOUT, "Navier-Stokes solver: a bounded device wait timed out");
        if (c.err == DERR_NAN) return fail(ST_OUTSIDE, "Navier-Stokes solver: normalized residual is NaN");
        if ((it % (int64_t)ns->N.ndem) == 0 && ns->N.maxiter > 0) {
            if (c.converged) {
                if (convlog && it % 10 == 0) std::fprintf(convlog, "%lld\t%lld\n", (long long)it + 1, c.nijac_last);
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
