/*
 * Host build of the reference's own DEM step -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference kernels (sorting.cuh, contactmodels.cuh, cohesion.cuh,
 * contactsearch.cuh, integration.cuh) are #included unchanged from the
 * reference tree (REF_DIR) and run one thread at a time through a serial
 * launch loop.  The reference's own DEM constructor, readbin/writebin and
 * checkValues (sphere.cpp, file_io.cpp) are linked unchanged; this file
 * supplies host versions of the device-memory members of device.cu and a
 * step driver that follows the stage order of DEM::startTime
 * (device.cu:1038-2550).  The result is the reference run here, used to pin
 * the C oracle.  Thrust's stable sort_by_key is replaced by std::stable_sort
 * of (key, index) pairs, which yields the same permutation.
 */
#include "ref_shim.h"

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#define private public
#include "sphere.h"
#undef private
#include "datatypes.h"
#include "constants.cuh"
#include "vector_arithmetic.h"

uint3 ref_threadIdx, ref_blockIdx;
dim3 ref_blockDim, ref_gridDim;
/* backing store for `extern __shared__` arrays (reorderArrays) */
unsigned int shared_data[1025];

#include "sorting.cuh"
#include "contactmodels.cuh"
#include "cohesion.cuh"
#include "contactsearch.cuh"
#include "integration.cuh"
#include "navierstokes.cuh"
#include "darcy.cuh"

template <class F> static void launch(unsigned grid, unsigned block, F f)
{
    ref_gridDim = dim3(grid, 1, 1);
    ref_blockDim = dim3(block, 1, 1);
    for (unsigned b = 0; b < grid; ++b) {
        ref_blockIdx = make_uint3(b, 0, 0);
        for (unsigned t = 0; t < block; ++t) {
            ref_threadIdx = make_uint3(t, 0, 0);
            f();
        }
    }
}

template <class F> static void launch3(dim3 grid, dim3 block, F f)
{
    ref_gridDim = grid;
    ref_blockDim = block;
    for (unsigned bz = 0; bz < grid.z; ++bz)
        for (unsigned by = 0; by < grid.y; ++by)
            for (unsigned bx = 0; bx < grid.x; ++bx) {
                ref_blockIdx = make_uint3(bx, by, bz);
                for (unsigned tz = 0; tz < block.z; ++tz)
                    for (unsigned ty = 0; ty < block.y; ++ty)
                        for (unsigned tx = 0; tx < block.x; ++tx) {
                            ref_threadIdx = make_uint3(tx, ty, tz);
                            f();
                        }
            }
}

/* The reference's ray-tracing kernels (src/raytracer.cuh:14-275), compiled
 * from the reference's file in a unit of their own (oracle/Makefile). */
void imageInit(unsigned char *dev_img, const unsigned int pixels);
void rayInitPerspective(float4 *dev_ray_origo, float4 *dev_ray_direction, const float4 eye,
                        const unsigned int width, const unsigned int height);
void rayIntersectSpheres(const float4 *dev_ray_origo, const float4 *dev_ray_direction,
                         const Float4 *dev_x, unsigned char *dev_img);
void rayIntersectSpheresColormap(const float4 *dev_ray_origo, const float4 *dev_ray_direction,
                                 const Float4 *dev_x, const Float4 *dev_vel, const Float *dev_linarr,
                                 const float max_val, const float lower_cutoff,
                                 unsigned char *dev_img);

static unsigned idiv_up(unsigned a, unsigned b) { return (a % b != 0) ? (a / b + 1) : (a / b); }

/* ---- host stand-ins for the device-memory members of device.cu ---- */
void DEM::initializeGPU() {}
void DEM::checkForCudaErrors(const char *, const int) {}
void DEM::checkForCudaErrorsIter(const char *, const unsigned int, const int) {}
void DEM::transferToConstantDeviceMemory()
{
    /* device.cu:331-357 */
    devC_nd = nd;
    devC_np = np;
    devC_nw = walls.nw;
    devC_nc = NC;
    devC_dt = time.dt;
    devC_nb0 = params.nb0;
    devC_params = params;
    devC_grid = grid;
}

template <class T> static T *halloc(size_t n)
{
    T *p = new T[n ? n : 1];
    std::memset((void *)p, 0, sizeof(T) * (n ? n : 1));
    return p;
}

void DEM::allocateGlobalDeviceMemory()
{
    /* device.cu:405-487; the history arrays start at zero (the reference
     * copies uninitialised host memory). */
    k.acc = halloc<Float4>(np);
    k.angacc = halloc<Float4>(np);
    dev_x = halloc<Float4>(np); dev_xyzsum = halloc<Float4>(np);
    dev_vel = halloc<Float4>(np); dev_vel0 = halloc<Float4>(np);
    dev_acc = halloc<Float4>(np); dev_force = halloc<Float4>(np);
    dev_angpos = halloc<Float4>(np); dev_angvel = halloc<Float4>(np);
    dev_angvel0 = halloc<Float4>(np); dev_angacc = halloc<Float4>(np);
    dev_torque = halloc<Float4>(np);
    dev_contacts = halloc<unsigned int>((size_t)np * NC);
    dev_distmod = halloc<Float4>((size_t)np * NC);
    dev_delta_t = halloc<Float4>((size_t)np * NC);
    dev_bonds = halloc<uint2>(params.nb0);
    dev_bonds_delta = halloc<Float4>(params.nb0);
    dev_bonds_omega = halloc<Float4>(params.nb0);
    dev_x_sorted = halloc<Float4>(np); dev_vel_sorted = halloc<Float4>(np);
    dev_angvel_sorted = halloc<Float4>(np);
    dev_es_dot = halloc<Float>(np); dev_es = halloc<Float>(np);
    dev_ev_dot = halloc<Float>(np); dev_ev = halloc<Float>(np);
    dev_p = halloc<Float>(np);
    dev_gridParticleCellID = halloc<unsigned int>(np);
    dev_gridParticleIndex = halloc<unsigned int>(np);
    size_t ncell = (size_t)grid.num[0] * grid.num[1] * grid.num[2];
    dev_cellStart = halloc<unsigned int>(ncell);
    dev_cellEnd = halloc<unsigned int>(ncell);
    k.contacts = halloc<unsigned int>((size_t)np * NC);
    for (size_t i = 0; i < (size_t)np * NC; ++i) k.contacts[i] = np;
    k.distmod = halloc<Float4>((size_t)np * NC);
    k.delta_t = halloc<Float4>((size_t)np * NC);
    unsigned nw = walls.nw;
    dev_walls_wmode = halloc<int>(nw);
    dev_walls_nx = halloc<Float4>(nw);
    dev_walls_mvfd = halloc<Float4>(nw);
    dev_walls_tau_x = halloc<Float>(nw);
    dev_walls_tau_eff_x_pp = halloc<Float>((size_t)nw * np);
    dev_walls_force_pp = halloc<Float>((size_t)nw * np);
    dev_walls_acc = halloc<Float>(nw);
    unsigned blocks = idiv_up(np, 256);
    dev_walls_force_partial = halloc<Float>((size_t)blocks * (nw ? nw : 1));
    dev_walls_tau_eff_x_partial = halloc<Float>((size_t)blocks * (nw ? nw : 1));
}

void DEM::transferToGlobalDeviceMemory(int)
{
    /* device.cu:667-752 */
    size_t f4 = sizeof(Float4) * np, f1 = sizeof(Float) * np;
    std::memcpy(dev_x, k.x, f4); std::memcpy(dev_xyzsum, k.xyzsum, f4);
    std::memcpy(dev_vel, k.vel, f4); std::memcpy(dev_vel0, k.vel, f4);
    std::memcpy(dev_acc, k.acc, f4); std::memcpy(dev_force, k.force, f4);
    std::memcpy(dev_angpos, k.angpos, f4); std::memcpy(dev_angvel, k.angvel, f4);
    std::memcpy(dev_angvel0, k.angvel, f4); std::memcpy(dev_angacc, k.angacc, f4);
    std::memcpy(dev_torque, k.torque, f4);
    std::memcpy(dev_contacts, k.contacts, sizeof(unsigned int) * np * NC);
    std::memcpy(dev_distmod, k.distmod, f4 * NC);
    std::memcpy(dev_delta_t, k.delta_t, f4 * NC);
    if (params.nb0) {
        std::memcpy(dev_bonds, k.bonds, sizeof(uint2) * params.nb0);
        std::memcpy(dev_bonds_delta, k.bonds_delta, sizeof(Float4) * params.nb0);
        std::memcpy(dev_bonds_omega, k.bonds_omega, sizeof(Float4) * params.nb0);
    }
    std::memcpy(dev_es_dot, e.es_dot, f1); std::memcpy(dev_es, e.es, f1);
    std::memcpy(dev_ev_dot, e.ev_dot, f1); std::memcpy(dev_ev, e.ev, f1);
    std::memcpy(dev_p, e.p, f1);
    std::memcpy(dev_walls_wmode, walls.wmode, sizeof(int) * walls.nw);
    std::memcpy(dev_walls_nx, walls.nx, sizeof(Float4) * walls.nw);
    std::memcpy(dev_walls_mvfd, walls.mvfd, sizeof(Float4) * walls.nw);
    if (walls.nw) std::memcpy(dev_walls_tau_x, walls.tau_x, sizeof(Float));
    if (fluid == 1 && cfd_solver == 1) transferDarcyToGlobalDeviceMemory(0);
    if (fluid == 1 && cfd_solver == 0) transferNStoGlobalDeviceMemory(0);
}

void DEM::transferFromGlobalDeviceMemory()
{
    /* device.cu:754-829 */
    size_t f4 = sizeof(Float4) * np, f1 = sizeof(Float) * np;
    std::memcpy(k.x, dev_x, f4); std::memcpy(k.xyzsum, dev_xyzsum, f4);
    std::memcpy(k.vel, dev_vel, f4); std::memcpy(k.acc, dev_acc, f4);
    std::memcpy(k.force, dev_force, f4); std::memcpy(k.angpos, dev_angpos, f4);
    std::memcpy(k.angvel, dev_angvel, f4); std::memcpy(k.angacc, dev_angacc, f4);
    std::memcpy(k.torque, dev_torque, f4);
    std::memcpy(k.contacts, dev_contacts, sizeof(unsigned int) * np * NC);
    std::memcpy(k.distmod, dev_distmod, f4 * NC);
    std::memcpy(k.delta_t, dev_delta_t, f4 * NC);
    if (params.nb0) {
        std::memcpy(k.bonds, dev_bonds, sizeof(uint2) * params.nb0);
        std::memcpy(k.bonds_delta, dev_bonds_delta, sizeof(Float4) * params.nb0);
        std::memcpy(k.bonds_omega, dev_bonds_omega, sizeof(Float4) * params.nb0);
    }
    std::memcpy(e.es_dot, dev_es_dot, f1); std::memcpy(e.es, dev_es, f1);
    std::memcpy(e.ev_dot, dev_ev_dot, f1); std::memcpy(e.ev, dev_ev, f1);
    std::memcpy(e.p, dev_p, f1);
    std::memcpy(walls.nx, dev_walls_nx, sizeof(Float4) * walls.nw);
    std::memcpy(walls.mvfd, dev_walls_mvfd, sizeof(Float4) * walls.nw);
    if (fluid == 1 && cfd_solver == 1) transferDarcyFromGlobalDeviceMemory(0);
    if (fluid == 1 && cfd_solver == 0) transferNSfromGlobalDeviceMemory(0);
}

void DEM::freeGlobalDeviceMemory() {}

/* ---- the step driver: DEM::startTime's loop body, dry part ---- */
struct RefRun {
    DEM *dem;
    long iter;
    int velocity_state;
    unsigned wall0_iz;
    long nijac_last;
    long nijac_total;
    double filetimeclock;
    int ns_converged;
};

/* summation (integration.cuh:309-341) uses a 256-wide shared-memory tree
 * across the threads of a block; that cannot run one thread at a time, so
 * it is restated here with the same order of additions. */
static void ref_summation(const Float *in, Float *out, unsigned np, unsigned blocks)
{
    Float cache[256];
    for (unsigned b = 0; b < blocks; ++b) {
        for (unsigned t = 0; t < 256; ++t) {
            unsigned idx = t + b * 256;
            Float temp = 0.0f;
            while (idx < np) { temp += in[idx]; idx += 256 * blocks; }
            cache[t] = temp;
        }
        for (unsigned i = 128; i != 0; i /= 2)
            for (unsigned t = 0; t < i; ++t) cache[t] += cache[t + i];
        out[b] = cache[0];
    }
}


/* The Darcy block of DEM::startTime, device.cu:1901-2426 (cfd_solver 1),
 * kernels launched one thread at a time. */
static void ref_darcy(RefRun *r)
{
    DEM &d = *r->dem;
    unsigned np = d.np;
    unsigned tpb = 256, bpg = idiv_up(np, tpb);
    dim3 blk(8, 8, 8);
    dim3 grd(idiv_up(d.grid.num[0], 8), idiv_up(d.grid.num[1], 8), idiv_up(d.grid.num[2], 8));
    Darcy &D = d.darcy;
    if (d.walls.nw > 0 && (d.walls.wmode[0] == 1 || d.walls.wmode[0] == 3))
        r->wall0_iz = d.walls.nx->w / (d.grid.L[2] / d.grid.num[2]);
    unsigned wall0_iz = r->wall0_iz;
    auto ghost = [&](Float *f) {
        launch3(grd, blk, [&] { setDarcyGhostNodes<Float>(f, D.bc_xn, D.bc_xp, D.bc_yn, D.bc_yp, D.bc_bot, D.bc_top); });
    };
    if (np > 0) {
        ghost(d.dev_darcy_p);
        launch3(grd, blk, [&] { findDarcyPressureGradient(d.dev_darcy_p, d.dev_darcy_grad_p); });
        launch3(grd, blk, [&] { setDarcyGhostNodes<Float3>(d.dev_darcy_grad_p, D.bc_xn, D.bc_xp, D.bc_yn, D.bc_yp, D.bc_bot, D.bc_top); });
        launch(bpg, tpb, [&] {
            findDarcyPressureForceLinear(d.dev_x, d.dev_darcy_grad_p, d.dev_darcy_phi, wall0_iz,
                                         D.rho_f, D.bc_top, d.dev_force, d.dev_darcy_f_p);
        });
    }
    if ((r->iter % D.ndem) == 0) {
        launch3(grd, blk, [&] {
            findDarcyPorositiesLinear(d.dev_cellStart, d.dev_cellEnd, d.dev_x_sorted, d.dev_vel_sorted,
                                      (unsigned)r->iter, D.ndem, np, D.c_phi, d.dev_darcy_phi,
                                      d.dev_darcy_dphi, d.dev_darcy_div_v_p, d.dev_darcy_vp_avg);
        });
        if (d.grid.periodic == 2) {
            launch3(grd, blk, [&] { copyDarcyPorositiesToEdges(d.dev_darcy_phi, d.dev_darcy_dphi, d.dev_darcy_div_v_p, d.dev_darcy_vp_avg); });
            launch3(grd, blk, [&] { copyDarcyPorositiesToBottom(d.dev_darcy_phi, d.dev_darcy_dphi, d.dev_darcy_div_v_p, d.dev_darcy_vp_avg); });
        }
        if ((D.p_mod_A > 1.0e-5 || D.p_mod_A < -1.0e-5) && D.p_mod_f > 1.0e-7) {
            Float new_pressure = D.p_top_orig + D.p_mod_A * sin(2.0 * M_PI * D.p_mod_f * d.time.current + D.p_mod_phi);
            launch3(grd, blk, [&] { setDarcyTopPressure(new_pressure, d.dev_darcy_p, wall0_iz); });
            launch3(grd, blk, [&] { setDarcyTopWallPressure(new_pressure, wall0_iz, d.dev_darcy_p); });
        }
        launch3(grd, blk, [&] { findDarcyPermeabilities(D.k_c, d.dev_darcy_phi, d.dev_darcy_k); });
        ghost(d.dev_darcy_phi);
        ghost(d.dev_darcy_k);
        launch3(grd, blk, [&] { findDarcyPermeabilityGradients(d.dev_darcy_k, d.dev_darcy_grad_k); });
        if (r->iter == 0) {
            launch3(grd, blk, [&] { setDarcyNormZero(d.dev_darcy_norm); });
            launch3(grd, blk, [&] { copyValues<Float>(d.dev_darcy_p, d.dev_darcy_p_old); });
        }
        auto flux = [&] {
            launch3(grd, blk, [&] {
                setDarcyGhostNodesFlux<Float>(d.dev_darcy_p, D.bc_bot, D.bc_top, D.bc_bot_flux,
                                              D.bc_top_flux, d.dev_darcy_k, D.mu);
            });
        };
        if (D.bc_bot == 4 || D.bc_top == 4) flux();
        long done = 0;
        for (unsigned int nijac = 0; nijac < D.maxiter; ++nijac) {
            if (nijac == 0)
                launch3(grd, blk, [&] { copyValues<Float>(d.dev_darcy_p, d.dev_darcy_p_old); });
            ghost(d.dev_darcy_p);
            if (nijac == 0)
                launch3(grd, blk, [&] {
                    firstDarcySolution(d.dev_darcy_p, d.dev_darcy_k, d.dev_darcy_phi, d.dev_darcy_dphi,
                                       d.dev_darcy_div_v_p, d.dev_darcy_vp_avg, d.dev_darcy_grad_k,
                                       D.beta_f, D.mu, D.bc_xn, D.bc_xp, D.bc_yn, D.bc_yp, D.bc_bot,
                                       D.bc_top, D.ndem, wall0_iz, d.dev_darcy_p_constant,
                                       d.dev_darcy_dp_expl);
                });
            launch3(grd, blk, [&] {
                updateDarcySolution(d.dev_darcy_p_old, d.dev_darcy_dp_expl, d.dev_darcy_p, d.dev_darcy_k,
                                    d.dev_darcy_phi, d.dev_darcy_dphi, d.dev_darcy_div_v_p,
                                    d.dev_darcy_vp_avg, d.dev_darcy_grad_k, D.beta_f, D.mu, D.bc_xn,
                                    D.bc_xp, D.bc_yn, D.bc_yp, D.bc_bot, D.bc_top, D.ndem, wall0_iz,
                                    d.dev_darcy_p_constant, d.dev_darcy_p_new, d.dev_darcy_norm);
            });
            if (D.bc_top == 1) launch3(grd, blk, [&] { setDarcyTopWallFixedFlow(wall0_iz, d.dev_darcy_p); });
            if (D.bc_bot == 4 || D.bc_top == 4) flux();
            launch3(grd, blk, [&] { copyValues<Float>(d.dev_darcy_p_new, d.dev_darcy_p); });
            done = nijac;
            if (nijac % nijacnorm == 0) {
                d.transferDarcyNormFromGlobalDeviceMemory();
                double max_norm_res = d.maxNormResDarcy();
                if (max_norm_res <= D.tolerance) break;
            }
        }
        r->nijac_last = done;
        r->nijac_total += done + 1;
        if (r->filetimeclock + d.time.dt < d.time.file_dt)
            launch3(grd, blk, [&] { setDarcyZeros<Float>(d.dev_darcy_dphi); });
        ghost(d.dev_darcy_p);
        launch3(grd, blk, [&] { findDarcyVelocities(d.dev_darcy_p, d.dev_darcy_phi, d.dev_darcy_k, D.mu, d.dev_darcy_v); });
    }
}

/* The Navier-Stokes block of DEM::startTime, device.cu:1213-1898
 * (cfd_solver 0, CFD_DEM_COUPLING), kernels launched one thread at a time. */
static void ref_ns(RefRun *r)
{
    DEM &d = *r->dem;
    NavierStokes &ns = d.ns;
    unsigned np = d.np;
    unsigned tpb = 256, bpg = idiv_up(np, tpb);
    dim3 blk(8, 8, 8);
    dim3 grd(idiv_up(d.grid.num[0], 8), idiv_up(d.grid.num[1], 8), idiv_up(d.grid.num[2], 8));
    dim3 grdf(idiv_up(d.grid.num[0] + 1, 8), idiv_up(d.grid.num[1] + 1, 8), idiv_up(d.grid.num[2] + 1, 8));
    const int bb = ns.bc_bot, bt = ns.bc_top;
    const unsigned iter = (unsigned)r->iter;
    const Float dp_dz = fabs(ns.rho_f * d.params.g[2] * d.grid.L[2] / d.grid.num[2]);
    auto ghost = [&](Float *f) { launch3(grd, blk, [&] { setNSghostNodes<Float>(f, bb, bt); }); };
    auto ghost3 = [&](Float3 *f) { launch3(grd, blk, [&] { setNSghostNodes<Float3>(f, bb, bt); }); };
    auto ghostf = [&](Float *x, Float *y, Float *z) {
        launch3(grdf, blk, [&] { setNSghostNodesFace<Float>(x, y, z, bb, bt); });
    };
    launch3(grd, blk, [&] {
        findPorositiesVelocitiesDiametersSpherical(d.dev_cellStart, d.dev_cellEnd, d.dev_x_sorted,
                                                   d.dev_vel_sorted, d.dev_ns_phi, d.dev_ns_dphi,
                                                   d.dev_ns_vp_avg, d.dev_ns_d_avg, iter, np, ns.c_phi);
    });
    if (iter == 0) {
        ghost3(d.dev_ns_v);
        launch3(grdf, blk, [&] { interpolateCenterToFace(d.dev_ns_v, d.dev_ns_v_x, d.dev_ns_v_y, d.dev_ns_v_z); });
    }
    ghostf(d.dev_ns_v_x, d.dev_ns_v_y, d.dev_ns_v_z);
    launch3(grdf, blk, [&] {
        findFaceDivTau(d.dev_ns_v_x, d.dev_ns_v_y, d.dev_ns_v_z, ns.mu, d.dev_ns_div_tau_x,
                       d.dev_ns_div_tau_y, d.dev_ns_div_tau_z);
    });
    ghostf(d.dev_ns_div_tau_x, d.dev_ns_div_tau_y, d.dev_ns_div_tau_z);
    ghost(d.dev_ns_p);
    ghost(d.dev_ns_phi);
    if (np > 0) {
        launch(bpg, tpb, [&] {
            findInteractionForce(d.dev_x, d.dev_vel, d.dev_ns_phi, d.dev_ns_p, d.dev_ns_v_x, d.dev_ns_v_y,
                                 d.dev_ns_v_z, d.dev_ns_div_tau_x, d.dev_ns_div_tau_y, d.dev_ns_div_tau_z,
                                 ns.mu, ns.rho_f, d.dev_ns_f_pf, d.dev_force, d.dev_ns_f_d, d.dev_ns_f_p,
                                 d.dev_ns_f_v, d.dev_ns_f_sum);
        });
        ghost(d.dev_ns_p);
        launch3(grd, blk, [&] {
            applyInteractionForceToFluid(d.dev_gridParticleIndex, d.dev_cellStart, d.dev_cellEnd,
                                         d.dev_ns_f_pf, d.dev_ns_F_pf);
        });
        ghost3(d.dev_ns_F_pf);
    }
    if ((r->iter % ns.ndem) != 0) return;
    Float pressure = ns.p[d.idx(0, 0, ns.nz - 1)];
    Float epsilon_value = pressure - ns.beta * pressure;
    launch3(grd, blk, [&] { setNSepsilonTop(d.dev_ns_epsilon, d.dev_ns_epsilon_new, epsilon_value); });
    if (d.walls.nw > 0 && (d.walls.wmode[0] == 1 || d.walls.wmode[0] == 3)) {
        r->wall0_iz = d.walls.nx->w / (d.grid.L[2] / d.grid.num[2]);
        launch3(grd, blk, [&] {
            setNSepsilonAtTopWall(d.dev_ns_epsilon, d.dev_ns_epsilon_new, r->wall0_iz, epsilon_value, dp_dz);
        });
    }
    const unsigned wall0_iz = r->wall0_iz;
    if ((ns.p_mod_A > 1.0e-5 || ns.p_mod_A < -1.0e-5) && ns.p_mod_f > 1.0e-7) {
        Float new_pressure = ns.p[d.idx(0, 0, ns.nz - 1)] +
                             ns.p_mod_A * sin(2.0 * M_PI * ns.p_mod_f * d.time.current + ns.p_mod_phi);
        launch3(grd, blk, [&] {
            setUpperPressureNS(d.dev_ns_p, d.dev_ns_epsilon, d.dev_ns_epsilon_new, ns.beta, new_pressure);
        });
    }
    ghost(d.dev_ns_p);
    ghostf(d.dev_ns_v_p_x, d.dev_ns_v_p_y, d.dev_ns_v_p_z);
    ghost(d.dev_ns_phi);
    ghost(d.dev_ns_dphi);
    launch3(grd, blk, [&] { interpolateFaceToCenter(d.dev_ns_v_x, d.dev_ns_v_y, d.dev_ns_v_z, d.dev_ns_v); });
    ghost3(d.dev_ns_v);
    launch3(grd, blk, [&] { findNSdivphiviv(d.dev_ns_phi, d.dev_ns_v, d.dev_ns_div_phi_vi_v); });
    ghost3(d.dev_ns_div_phi_vi_v);
    launch3(grdf, blk, [&] {
        findPredNSvelocities(d.dev_ns_p, d.dev_ns_v_x, d.dev_ns_v_y, d.dev_ns_v_z, d.dev_ns_phi, d.dev_ns_dphi,
                             d.dev_ns_div_tau_x, d.dev_ns_div_tau_y, d.dev_ns_div_tau_z,
                             d.dev_ns_div_phi_vi_v, bb, bt, ns.beta, d.dev_ns_F_pf, ns.ndem, wall0_iz,
                             ns.c_v, ns.mu, ns.rho_f, d.dev_ns_v_p_x, d.dev_ns_v_p_y, d.dev_ns_v_p_z);
    });
    ghostf(d.dev_ns_v_p_x, d.dev_ns_v_p_y, d.dev_ns_v_p_z);
    launch3(grd, blk, [&] { interpolateFaceToCenter(d.dev_ns_v_p_x, d.dev_ns_v_p_y, d.dev_ns_v_p_z, d.dev_ns_v_p); });
    if (iter == 0) {
        pressure = ns.p[d.idx(2, 2, 2)];
        epsilon_value = pressure - ns.beta * pressure;
        launch3(grd, blk, [&] { setNSepsilonInterior(d.dev_ns_epsilon, epsilon_value); });
        launch3(grd, blk, [&] { setNSnormZero(d.dev_ns_norm); });
        pressure = ns.p[d.idx(0, 0, 0)];
        epsilon_value = pressure - ns.beta * pressure;
        launch3(grd, blk, [&] { setNSepsilonBottom(d.dev_ns_epsilon, d.dev_ns_epsilon_new, epsilon_value); });
        ghost(d.dev_ns_epsilon);
    }
    double max_norm_res = 0.0;
    long done = -1;
    int conv = 0;
    for (unsigned int nijac = 0; nijac < ns.maxiter; ++nijac) {
        launch3(grd, blk, [&] {
            findNSforcing(d.dev_ns_epsilon, d.dev_ns_phi, d.dev_ns_dphi, d.dev_ns_v_p, d.dev_ns_v_p_x,
                          d.dev_ns_v_p_y, d.dev_ns_v_p_z, nijac, ns.ndem, ns.c_v, ns.rho_f, d.dev_ns_f1,
                          d.dev_ns_f2, d.dev_ns_f);
        });
        ghost(d.dev_ns_epsilon);
        launch3(grd, blk, [&] {
            jacobiIterationNS(d.dev_ns_epsilon, d.dev_ns_epsilon_new, d.dev_ns_norm, d.dev_ns_f, bb, bt,
                              ns.theta, wall0_iz, dp_dz);
        });
        launch3(grd, blk, [&] { copyValues<Float>(d.dev_ns_epsilon_new, d.dev_ns_epsilon); });
        done = nijac;
        if (nijac % nijacnorm == 0) {
            d.transferNSnormFromGlobalDeviceMemory();
            max_norm_res = d.maxNormResNS();
        }
        if (max_norm_res < ns.tolerance) {
            conv = 1;
            ghost(d.dev_ns_epsilon);
            if (ns.gamma > 0.0) {
                launch3(grd, blk, [&] { smoothing<Float>(d.dev_ns_epsilon, ns.gamma, bb, bt); });
                ghost(d.dev_ns_epsilon);
            }
            break;
        }
    }
    r->nijac_last = done;
    r->nijac_total += done + 1;
    r->ns_converged = conv;
    launch3(grd, blk, [&] { updateNSpressure(d.dev_ns_epsilon, ns.beta, d.dev_ns_p); });
    launch3(grdf, blk, [&] {
        updateNSvelocity(d.dev_ns_v_p_x, d.dev_ns_v_p_y, d.dev_ns_v_p_z, d.dev_ns_phi, d.dev_ns_epsilon,
                         ns.beta, bb, bt, ns.ndem, ns.c_v, ns.rho_f, wall0_iz, iter, d.dev_ns_v_x,
                         d.dev_ns_v_y, d.dev_ns_v_z);
    });
    ghostf(d.dev_ns_v_p_x, d.dev_ns_v_p_y, d.dev_ns_v_p_z);
    launch3(grd, blk, [&] { interpolateFaceToCenter(d.dev_ns_v_x, d.dev_ns_v_y, d.dev_ns_v_z, d.dev_ns_v); });
}

static int ref_one_step(RefRun *r)
{
    DEM &d = *r->dem;
    unsigned np = d.np;
    unsigned tpb = 256, bpg = idiv_up(np, tpb);
    unsigned bpg_bonds = idiv_up(d.params.nb0, tpb);
    if (np > 0) {
        launch(bpg, tpb, [&] {
            calcParticleCellID(d.dev_gridParticleCellID, d.dev_gridParticleIndex, d.dev_x);
        });
        /* thrust::sort_by_key (device.cu:1082-1085): stable */
        std::vector<std::pair<unsigned, unsigned>> kv(np);
        for (unsigned i = 0; i < np; ++i) kv[i] = {d.dev_gridParticleCellID[i], d.dev_gridParticleIndex[i]};
        std::stable_sort(kv.begin(), kv.end(),
                         [](const std::pair<unsigned, unsigned> &a,
                            const std::pair<unsigned, unsigned> &b) { return a.first < b.first; });
        for (unsigned i = 0; i < np; ++i) {
            d.dev_gridParticleCellID[i] = kv[i].first;
            d.dev_gridParticleIndex[i] = kv[i].second;
        }
        std::memset(d.dev_cellStart, 0xff,
                    sizeof(unsigned) * d.grid.num[0] * d.grid.num[1] * d.grid.num[2]);
        launch(bpg, tpb, [&] {
            reorderArrays(d.dev_cellStart, d.dev_cellEnd, d.dev_gridParticleCellID,
                          d.dev_gridParticleIndex, d.dev_x, d.dev_vel, d.dev_angvel,
                          d.dev_x_sorted, d.dev_vel_sorted, d.dev_angvel_sorted);
        });
        if (d.params.contactmodel == 2 || d.params.contactmodel == 3) {
            launch(bpg, tpb, [&] {
                topology(d.dev_cellStart, d.dev_cellEnd, d.dev_gridParticleIndex,
                         d.dev_x_sorted, d.dev_contacts, d.dev_distmod);
            });
        }
        launch(bpg, tpb, [&] {
            interact(d.dev_gridParticleIndex, d.dev_cellStart, d.dev_cellEnd, d.dev_x,
                     d.dev_x_sorted, d.dev_vel_sorted, d.dev_angvel_sorted, d.dev_vel,
                     d.dev_angvel, d.dev_force, d.dev_torque, d.dev_es_dot,
                     d.dev_ev_dot, d.dev_es, d.dev_ev, d.dev_p, d.dev_walls_nx,
                     d.dev_walls_mvfd, d.dev_walls_force_pp, d.dev_contacts,
                     d.dev_distmod, d.dev_delta_t);
        });
        if (d.params.nb0 > 0) {
            launch(bpg_bonds, tpb, [&] {
                bondsLinear(d.dev_bonds, d.dev_bonds_delta, d.dev_bonds_omega, d.dev_x,
                            d.dev_vel, d.dev_angvel, d.dev_force, d.dev_torque);
            });
        }
    }
    if (d.fluid == 1 && d.cfd_solver == 1) ref_darcy(r);
    if (d.fluid == 1 && d.cfd_solver == 0) ref_ns(r);
    if (np > 0) {
        if (d.walls.nw > 0 && d.walls.wmode[0] == 3) {
            launch(bpg, tpb, [&] {
                findShearStressOnFixedMovingParticles(d.dev_x, d.dev_vel, d.dev_force,
                                                      d.dev_walls_tau_eff_x_pp);
            });
            ref_summation(d.dev_walls_tau_eff_x_pp, d.dev_walls_tau_eff_x_partial, np, bpg);
        }
        int change_velocity_state = 0;
        const Float velocity_factor = 10.0, v2_start = 10.0, v2_end = 15.0;
        if (d.time.current >= v2_start && d.time.current < v2_end && r->velocity_state == 1) {
            change_velocity_state = 1;
            r->velocity_state = 2;
        } else if (d.time.current >= v2_end && r->velocity_state == 2) {
            change_velocity_state = -1;
            r->velocity_state = 1;
        }
        launch(bpg, tpb, [&] {
            integrate(d.dev_x_sorted, d.dev_vel_sorted, d.dev_angvel_sorted, d.dev_x,
                      d.dev_vel, d.dev_angvel, d.dev_force, d.dev_torque, d.dev_angpos,
                      d.dev_acc, d.dev_angacc, d.dev_vel0, d.dev_angvel0, d.dev_xyzsum,
                      d.dev_gridParticleIndex, (unsigned)r->iter, d.dev_walls_wmode,
                      d.dev_walls_mvfd, d.dev_walls_tau_eff_x_partial,
                      d.dev_walls_tau_x, d.walls.nw ? d.walls.tau_x[0] : 0.0,
                      change_velocity_state, velocity_factor, bpg);
        });
        if (d.walls.nw > 0) {
            ref_summation(d.dev_walls_force_pp, d.dev_walls_force_partial, np, bpg);
            launch(1, d.walls.nw, [&] {
                integrateWalls(d.dev_walls_nx, d.dev_walls_mvfd, d.dev_walls_wmode,
                               d.dev_walls_force_partial, d.dev_walls_acc, bpg,
                               d.time.current, (unsigned)r->iter);
            });
        }
    }
    d.time.current += d.time.dt;
    r->filetimeclock += d.time.dt;
    ++r->iter;
    return 0;
}

extern "C" {

void *ref_open(const char *path, int fluid)
{
    /* DEM(inputbin, verbosity, checkVals, dry, initCuda, transferConstMem,
     *     fluidFlow, device) -- sphere.h */
    DEM *d = new DEM(std::string(path), 0, 1, 0, 1, 1, fluid, 0);
    RefRun *r = new RefRun{d, 0, 1, 10000000u, 0, 0, 0.0, 0};
    if (fluid && d->cfd_solver == 0) {
        // deterministic ghost nodes (the reference copies them from
        // uninitialised host memory)
        unsigned nx = d->grid.num[0], ny = d->grid.num[1], nz = d->grid.num[2];
        for (int z = -1; z <= (int)nz; ++z)
            for (int y = -1; y <= (int)ny; ++y)
                for (int x = -1; x <= (int)nx; ++x) {
                    bool ghost = x < 0 || y < 0 || z < 0 || x == (int)nx || y == (int)ny || z == (int)nz;
                    if (!ghost) continue;
                    unsigned i = d->idx(x, y, z);
                    d->dev_ns_p[i] = 0.0;
                    d->dev_ns_phi[i] = 0.0;
                    d->dev_ns_dphi[i] = 0.0;
                    d->dev_ns_v[i] = make_double3(0.0, 0.0, 0.0);
                }
    }
    if (fluid && d->cfd_solver == 1) {
        // deterministic ghost cells (the reference leaves them uninitialised)
        unsigned nx = d->grid.num[0], ny = d->grid.num[1], nz = d->grid.num[2];
        for (int z = -1; z <= (int)nz; ++z)
            for (int y = -1; y <= (int)ny; ++y)
                for (int x = -1; x <= (int)nx; ++x) {
                    bool ghost = x < 0 || y < 0 || z < 0 || x == (int)nx || y == (int)ny || z == (int)nz;
                    if (!ghost) continue;
                    unsigned i = d->d_idx(x, y, z);
                    d->dev_darcy_p[i] = 0.0;
                    d->dev_darcy_phi[i] = 0.0;
                    d->dev_darcy_dphi[i] = 0.0;
                    d->dev_darcy_p_constant[i] = 0;
                }
        // device.cu:1017-1020
        d->darcy.p_top_orig = d->darcy.p[d->d_idx(0, 0, d->darcy.nz - 1)] -
                              d->darcy.p_mod_A * sin(2.0 * M_PI * d->darcy.p_mod_f * d->time.current +
                                                     d->darcy.p_mod_phi);
    }
    return r;
}

int ref_step(void *h, long n)
{
    RefRun *r = (RefRun *)h;
    for (long i = 0; i < n; ++i) {
        r->dem->transferToConstantDeviceMemory();
        int rc = ref_one_step(r);
        if (rc) return rc;
    }
    return 0;
}

int ref_write(void *h, const char *path)
{
    RefRun *r = (RefRun *)h;
    DEM &d = *r->dem;
    if (d.fluid == 1 && d.cfd_solver == 0) {
        /* device.cu:2586-2593 */
        dim3 blk(8, 8, 8);
        dim3 grd(idiv_up(d.grid.num[0], 8), idiv_up(d.grid.num[1], 8), idiv_up(d.grid.num[2], 8));
        launch3(grd, blk, [&] { interpolateFaceToCenter(d.dev_ns_v_x, d.dev_ns_v_y, d.dev_ns_v_z, d.dev_ns_v); });
    }
    r->dem->transferFromGlobalDeviceMemory();
    r->dem->writebin(path);
    /* a file output restarts the file clock (device.cu:2556-2600) */
    r->filetimeclock = 0.0;
    return 0;
}

long ref_get(void *h, const char *name, void *dst, size_t bytes)
{
    RefRun *r = (RefRun *)h;
    DEM &d = *r->dem;
    const void *src = nullptr;
    size_t need = 0;
    size_t np = d.np, slots = (size_t)d.np * NC;
    std::string n(name);
    if (n == "x") { src = d.dev_x; need = np * 32; }
    else if (n == "vel") { src = d.dev_vel; need = np * 32; }
    else if (n == "angvel") { src = d.dev_angvel; need = np * 32; }
    else if (n == "angpos") { src = d.dev_angpos; need = np * 32; }
    else if (n == "force") { src = d.dev_force; need = np * 32; }
    else if (n == "torque") { src = d.dev_torque; need = np * 32; }
    else if (n == "acc") { src = d.dev_acc; need = np * 32; }
    else if (n == "angacc") { src = d.dev_angacc; need = np * 32; }
    else if (n == "xyzsum") { src = d.dev_xyzsum; need = np * 32; }
    else if (n == "es_dot") { src = d.dev_es_dot; need = np * 8; }
    else if (n == "es") { src = d.dev_es; need = np * 8; }
    else if (n == "ev_dot") { src = d.dev_ev_dot; need = np * 8; }
    else if (n == "ev") { src = d.dev_ev; need = np * 8; }
    else if (n == "p") { src = d.dev_p; need = np * 8; }
    else if (n == "cellid") { src = d.dev_gridParticleCellID; need = np * 4; }
    else if (n == "index") { src = d.dev_gridParticleIndex; need = np * 4; }
    else if (n == "contacts") { src = d.dev_contacts; need = slots * 4; }
    else if (n == "delta_t") { src = d.dev_delta_t; need = slots * 32; }
    else if (n == "distmod") { src = d.dev_distmod; need = slots * 32; }
    else if (n == "walls_nx") { src = d.dev_walls_nx; need = d.walls.nw * 32; }
    else if (n == "walls_mvfd") { src = d.dev_walls_mvfd; need = d.walls.nw * 32; }
    else if (n == "cellstart") {
        src = d.dev_cellStart; need = 4 * (size_t)d.grid.num[0] * d.grid.num[1] * d.grid.num[2];
    } else if (n == "bonds") { src = d.dev_bonds; need = 8 * (size_t)d.params.nb0; }
    else if (n == "bonds_delta") { src = d.dev_bonds_delta; need = 32 * (size_t)d.params.nb0; }
    else if (n == "bonds_omega") { src = d.dev_bonds_omega; need = 32 * (size_t)d.params.nb0; }
    else if (n.rfind("darcy_", 0) == 0 && d.fluid == 1) {
        unsigned nx = d.grid.num[0], ny = d.grid.num[1], nz = d.grid.num[2];
        size_t nc = (size_t)nx * ny * nz;
        static thread_local std::vector<double> buf;
        if (n == "darcy_nijac_last" || n == "darcy_nijac_total") {
            static thread_local long v;
            v = n == "darcy_nijac_last" ? r->nijac_last : r->nijac_total;
            src = &v; need = 8;
        } else if (n == "darcy_f_p") {
            src = d.dev_darcy_f_p; need = (size_t)np * 32;
        } else {
            const double *f = nullptr;
            int comps = 1;
            if (n == "darcy_p") f = d.dev_darcy_p;
            else if (n == "darcy_phi") f = d.dev_darcy_phi;
            else if (n == "darcy_dphi") f = d.dev_darcy_dphi;
            else if (n == "darcy_k") f = d.dev_darcy_k;
            else if (n == "darcy_norm") f = d.dev_darcy_norm;
            else if (n == "darcy_v") { f = (const double *)d.dev_darcy_v; comps = 3; }
            else if (n == "darcy_vp_avg") { f = (const double *)d.dev_darcy_vp_avg; comps = 3; }
            else return -1;
            buf.assign(nc * comps, 0.0);
            for (unsigned z = 0; z < nz; ++z)
                for (unsigned y = 0; y < ny; ++y)
                    for (unsigned x = 0; x < nx; ++x)
                        for (int c = 0; c < comps; ++c)
                            buf[((size_t)(z * ny + y) * nx + x) * comps + c] =
                                f[(size_t)d.d_idx(x, y, z) * comps + c];
            src = buf.data(); need = buf.size() * 8;
        }
    }
    else if (n.rfind("ns_", 0) == 0 && d.fluid == 1 && d.cfd_solver == 0) {
        unsigned nx = d.grid.num[0], ny = d.grid.num[1], nz = d.grid.num[2];
        size_t nc = (size_t)nx * ny * nz;
        static thread_local std::vector<double> buf;
        static thread_local long v;
        if (n == "ns_nijac_last" || n == "ns_nijac_total" || n == "ns_converged") {
            v = n == "ns_nijac_last" ? r->nijac_last : n == "ns_nijac_total" ? r->nijac_total : r->ns_converged;
            src = &v; need = 8;
        } else if (n == "ns_f_d" || n == "ns_f_p" || n == "ns_f_v" || n == "ns_f_sum") {
            src = n == "ns_f_d" ? d.dev_ns_f_d : n == "ns_f_p" ? d.dev_ns_f_p
                  : n == "ns_f_v" ? d.dev_ns_f_v : d.dev_ns_f_sum;
            need = (size_t)np * 32;
        } else if (n == "ns_v_face") {
            size_t nf = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
            buf.assign(nf * 3, 0.0);
            size_t q = 0;
            for (unsigned z = 0; z <= nz; ++z)
                for (unsigned y = 0; y <= ny; ++y)
                    for (unsigned x = 0; x <= nx; ++x, ++q) {
                        unsigned f = d.vidx(x, y, z);
                        buf[3 * q] = d.dev_ns_v_x[f];
                        buf[3 * q + 1] = d.dev_ns_v_y[f];
                        buf[3 * q + 2] = d.dev_ns_v_z[f];
                    }
            src = buf.data(); need = buf.size() * 8;
        } else {
            const double *f = nullptr;
            int comps = 1;
            if (n == "ns_p") f = d.dev_ns_p;
            else if (n == "ns_phi") f = d.dev_ns_phi;
            else if (n == "ns_dphi") f = d.dev_ns_dphi;
            else if (n == "ns_epsilon") f = d.dev_ns_epsilon;
            else if (n == "ns_norm") f = d.dev_ns_norm;
            else if (n == "ns_v") { f = (const double *)d.dev_ns_v; comps = 3; }
            else if (n == "ns_F_pf") { f = (const double *)d.dev_ns_F_pf; comps = 3; }
            else return -1;
            buf.assign(nc * comps, 0.0);
            for (unsigned z = 0; z < nz; ++z)
                for (unsigned y = 0; y < ny; ++y)
                    for (unsigned x = 0; x < nx; ++x)
                        for (int c = 0; c < comps; ++c)
                            buf[((size_t)(z * ny + y) * nx + x) * comps + c] =
                                f[(size_t)d.idx(x, y, z) * comps + c];
            src = buf.data(); need = buf.size() * 8;
        }
    }
    else return -1;
    if (!dst || bytes < need) return (long)need;
    std::memcpy(dst, src, need);
    return 0;
}

/* DEM::porosity (sphere.cpp:487-605) on the current state.  It prints
 * "z\tporosity" lines; they are read back at full precision.  Returns the
 * number of lines parsed.  The caller keeps z_slices valid: the reference
 * exits on a slice height below twice the last radius. */
long ref_porosity(void *h, int z_slices, double *z_pos, double *porosity)
{
    RefRun *r = (RefRun *)h;
    r->dem->transferFromGlobalDeviceMemory();
    std::ostringstream text;
    std::streambuf *old = std::cout.rdbuf(text.rdbuf());
    std::streamsize prec = std::cout.precision(17);
    r->dem->porosity(z_slices);
    std::cout.precision(prec);
    std::cout.rdbuf(old);
    std::istringstream in(text.str());
    long n = 0;
    double z, p;
    while (n < z_slices && in >> z >> p) {
        z_pos[n] = z;
        porosity[n] = p;
        ++n;
    }
    return n;
}

/* DEM::findOverlaps (sphere.cpp:677-725) on the current state: writes up
 * to cap pairs and separations, returns the number found. */
long ref_overlaps(void *h, unsigned *pairs, double *delta, long cap)
{
    RefRun *r = (RefRun *)h;
    r->dem->transferFromGlobalDeviceMemory();
    std::vector<std::vector<unsigned int>> ij;
    std::vector<Float> d;
    r->dem->findOverlaps(ij, d);
    for (long q = 0; q < (long)ij.size() && q < cap; ++q) {
        pairs[2 * q] = ij[q][0];
        pairs[2 * q + 1] = ij[q][1];
        delta[q] = d[q];
    }
    return (long)ij.size();
}

/* DEM::render and DEM::cameraInit (src/raytracer.cuh:278-520): the camera
 * from the grid and the largest particle coordinates, the rays of
 * rayInitPerspective, then rayIntersectSpheres (method 0) or
 * rayIntersectSpheresColormap with the method's per-particle values, each
 * kernel run one thread at a time.  img receives width * height RGBA bytes.
 * The kernels' bound checks let the thread with index width * height run;
 * the ray and image buffers carry one spare entry for it. */
int ref_render(void *h, int method, float maxval, float lower_cutoff, unsigned width,
               unsigned height, unsigned char *img)
{
    RefRun *r = (RefRun *)h;
    DEM &d = *r->dem;
    d.transferFromGlobalDeviceMemory();
    const unsigned np = d.np;
    const unsigned pixels = width * height;
    const unsigned tpb = 256, bpg = idiv_up(pixels, tpb);
    std::vector<unsigned char> dev_img(4 * ((size_t)pixels + 1), 0);
    std::vector<float4> ray_o((size_t)pixels + 1), ray_d((size_t)pixels + 1);
    launch(bpg, tpb, [&] { imageInit(dev_img.data(), pixels); });
    /* DEM::render */
    const float imgw = d.grid.L[0] * 1.35f;
    const Float3 maxpos = d.maxPos();
    const float3 lookat = make_float3(maxpos.x, maxpos.y, maxpos.z) / 2.0f;
    const float3 eye = make_float3(d.grid.L[0] * 2.3f, d.grid.L[1] * -5.0f, d.grid.L[2] * 1.3f);
    /* DEM::cameraInit */
    {
        const float hw_ratio = height / width;
        const float4 imgplane = make_float4(-0.5f * imgw, 0.5f * imgw, -0.5f * imgw * hw_ratio,
                                            0.5f * imgw * hw_ratio);
        const float3 view = eye - lookat;
        const float3 up = make_float3(0.0f, 0.0f, 1.0f);
        const float3 w = -view / length(view);
        const float3 u = cross(up, w) / length(cross(up, w));
        const float3 v = cross(w, u);
        const float dd = length(view) * 0.8f;
        const float3 light = normalize(-1.0f * eye * make_float3(1.0f, 0.2f, 0.6f));
        devC_u = u;
        devC_v = v;
        devC_w = w;
        devC_eye = eye;
        devC_imgplane = imgplane;
        devC_d = dd;
        devC_light = light;
        devC_pixels = pixels;
    }
    devC_np = np;
    launch(bpg, tpb, [&] {
        rayInitPerspective(ray_o.data(), ray_d.data(), make_float4(eye.x, eye.y, eye.z, 0.0f),
                           width, height);
    });
    if (method == 0) {
        launch(bpg, tpb, [&] { rayIntersectSpheres(ray_o.data(), ray_d.data(), d.dev_x, dev_img.data()); });
    } else {
        std::vector<Float> linarr(np ? np : 1);
        const Float *vals = linarr.data();
        for (unsigned i = 0; i < np; ++i) {
            const Float4 &ve = d.k.vel[i], &w = d.k.angvel[i], &xs = d.k.xyzsum[i], &ap = d.k.angpos[i];
            if (method == 2) linarr[i] = sqrt(ve.x * ve.x + ve.y * ve.y + ve.z * ve.z);
            else if (method == 3) linarr[i] = sqrt(w.x * w.x + w.y * w.y + w.z * w.z);
            else if (method == 4) linarr[i] = xs.x;
            else if (method == 5) linarr[i] = sqrt(ap.x * ap.x + ap.y * ap.y + ap.z * ap.z);
        }
        if (method == 1) vals = d.dev_p;
        else if (method < 1 || method > 5) return -1;
        launch(bpg, tpb, [&] {
            rayIntersectSpheresColormap(ray_o.data(), ray_d.data(), d.dev_x, d.dev_vel, vals, maxval,
                                        lower_cutoff, dev_img.data());
        });
    }
    std::memcpy(img, dev_img.data(), 4 * (size_t)pixels);
    return 0;
}

void ref_close(void *h)
{
    RefRun *r = (RefRun *)h;
    delete r->dem;
    delete r;
}

}  /* extern "C" */
