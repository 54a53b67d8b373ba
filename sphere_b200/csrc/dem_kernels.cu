// DEM step kernels, FP64 (faithful and true-FP64 lengths).
//
// Compiled with -fmad=false: every expression keeps the reference's
// operation order and rounding (the reference is built with --fmad=false,
// src/CMakeLists.txt:25).  One thread per particle in sorted order.
#include "dem_device.cuh"
#include "contacts_staged.cuh"
#include "dem_launch.h"
#include "reduce_device.cuh"

namespace sphb {

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
    __shared__ double stage[2048];
    __shared__ bool last;
    if (S.ctl->err) return;
    double s = block_tree_sum(S.tau_pp, P.np, P.nblocks256, cache);
    if (threadIdx.x == 0) {
        S.tau_partials[blockIdx.x] = s;
        __threadfence();
        last = atomicAdd(&S.ctl->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double tau = 0.0;
    tau = ordered_sum(S.tau_partials, P.nblocks256, stage);
    if (threadIdx.x == 0) {
        S.ctl->tau_eff_x = tau;
        S.ctl->ticket = 0;
    }
}

// ---------------------------------------------------------------------
// integrate, src/integration.cuh:14-305 (TY3 default, TY2 selectable),
// then the cell hash of the new position (src/sorting.cuh:7-51) so the
// next step knows whether the sort changes.
// ---------------------------------------------------------------------
// integrate (src/integration.cuh:14-305) of the 256 sorted particles of
// this block, then the wall reduction and wall update
// (integration.cuh:309-450): block j forms the reference's partial sum j
// (256 consecutive ORIGINAL indices, same tree), the block that finishes
// last adds the partials in block order, moves the walls and advances the
// loop counters (device.cu:2543-2545).  Launched with the reference's
// ceil(np / 256) blocks (one block when np == 0).
// Resident 256-thread blocks per SM of the integration kernel: 3 caps it at
// 80 registers, so 1e5 particles integrate in one wave (measured 68 -> 61 us
// per shear step against the uncapped 102 registers and two waves).
#ifndef SPHB_INTEGRATE_MINB
#define SPHB_INTEGRATE_MINB 3
#endif
__global__ void __launch_bounds__(256, SPHB_INTEGRATE_MINB) k_integrate(DevParams P, DevState S)
{
    __shared__ double cache[256];
    __shared__ bool last;
    DevCtl *ctl = S.ctl;
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = ctl->err == 0;
    StepClock clk;
    clk.iter = ctl->iter;
    clk.t_current = ctl->t_current;
    clk.velocity_state = ctl->velocity_state;
    clk.tau_eff_x = ctl->tau_eff_x;
    if (ok && k < P.np)
        integrate_particle(P, S, k, S.force[k], S.torque[k], clk, S.x, S.vel, S.angvel, S.vel_f,
                           S.angvel_f, &ctl->resort, &ctl->nl_rebuild);
    if (P.nw > 0 && P.np > 0) {
        double s = chunk_tree_sum(S.walls_force_pp, P.np, blockIdx.x, cache);
        if (threadIdx.x == 0) S.partials[blockIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&ctl->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // every wall sums the same (wall-0) partials, as the reference does
    double wforce = (P.nw > 0 && P.np > 0) ? ordered_sum<256>(S.partials, P.nblocks256, cache) : 0.0;
    if (threadIdx.x != 0) return;
    ctl->ticket = 0;
    if (!ok || *(volatile int *)&ctl->err) return;
    walls_integrate(P, S, wforce, clk.iter, clk.t_current);
    ctl->velocity_state = next_velocity_state(clk.velocity_state, clk.t_current);
    ctl->t_current = clk.t_current + P.dt;
    ctl->iter = clk.iter + 1;
}

// The rest of a DEM step whose particles k_contacts_integrate advanced: the
// wall reduction and wall update of k_integrate in the same arithmetic.
// Warp j forms the tree sum of chunk j (the reference's partial of block j,
// warp_chunk_tree_sum) and counts itself done (DevCtl::ticket); the warp
// that counts last adds the partials in chunk order, moves the walls,
// advances the loop counters and publishes the cell / list flags of the next
// step (finish_step).  One warp per 256-index chunk, SPHB_WALLS_WARPS warps
// per block, no block barrier.
#ifndef SPHB_WALLS_WARPS
#define SPHB_WALLS_WARPS 8
#endif
__global__ void __launch_bounds__(32 * SPHB_WALLS_WARPS) k_walls_step(DevParams P, DevState S)
{
    DevCtl *ctl = S.ctl;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const unsigned nchunks = P.np > 0 ? P.nblocks256 : 1;
    if (j >= nchunks) return;   // whole warps
    if (P.nw > 0 && P.np > 0) {
        const double part = warp_chunk_tree_sum(S.walls_force_pp, P.np, j);
        if (lane == 0) S.partials[j] = part;
    }
    int last = 0;
    if (lane == 0) {
        __threadfence();
        last = atomicAdd(&ctl->ticket, 1u) == nchunks - 1;
    }
    if (!__shfl_sync(0xffffffffu, last, 0)) return;
    __threadfence();
    finish_step(P, S);
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

// New positions (and radii) from the host, in ORIGINAL order, into the
// sorted storage.  Each particle's cell is hashed (src/sorting.cuh:7-51) and
// DevCtl::resort raised when it changed, DevCtl::nl_rebuild when the
// particle left 0.45 skin of its position at the list build or its radius
// changed -- the conditions under which the integration raises them -- so
// the next step's k_resort sorts and rebuilds exactly when a forced sort
// would have changed something (a stable sort of unchanged cells is the
// identity).
__global__ void k_set_positions(DevParams P, DevState S, const double4 *src)
{
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P.np) return;
    const unsigned o = S.orig_of[k];
    const double4 xo = S.x[k], xn = src[o];
    int ix, iy, iz;
    if (!cell_coord(P, xn.x, 0, ix) || !cell_coord(P, xn.y, 1, iy) || !cell_coord(P, xn.z, 2, iz)) {
        raise_err(S.ctl, DERR_OUTSIDE, (int)o);
        return;
    }
    const unsigned c = ((unsigned)iz * P.num[1]) * P.num[0] + (unsigned)iy * P.num[0] + (unsigned)ix;
    S.x[k] = xn;
    S.cell_new[k] = c;
    if (c != S.cell_of[k]) S.ctl->resort = 1;
    const float4 xr = S.x_ref[k];
    const double ddx = xn.x - (double)xr.x, ddy = xn.y - (double)xr.y, ddz = xn.z - (double)xr.z;
    const double lim = 0.45 * P.skin;
    if (xn.w != xo.w || ddx * ddx + ddy * ddy + ddz * ddz > lim * lim) S.ctl->nl_rebuild = 1;
}

// ---------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------
static inline unsigned blocks_for(unsigned n, unsigned b) { return (n + b - 1) / b; }

// SPHB_STAGED_MINB resident blocks per SM: each block's dynamic shared memory
// leaves room for the others (228 KB per SM, 1 KB reserved per block, and the
// block's static shared memory), at most 227 KB per block.
void staged_contact_shape(unsigned nc, size_t per_particle, size_t &smem, unsigned &cap)
{
    size_t budget = 233472 / SPHB_STAGED_MINB - 1024 - 512;
    if (budget > 232448 - 512) budget = 232448 - 512;
    const size_t fixed = stage_smem_bytes(nc, SPHB_STAGED_B, 0, per_particle);
    if (!SPHB_STAGED_ON) {
        cap = 0;
        smem = fixed;
        return;
    }
    cap = fixed + 256 * per_particle > budget ? 256u : (unsigned)((budget - fixed) / per_particle);
    smem = stage_smem_bytes(nc, SPHB_STAGED_B, cap, per_particle);
}

cudaError_t launch_contacts(const DevParams &P, const DevState &S, int prec, cudaStream_t st,
                            int staged)
{
    if (P.np == 0) return cudaSuccess;
    if (P.contactmodel == 2 && staged) {
        size_t smem;
        unsigned cap;
        staged_contact_shape(P.nc, stage_bytes_per_particle<0>(), smem, cap);
        static size_t attr = 0;
        if (attr < smem) {
            cudaFuncSetAttribute(k_contacts_staged<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            cudaFuncSetAttribute(k_contacts_staged<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            attr = smem;
        }
        dim3 grid(blocks_for(P.np, SPHB_STAGED_B));
        if (prec == 0) k_contacts_staged<0><<<grid, SPHB_STAGED_B, smem, st>>>(P, S, cap);
        else k_contacts_staged<1><<<grid, SPHB_STAGED_B, smem, st>>>(P, S, cap);
        return cudaGetLastError();
    }
    const unsigned B = SPHB_CONTACT_B;
    dim3 grid(blocks_for(P.np, B));
    if (P.contactmodel == 2) {
        size_t smem = (size_t)B * P.nc * sizeof(uint32_t);
        static bool attr = false;
        if (!attr) {
            int mx = (int)((size_t)B * 64 * sizeof(uint32_t));
            cudaFuncSetAttribute(k_contacts<0, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
            cudaFuncSetAttribute(k_contacts<1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
            attr = true;
        }
        if (prec == 0) k_contacts<0, 2><<<grid, B, smem, st>>>(P, S);
        else k_contacts<1, 2><<<grid, B, smem, st>>>(P, S);
    } else {
        if (prec == 0) k_contacts<0, 1><<<grid, B, 0, st>>>(P, S);
        else k_contacts<1, 1><<<grid, B, 0, st>>>(P, S);
    }
    return cudaGetLastError();
}

cudaError_t launch_contacts_integrate(const DevParams &P, const DevState &S, int prec,
                                      cudaStream_t st)
{
    if (P.np == 0) return cudaSuccess;
    const unsigned B = SPHB_CONTACT_B;
    dim3 grid(blocks_for(P.np, B));
    if (P.contactmodel == 2) {
        size_t smem = (size_t)B * P.nc * sizeof(uint32_t);
        static bool attr = false;
        if (!attr) {
            int mx = (int)((size_t)B * 64 * sizeof(uint32_t));
            cudaFuncSetAttribute(k_contacts_integrate<0, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
            cudaFuncSetAttribute(k_contacts_integrate<1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
            attr = true;
        }
        if (prec == 0) k_contacts_integrate<0, 2><<<grid, B, smem, st>>>(P, S);
        else k_contacts_integrate<1, 2><<<grid, B, smem, st>>>(P, S);
    } else {
        if (prec == 0) k_contacts_integrate<0, 1><<<grid, B, 0, st>>>(P, S);
        else k_contacts_integrate<1, 1><<<grid, B, 0, st>>>(P, S);
    }
    return cudaGetLastError();
}

cudaError_t launch_walls_step(const DevParams &P, const DevState &S, cudaStream_t st)
{
    const unsigned chunks = P.np > 0 ? P.nblocks256 : 1;
    k_walls_step<<<blocks_for(chunks, SPHB_WALLS_WARPS), 32 * SPHB_WALLS_WARPS, 0, st>>>(P, S);
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
    }
    k_integrate<<<P.np > 0 ? P.nblocks256 : 1, 256, 0, st>>>(P, S);
    return cudaGetLastError();
}

cudaError_t launch_occ_from_rows(const DevParams &P, const DevState &S, cudaStream_t st)
{
    if (P.np == 0) return cudaSuccess;
    k_occ_from_rows<<<blocks_for(P.np, 256), 256, 0, st>>>(P, S);
    return cudaGetLastError();
}

cudaError_t launch_set_positions(const DevParams &P, const DevState &S, const double4 *src,
                                 cudaStream_t st)
{
    if (P.np == 0) return cudaSuccess;
    k_set_positions<<<blocks_for(P.np, 256), 256, 0, st>>>(P, S, src);
    return cudaGetLastError();
}

cudaError_t launch_hash(const DevParams &P, const DevState &S, cudaStream_t st)
{
    if (P.np == 0) return cudaSuccess;
    k_hash<<<blocks_for(P.np, 256), 256, 0, st>>>(P, S);
    return cudaGetLastError();
}

}  // namespace sphb
