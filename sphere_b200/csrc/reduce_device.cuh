// Wall-force reductions and the wall update, shared by the per-stage
// kernels and the persistent step kernel.
#pragma once

#include "dem_state.h"

namespace sphb {

// summation, src/integration.cuh:309-341, for block j of the reference's
// launch: the tree sum over the 256 consecutive ORIGINAL indices
// [256 j, 256 j + 256) exactly as the reference's block j forms it, done by
// a block of any power-of-two size.  cache holds 256 doubles.
__device__ __forceinline__ double chunk_tree_sum(const double *in, unsigned np, unsigned j,
                                                 double *cache)
{
    for (unsigned e = threadIdx.x; e < 256; e += blockDim.x) {
        unsigned idx = e + j * 256;
        double temp = 0.0f;
        if (idx < np) temp += __ldcg(in + idx);
        cache[e] = temp;
    }
    __syncthreads();
    for (unsigned i = 128; i != 0; i /= 2) {
        for (unsigned e = threadIdx.x; e < i; e += blockDim.x) cache[e] += cache[e + i];
        __syncthreads();
    }
    double r = cache[0];
    __syncthreads();
    return r;
}

// Adds in[0..n) in index order (the reference's serial loop over block
// partials, integration.cuh:67-68, 376-378).  All threads of the calling
// block stage chunks of CHUNK values in shared memory (stage holds CHUNK
// doubles); thread 0 adds them one by one.  The result is valid in thread 0.
template <unsigned CHUNK = 2048>
__device__ __forceinline__ double ordered_sum(const double *in, unsigned n, double *stage)
{
    double acc = 0.0;
    for (unsigned base = 0; base < n; base += CHUNK) {
        unsigned m = min(CHUNK, n - base);
        __syncthreads();
        for (unsigned i = threadIdx.x; i < m; i += blockDim.x) stage[i] = __ldcg(in + base + i);
        __syncthreads();
        if (threadIdx.x == 0)
            for (unsigned i = 0; i < m; ++i) acc += stage[i];
    }
    __syncthreads();
    return acc;
}

// integrateWalls, src/integration.cuh:344-450, given the summed wall-0
// force (every wall uses it, as the reference does).  One thread.
__device__ __forceinline__ void walls_integrate(const DevParams &P, const DevState &S, double wforce,
                                                long long iter, double t_current)
{
    const double dt = P.dt;
    for (unsigned w = 0; w < P.nw; ++w) {
        double4 w_nx = S.wnx[w], w_mvfd = S.wmvfd[w];
        int wmode = P.wmode[w];
        if (wmode == 0) continue;
        double acc0 = iter == 0 ? 0.0 : S.wacc[w];
        w_mvfd.z = 0.0;
        w_mvfd.z += wforce;
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
}

// rate-state bookkeeping (device.cu:2461-2469): the velocity state after
// the step that started at t_current.
__device__ __forceinline__ int next_velocity_state(int vs, double t_current)
{
    if (t_current >= 10.0 && t_current < 15.0 && vs == 1) return 2;
    if (t_current >= 15.0 && vs == 2) return 1;
    return vs;
}

}  // namespace sphb
