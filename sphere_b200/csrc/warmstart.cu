// Learned warm start for the Darcy pressure solve: a 3-layer 3D convolution
// network (4 -> 16 -> 16 -> 1 channels, 3x3x3 kernels, ReLU) maps the
// previous pressure, the porosity, the porosity change of a fluid step and
// the previous solve's pressure change to the pressure change of the step's
// solve.  It is trained online on the
// solves the engine itself makes: after each solve the converged pressure
// is the target, one Adam step follows.
//
// Every convolution is an implicit GEMM on the tensor cores (tcgen05, BF16
// operands in shared memory, FP32 accumulators in TMEM):
//   forward / input gradient: D[128 cells x 16 out ch] = sum over the 27
//     taps of A_tap[128 cells x 16 in ch] * B_tap[16 x 16], A gathered from
//     the neighbour cells (zero outside the grid);
//   weight gradient: D[(tap, in ch) x 16 out ch] = sum over cells of
//     X_shifted^T * dY, split over blocks (deterministic partials, reduced
//     in a fixed order).
// Activations and gradients are stored BF16 channels-last (16 per cell, 32
// bytes); master weights, Adam moments and all reductions are FP32.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include <cuda_bf16.h>

#include "tc_sm100.cuh"
#include "warmstart.h"

namespace sphb {

namespace {

constexpr int kCh = 16;          // channels of every activation (inputs padded)
constexpr int kInputs = 4;       // p_prev, phi, dphi, previous pressure change
constexpr int kTaps = 27;
constexpr int kWElems = kTaps * kCh * kCh;   // weights per layer
constexpr int kTile = 128;       // cells per MMA tile (M)
constexpr int kRound = 9;        // taps gathered per round of the convolution
constexpr size_t kConvSmem = kRound * 4096 + kTaps * 512;
constexpr int kWChunk = 64;      // cells per K chunk of the weight gradient
constexpr size_t kWgradSmem = 16 * 4096 + 4 * 512;
constexpr unsigned kWaitLimit = 1u << 22;

using bf16 = __nv_bfloat16;

struct ConvArgs {
    int nx, ny, nz;
    unsigned ncells;
    const bf16 *in;        // [ncells][16]
    const bf16 *w;         // [27][16 out][16 in]
    const float *bias;     // [16]
    const bf16 *relu_ref;  // mode 2: activation whose ReLU mask gates the output
    bf16 *out_bf;          // modes 0, 2: [ncells][16]
    float *out_f;          // mode 1: [ncells] (channel 0)
    int *err;
};

// mode 0: out = ReLU(conv + bias) (BF16); mode 1: out channel 0 = conv +
// bias (FP32); mode 2: out = conv * [relu_ref > 0] (BF16, no bias).
//
// The 27 taps go through in three rounds of 9: the block gathers a round's
// shifted operand tiles into shared memory (36 KB), one thread issues their
// MMAs, and the round's commit frees the tiles for the next round.  The
// small footprint (50 KB with the weights) keeps four blocks resident per
// SM, so one block's gathers overlap another's MMAs and epilogue.
template <int MODE>
__global__ void __launch_bounds__(128, 4) k_conv_tc(ConvArgs a)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *sA = sm, *sB = sm + kRound * 4096;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5;
    const unsigned c0 = blockIdx.x * kTile;
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, 32);
        tc::tmem_relinquish();
    }
    if (tid == 0) tc::mbar_init(&mbar, 1);
    // B: weights of every tap, row n = output channel, k = input channel
    for (int i = tid; i < kTaps * 32; i += 128) {
        const int tap = i >> 5, n = (i >> 1) & 15, h = i & 1;
        uint4 v = *reinterpret_cast<const uint4 *>(a.w + ((size_t)tap * 16 + n) * 16 + h * 8);
        *reinterpret_cast<uint4 *>(sB + tap * 512 + tc::kmajor_off(n, h * 8)) = v;
    }
    bool ok = true;
    const uint32_t aaddr = tc::smem_u32(sA), baddr = tc::smem_u32(sB);
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, 16);
    // this thread gathers the channel half h of tile rows r0 and r0 + 64:
    // their grid coordinates once, then one offset per tap.  The eight lanes
    // of a shared-memory store phase take eight consecutive rows (eight
    // different bank groups of the no-swizzle layout).
    const int h = (tid >> 3) & 1, r0 = ((tid >> 4) << 3) | (tid & 7);
    int gx[2], gy[2], gz[2];
    bool gv[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const unsigned c = c0 + (unsigned)(r0 + 64 * q);
        gv[q] = c < a.ncells;
        gx[q] = (int)(c % (unsigned)a.nx);
        gy[q] = (int)((c / (unsigned)a.nx) % (unsigned)a.ny);
        gz[q] = (int)(c / ((unsigned)a.nx * (unsigned)a.ny));
    }
    for (int round = 0; round < kTaps / kRound; ++round) {
        // A: the tile's neighbour values per tap of this round, row = cell,
        // k = channel
#pragma unroll
        for (int tl = 0; tl < kRound; ++tl) {
            const int tap = round * kRound + tl;
            const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int xx = gx[q] + dx, yy = gy[q] + dy, zz = gz[q] + dz;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (gv[q] && xx >= 0 && xx < a.nx && yy >= 0 && yy < a.ny && zz >= 0 && zz < a.nz) {
                    const size_t nb = (size_t)xx + (size_t)a.nx * ((size_t)yy + (size_t)a.ny * (size_t)zz);
                    v = *reinterpret_cast<const uint4 *>(a.in + nb * 16 + h * 8);
                }
                *reinterpret_cast<uint4 *>(sA + tl * 4096 + tc::kmajor_off((uint32_t)(r0 + 64 * q), h * 8)) = v;
            }
        }
        tc::fence_smem_to_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        const uint32_t tbase = tmem_base;
        if (tid == 0) {
            for (int tl = 0; tl < kRound; ++tl)
                tc::mma_bf16(tbase, tc::sdesc(aaddr + tl * 4096, 128, 256),
                             tc::sdesc(baddr + (round * kRound + tl) * 512, 128, 256), idesc,
                             (round > 0 || tl > 0) ? 1u : 0u);
            tc::mma_commit(&mbar);
        }
        // the round's MMAs are done before its tiles are overwritten (and
        // before the accumulator is read)
        if (!tc::mbar_wait_bounded(&mbar, (uint32_t)(round & 1), kWaitLimit)) {
            if (tid == 0) atomicExch(a.err, 1);
            (void)tc::mbar_wait_bounded(&mbar, (uint32_t)(round & 1), kWaitLimit);
            ok = false;
        }
        tc::fence_after_sync();
        __syncthreads();
        if (!ok) break;
    }
    const uint32_t tbase = tmem_base;
    tc::fence_after_sync();
    uint32_t r[16];
    tc::tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16), r);
    tc::tmem_wait_ld();
    const unsigned c = c0 + (unsigned)tid;
    if (ok && c < a.ncells) {
        if (MODE == 1) {
            a.out_f[c] = __uint_as_float(r[0]) + a.bias[0];
        } else {
            float v[16];
            if (MODE == 0) {
                for (int j = 0; j < 16; ++j) v[j] = fmaxf(__uint_as_float(r[j]) + a.bias[j], 0.0f);
            } else {
                const bf16 *m = a.relu_ref + (size_t)c * 16;
                for (int j = 0; j < 16; ++j)
                    v[j] = __bfloat162float(m[j]) > 0.0f ? __uint_as_float(r[j]) : 0.0f;
            }
            __align__(16) __nv_bfloat162 pk[8];
            for (int j = 0; j < 8; ++j) pk[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
            uint4 *dst = reinterpret_cast<uint4 *>(a.out_bf + (size_t)c * 16);
            dst[0] = *reinterpret_cast<const uint4 *>(&pk[0]);
            dst[1] = *reinterpret_cast<const uint4 *>(&pk[4]);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tbase, 32);
}

struct WgradArgs {
    int nx, ny, nz;
    unsigned ncells;
    const bf16 *x;         // layer input [ncells][16]
    const bf16 *g;         // gradient of the layer output [ncells][16]
    unsigned cells_per_block;  // multiple of kWChunk
    float *partial_w;      // [grid][512][16]: row = tap * 16 + in channel
    float *partial_b;      // [grid][16]
    int *err;
};

// Weight and bias gradients of one layer over this block's range of cells,
// in chunks of 64 cells (K = 4 slices of 16).  A holds the shifted inputs
// transposed, columns = cells, in four M tiles of 128 rows: tile t holds
// taps 8t..8t+7, row = in channel * 8 + tap % 8.  One thread takes 8
// consecutive cells of one tap, loads their 16 channels and writes the 16
// rows' 16-byte segments (a register transpose instead of 2-byte
// shared-memory stores); consecutive lanes take consecutive taps, so the
// eight lanes of a store phase write eight different bank groups.  72 KB of
// shared memory keep three blocks resident per SM.
__global__ void __launch_bounds__(128, 3) k_wgrad_tc(WgradArgs a)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *sA = sm, *sB = sm + 16 * 4096;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ float bsum[kWChunk][17];
    __shared__ int3 cxyz[kWChunk];
    const int tid = threadIdx.x, warp = tid >> 5;
    const unsigned cb = blockIdx.x * a.cells_per_block;
    const unsigned ce = min(cb + a.cells_per_block, a.ncells);
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, 64);
        tc::tmem_relinquish();
    }
    if (tid == 0) tc::mbar_init(&mbar, 1);
    // rows of taps 27..31 (the padding of the last M tile) stay zero
    for (unsigned i = tid; i < 16 * 4096 / 16; i += 128)
        reinterpret_cast<uint4 *>(sA)[i] = make_uint4(0u, 0u, 0u, 0u);
    float bacc = 0.0f;   // thread co < 16: bias gradient of channel co
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tmem_base;
    bool ok = true;
    unsigned chunk = 0;
    for (unsigned base = cb; base < ce; base += kWChunk, ++chunk) {
        // grid coordinates of the chunk's cells (x, y, z; x < 0: past the range)
        if (tid < kWChunk) {
            const unsigned c = base + (unsigned)tid;
            cxyz[tid] = c < ce ? make_int3((int)(c % (unsigned)a.nx),
                                           (int)((c / (unsigned)a.nx) % (unsigned)a.ny),
                                           (int)(c / ((unsigned)a.nx * (unsigned)a.ny)))
                               : make_int3(-2, 0, 0);
        }
        __syncthreads();
        // A: item = (tap, group of 8 cells), taps fastest
        for (int item = tid; item < 32 * (kWChunk / 8); item += 128) {
            const int tap = item & 31, g = item >> 5;
            if (tap >= kTaps) continue;
            const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
            uint32_t w[8][8];   // [cell][channel pair]
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int3 p = cxyz[g * 8 + j];
                const int xx = p.x + dx, yy = p.y + dy, zz = p.z + dz;
                uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
                if (p.x >= 0 && xx >= 0 && xx < a.nx && yy >= 0 && yy < a.ny && zz >= 0 && zz < a.nz) {
                    const size_t nb = (size_t)xx + (size_t)a.nx * ((size_t)yy + (size_t)a.ny * (size_t)zz);
                    lo = *reinterpret_cast<const uint4 *>(a.x + nb * 16);
                    hi = *reinterpret_cast<const uint4 *>(a.x + nb * 16 + 8);
                }
                w[j][0] = lo.x; w[j][1] = lo.y; w[j][2] = lo.z; w[j][3] = lo.w;
                w[j][4] = hi.x; w[j][5] = hi.y; w[j][6] = hi.z; w[j][7] = hi.w;
            }
            unsigned char *tile = sA + ((tap >> 3) * 4 + (g >> 1)) * 4096;
            const uint32_t kseg = (uint32_t)(g & 1) * 8;
#pragma unroll
            for (int cp = 0; cp < 8; ++cp) {
                const uint32_t row = (uint32_t)(2 * cp) * 8 + (uint32_t)(tap & 7);
                uint4 vlo, vhi;   // channel 2cp and 2cp+1 of the 8 cells
                vlo.x = __byte_perm(w[0][cp], w[1][cp], 0x5410);
                vlo.y = __byte_perm(w[2][cp], w[3][cp], 0x5410);
                vlo.z = __byte_perm(w[4][cp], w[5][cp], 0x5410);
                vlo.w = __byte_perm(w[6][cp], w[7][cp], 0x5410);
                vhi.x = __byte_perm(w[0][cp], w[1][cp], 0x7632);
                vhi.y = __byte_perm(w[2][cp], w[3][cp], 0x7632);
                vhi.z = __byte_perm(w[4][cp], w[5][cp], 0x7632);
                vhi.w = __byte_perm(w[6][cp], w[7][cp], 0x7632);
                *reinterpret_cast<uint4 *>(tile + tc::kmajor_off(row, kseg)) = vlo;
                *reinterpret_cast<uint4 *>(tile + tc::kmajor_off(row + 8, kseg)) = vhi;
            }
        }
        // B: slice kc holds rows = output channel, columns = cells
        if (tid < kWChunk) {
            const unsigned c = base + tid;
            __align__(16) bf16 v[16];
            if (c < ce) {
                *reinterpret_cast<uint4 *>(&v[0]) = *reinterpret_cast<const uint4 *>(a.g + (size_t)c * 16);
                *reinterpret_cast<uint4 *>(&v[8]) = *reinterpret_cast<const uint4 *>(a.g + (size_t)c * 16 + 8);
            } else {
                *reinterpret_cast<uint4 *>(&v[0]) = make_uint4(0u, 0u, 0u, 0u);
                *reinterpret_cast<uint4 *>(&v[8]) = make_uint4(0u, 0u, 0u, 0u);
            }
            unsigned char *tile = sB + (tid >> 4) * 512;
            for (int co = 0; co < 16; ++co) {
                *reinterpret_cast<bf16 *>(tile + tc::kmajor_off((uint32_t)co, (uint32_t)(tid & 15))) = v[co];
                bsum[tid][co] = __bfloat162float(v[co]);
            }
        }
        tc::fence_smem_to_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
            const uint32_t aaddr = tc::smem_u32(sA), baddr = tc::smem_u32(sB);
            constexpr uint32_t idesc = tc::idesc_bf16_f32(128, 16);
            for (int t = 0; t < 4; ++t)
                for (int kc = 0; kc < kWChunk / 16; ++kc)
                    tc::mma_bf16(tbase + (uint32_t)(t * 16), tc::sdesc(aaddr + (t * 4 + kc) * 4096, 128, 256),
                                 tc::sdesc(baddr + kc * 512, 128, 256), idesc,
                                 (chunk > 0 || kc > 0) ? 1u : 0u);
            tc::mma_commit(&mbar);
        }
        if (tid < 16)
            for (int i = 0; i < kWChunk; ++i) bacc += bsum[i][tid];
        if (!tc::mbar_wait_bounded(&mbar, chunk & 1, kWaitLimit)) {
            if (tid == 0) atomicExch(a.err, 1);
            (void)tc::mbar_wait_bounded(&mbar, chunk & 1, kWaitLimit);
            ok = false;
        }
        tc::fence_after_sync();
        __syncthreads();   // smem tiles may be rewritten
        if (!ok) break;
    }
    float *pw = a.partial_w + (size_t)blockIdx.x * 512 * 16;
    for (int t = 0; t < 4; ++t) {
        uint32_t r[16];
        tc::tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(t * 16), r);
        tc::tmem_wait_ld();
        const int row = warp * 32 + (tid & 31);
        const int m = (t * 8 + (row & 7)) * 16 + (row >> 3);   // tap * 16 + in channel
        for (int co = 0; co < 16; ++co) pw[(size_t)m * 16 + co] = (chunk > 0 && ok) ? __uint_as_float(r[co]) : 0.0f;
    }
    if (tid < 16) a.partial_b[(size_t)blockIdx.x * 16 + tid] = bacc;
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tbase, 64);
}

// dW[tap][out][in] and db[out] from the block partials, summed in block order.
__global__ void k_wgrad_reduce(const float *partial_w, const float *partial_b, unsigned nblk,
                               float *dw, float *db)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (unsigned)kWElems) {
        const unsigned tap = i / 256, co = (i / 16) % 16, ci = i % 16;
        const size_t m = (size_t)tap * 16 + ci;
        float s = 0.0f;
        for (unsigned b = 0; b < nblk; ++b) s += partial_w[((size_t)b * 512 + m) * 16 + co];
        dw[i] = s;
    } else if (i < (unsigned)kWElems + 16) {
        const unsigned co = i - kWElems;
        float s = 0.0f;
        for (unsigned b = 0; b < nblk; ++b) s += partial_b[(size_t)b * 16 + co];
        db[co] = s;
    }
}

// FP32 master weights -> BF16 forward weights and the mirrored, transposed
// weights of the input-gradient convolution.
__global__ void k_pack(const float *w, bf16 *w_bf, bf16 *wt_bf)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (unsigned)kWElems) return;
    const unsigned tap = i / 256, n = (i / 16) % 16, k = i % 16;
    const bf16 v = __float2bfloat16_rn(w[i]);
    w_bf[i] = v;
    wt_bf[((size_t)(kTaps - 1 - tap) * 16 + k) * 16 + n] = v;
}

struct AdamArgs {
    float *w, *m, *v;
    const float *g;
    unsigned n;
    float lr, b1, b2, eps, c1, c2;   // c1 = 1 - b1^t, c2 = 1 - b2^t
};

__global__ void k_adam(AdamArgs a)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float g = a.g[i];
    const float m = a.b1 * a.m[i] + (1.0f - a.b1) * g;
    const float v = a.b2 * a.v[i] + (1.0f - a.b2) * g * g;
    a.m[i] = m;
    a.v[i] = v;
    a.w[i] -= a.lr * (m / a.c1) / (sqrtf(v / a.c2) + a.eps);
}

// ---- Darcy-side kernels: statistics, features, prediction, target ----

struct Scalars {
    unsigned pmax_bits, dphimax_bits, dpmax_bits, nfree;
    float dp_scale;
    int dp_init;
    float loss;
    float wsum;      // sum of the loss weights over free cells
    unsigned resmax_bits;   // this solve's largest extrapolation miss
    float res_scale;        // running scale of the misses (the network's output unit)
    int res_init;
};

// Loss weight of a cell: the solve stops on the largest RELATIVE change
// |dp| / |p| (darcy.cuh, device.cu:2340-2366), so cells with small |p|
// decide the iteration count; the loss weighs errors by 1 / (|p| / pmax +
// 1e-3)^2 to match.
__device__ __forceinline__ float loss_weight(double p, float pscale)
{
    const float r = fabsf((float)p) / pscale + 1e-3f;
    return 1.0f / (r * r);
}

__device__ __forceinline__ unsigned didx_ws(int nx, int ny, int x, int y, int z)
{
    return (unsigned)(x + 1) + ((unsigned)nx + 2u) * (unsigned)(y + 1) +
           ((unsigned)nx + 2u) * ((unsigned)ny + 2u) * (unsigned)(z + 1);
}

__global__ void k_stats(int nx, int ny, int nz, const double *p, const double *dphi,
                        const unsigned char *freec, Scalars *sc)
{
    const unsigned n = (unsigned)nx * ny * nz;
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    float pm = 0.0f, dm = 0.0f;
    unsigned nf = 0;
    if (c < n) {
        const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((unsigned)nx * ny));
        const unsigned g = didx_ws(nx, ny, x, y, z);
        pm = fabsf((float)p[g]);
        dm = fabsf((float)dphi[g]);
        nf = freec[c] ? 1u : 0u;
    }
    for (int o = 16; o > 0; o >>= 1) {
        pm = fmaxf(pm, __shfl_xor_sync(0xffffffffu, pm, o));
        dm = fmaxf(dm, __shfl_xor_sync(0xffffffffu, dm, o));
        nf += __shfl_xor_sync(0xffffffffu, nf, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&sc->pmax_bits, __float_as_uint(pm));
        atomicMax(&sc->dphimax_bits, __float_as_uint(dm));
        atomicAdd(&sc->nfree, nf);
    }
}

__global__ void k_features(int nx, int ny, int nz, const double *p, const double *phi,
                           const double *dphi, const float *dp_last, const Scalars *sc, bf16 *x0)
{
    const unsigned n = (unsigned)nx * ny * nz;
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((unsigned)nx * ny));
    const unsigned g = didx_ws(nx, ny, x, y, z);
    const float ps = fmaxf(__uint_as_float(sc->pmax_bits), 1.0f);
    const float ds = __uint_as_float(sc->dphimax_bits);
    float f[4];
    f[0] = (float)p[g] / ps;
    f[1] = ((float)phi[g] - 0.5f) * 2.0f;
    f[2] = ds > 0.0f ? (float)dphi[g] / ds : 0.0f;
    f[3] = sc->dp_init ? dp_last[c] / sc->dp_scale : 0.0f;
    __align__(16) __nv_bfloat162 pk[8];
    pk[0] = __floats2bfloat162_rn(f[0], f[1]);
    pk[1] = __floats2bfloat162_rn(f[2], f[3]);
    for (int j = 2; j < 8; ++j) pk[j] = __floats2bfloat162_rn(0.0f, 0.0f);
    uint4 *dst = reinterpret_cast<uint4 *>(x0 + (size_t)c * 16);
    dst[0] = *reinterpret_cast<const uint4 *>(&pk[0]);
    dst[1] = *reinterpret_cast<const uint4 *>(&pk[4]);
}

// guess = p_prev + free * (extrapolated change + out * res_scale) on
// interior cells (padded layout): the network corrects the extrapolation of
// the last solutions in units of the extrapolation's typical miss; without
// a network (out null) the guess is that extrapolation
__global__ void k_compose(int nx, int ny, int nz, const double *p, const float *out,
                          const double *dp_base, const unsigned char *freec, const Scalars *sc,
                          double *guess)
{
    const unsigned n = (unsigned)nx * ny * nz;
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((unsigned)nx * ny));
    const unsigned g = didx_ws(nx, ny, x, y, z);
    double v = p[g];
    if (freec[c] && sc->dp_init) {
        v += dp_base[c];
        if (out && sc->res_init) v += (double)out[c] * (double)sc->res_scale;
    }
    guess[g] = v;
}

// the pressure change of the solve just made: its maximum over free cells
// (for the running scale) and the change itself (an input of the next
// prediction)
__global__ void k_dpmax(int nx, int ny, int nz, const double *p_prev, const double *p_star,
                        const unsigned char *freec, Scalars *sc)
{
    const unsigned n = (unsigned)nx * ny * nz;
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    float m = 0.0f;
    if (c < n && freec[c]) {
        const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((unsigned)nx * ny));
        const unsigned g = didx_ws(nx, ny, x, y, z);
        m = fabsf((float)(p_star[g] - p_prev[g]));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&sc->dpmax_bits, __float_as_uint(m));
}

// the change of the solve just made, kept for the next extrapolation (FP64)
// and as the next network input (FP32)
// order of the extrapolation in time of the solutions: 3 = cubic (the next
// change from the last three; measured 2.13x fewer iterations on the
// consolidation workload), 2 = quadratic (1.83x), 1 = linear (1.32x)
#ifndef SPHB_EXTRAP_ORDER
#define SPHB_EXTRAP_ORDER 3
#endif
__global__ void k_dpstore(int nx, int ny, int nz, const double *p_prev, const double *p_star,
                          const unsigned char *freec, float *dp_last, double *dp_base,
                          double *dp_prev, double *dp_prev2)
{
    const unsigned n = (unsigned)nx * ny * nz;
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((unsigned)nx * ny));
    const unsigned g = didx_ws(nx, ny, x, y, z);
    const double dd = freec[c] ? p_star[g] - p_prev[g] : 0.0;
    if (SPHB_EXTRAP_ORDER == 3) {
        // cubic: the next change from the last three
        const double d1 = dp_prev[c], d2 = dp_prev2[c];
        dp_prev2[c] = d1;
        dp_prev[c] = dd;
        dp_base[c] = 3.0 * dd - 3.0 * d1 + d2;
    } else if (SPHB_EXTRAP_ORDER == 2) {
        // quadratic: the next change extrapolated from the last two
        const double d1 = dp_prev[c];
        dp_prev[c] = dd;
        dp_base[c] = dd + (dd - d1);
    } else {
        dp_base[c] = dd;
    }
    dp_last[c] = (float)dd;
}

// the largest miss of the extrapolation over free cells, and its running
// scale (the first value, then an exponential average)
__global__ void k_resmax(int nx, int ny, int nz, const double *p_prev, const double *p_star,
                         const double *dp_base, const unsigned char *freec, Scalars *sc)
{
    const unsigned n = (unsigned)nx * ny * nz;
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    float m = 0.0f;
    if (c < n && freec[c] && sc->dp_init) {
        const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((unsigned)nx * ny));
        const unsigned g = didx_ws(nx, ny, x, y, z);
        m = fabsf((float)(p_star[g] - p_prev[g] - dp_base[c]));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&sc->resmax_bits, __float_as_uint(m));
}

__global__ void k_resscale(Scalars *sc)
{
    const float m = fmaxf(__uint_as_float(sc->resmax_bits), 1e-30f);
    if (!sc->res_init) {
        sc->res_scale = m;
        sc->res_init = 1;
    } else {
        sc->res_scale = 0.9f * sc->res_scale + 0.1f * m;
    }
    sc->resmax_bits = 0u;
}

// running scale of the pressure change: the first solve's maximum, then an
// exponential average of the maxima
__global__ void k_dpscale(Scalars *sc)
{
    const float m = fmaxf(__uint_as_float(sc->dpmax_bits), 1e-30f);
    if (!sc->dp_init) {
        sc->dp_scale = m;
        sc->dp_init = 1;
    } else {
        sc->dp_scale = 0.9f * sc->dp_scale + 0.1f * m;
    }
}

// per-block sums of the loss weights over free cells (tree in block order)
__global__ void k_weight_partials(int nx, int ny, int nz, const double *p_prev,
                                  const unsigned char *freec, const Scalars *sc, float *partial)
{
    __shared__ float red[256];
    const unsigned n = (unsigned)nx * ny * nz;
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    float w = 0.0f;
    if (c < n && freec[c]) {
        const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((unsigned)nx * ny));
        w = loss_weight(p_prev[didx_ws(nx, ny, x, y, z)], fmaxf(__uint_as_float(sc->pmax_bits), 1.0f));
    }
    red[threadIdx.x] = w;
    __syncthreads();
    for (unsigned i = 128; i; i >>= 1) {
        if (threadIdx.x < i) red[threadIdx.x] += red[threadIdx.x + i];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void k_weight_sum(const float *partial, unsigned nb, Scalars *sc)
{
    float s = 0.0f;
    for (unsigned b = 0; b < nb; ++b) s += partial[b];
    sc->wsum = s;
}

// gradient of the loss over free cells at the output: the weighted mean
// squared error of the normalised pressure change, or with
// target_override the plain mean squared error against that target
__global__ void k_loss_grad(int nx, int ny, int nz, const double *p_prev, const double *p_star,
                            const double *dp_base, const float *out, const unsigned char *freec,
                            Scalars *sc, bf16 *g3, const float *target_override)
{
    const unsigned n = (unsigned)nx * ny * nz;
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float grad = 0.0f;
    if (freec[c]) {
        float t, w, wsum;
        if (target_override) {
            t = target_override[c];
            w = 1.0f;
            wsum = (float)max(sc->nfree, 1u);
        } else {
            const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((unsigned)nx * ny));
            const unsigned g = didx_ws(nx, ny, x, y, z);
            // the part of the solve's change the extrapolation missed
            const double base = (dp_base && sc->dp_init) ? dp_base[c] : 0.0;
            t = (float)((p_star[g] - p_prev[g] - base) / (double)sc->res_scale);
            w = loss_weight(p_prev[g], fmaxf(__uint_as_float(sc->pmax_bits), 1.0f));
            wsum = fmaxf(sc->wsum, 1e-30f);
        }
        const float e = out[c] - t;
        if (isfinite(e) && isfinite(w)) {   // a degenerate scale trains nothing
            grad = 2.0f * w * e / wsum;
            atomicAdd(&sc->loss, w * e * e / wsum);
        }
    }
    __align__(16) __nv_bfloat162 pk[8];
    pk[0] = __floats2bfloat162_rn(grad, 0.0f);
    for (int j = 1; j < 8; ++j) pk[j] = __floats2bfloat162_rn(0.0f, 0.0f);
    uint4 *dst = reinterpret_cast<uint4 *>(g3 + (size_t)c * 16);
    dst[0] = *reinterpret_cast<const uint4 *>(&pk[0]);
    dst[1] = *reinterpret_cast<const uint4 *>(&pk[4]);
}

// raw (already normalised) 4-channel inputs -> BF16 activations (test hook)
__global__ void k_pack_inputs(const float *x4, unsigned n, bf16 *x0)
{
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    __align__(16) __nv_bfloat162 pk[8];
    pk[0] = __floats2bfloat162_rn(x4[4 * c], x4[4 * c + 1]);
    pk[1] = __floats2bfloat162_rn(x4[4 * c + 2], x4[4 * c + 3]);
    for (int j = 2; j < 8; ++j) pk[j] = __floats2bfloat162_rn(0.0f, 0.0f);
    uint4 *dst = reinterpret_cast<uint4 *>(x0 + (size_t)c * 16);
    dst[0] = *reinterpret_cast<const uint4 *>(&pk[0]);
    dst[1] = *reinterpret_cast<const uint4 *>(&pk[4]);
}

}  // namespace

// Adam steps per training solve: one keeps the learned fluid step cheaper
// than the reference's plain start on the 40 x 40 x 80 consolidation grid
// (two measured 3.0 ms against 2.6 ms plain, with the same iteration counts)
#ifndef SPHB_WS_TRAIN_ITERS
#define SPHB_WS_TRAIN_ITERS 1
#endif

struct WarmStart {
    int nx = 0, ny = 0, nz = 0;
    unsigned ncells = 0;
    int train_budget = 0, trained = 0, predictions = 0;
    std::vector<void *> allocs;
    bf16 *x0 = nullptr, *a1 = nullptr, *a2 = nullptr, *g3 = nullptr, *g2 = nullptr, *g1 = nullptr;
    float *out = nullptr;
    float *w[3] = {}, *b[3] = {}, *mw[3] = {}, *vw[3] = {}, *mb[3] = {}, *vb[3] = {};
    float *dw[3] = {}, *db[3] = {};
    bf16 *w_bf[3] = {}, *wt_bf[3] = {};
    float *partial_w = nullptr, *partial_b = nullptr;
    unsigned wgrad_blocks = 0, cells_per_block = 0;
    unsigned char *freec = nullptr;
    float *dp_last = nullptr;       // pressure change of the last solve (free cells)
    double *dp_base = nullptr;      // the extrapolated change the guess adds (FP64)
    double *dp_prev = nullptr;      // the last change (FP64), for higher-order extrapolation
    double *dp_prev2 = nullptr;     // the change before it
    bool use_net = true;            // false: the guess is the extrapolation alone
    int solves = 0;                 // solves recorded by ws_train
    float *wpartial = nullptr;      // per-block loss-weight sums
    Scalars *sc = nullptr;
    int train_iters = SPHB_WS_TRAIN_ITERS;   // Adam steps per solve while training
    int *err = nullptr;
    const double *last_p_prev = nullptr;
    int adam_t = 0;
    float lr = 1e-3f;

    template <class T> T *alloc(size_t n)
    {
        void *p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T));
        allocs.push_back(p);
        return (T *)p;
    }
    ~WarmStart()
    {
        for (void *p : allocs) cudaFree(p);
    }
};

namespace {

unsigned blocks(unsigned n, unsigned b) { return (n + b - 1) / b; }

bool set_attrs()
{
    static bool done = false, ok = false;
    if (done) return ok;
    done = true;
    ok = cudaFuncSetAttribute(k_conv_tc<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kConvSmem) == cudaSuccess &&
         cudaFuncSetAttribute(k_conv_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kConvSmem) == cudaSuccess &&
         cudaFuncSetAttribute(k_conv_tc<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kConvSmem) == cudaSuccess &&
         cudaFuncSetAttribute(k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWgradSmem) == cudaSuccess;
    return ok;
}

cudaError_t conv(WarmStart &W, int mode, const bf16 *in, const bf16 *w, const float *bias,
                 const bf16 *relu_ref, bf16 *out_bf, float *out_f, cudaStream_t st)
{
    ConvArgs a;
    a.nx = W.nx; a.ny = W.ny; a.nz = W.nz; a.ncells = W.ncells;
    a.in = in; a.w = w; a.bias = bias; a.relu_ref = relu_ref; a.out_bf = out_bf; a.out_f = out_f;
    a.err = W.err;
    const unsigned g = blocks(W.ncells, kTile);
    if (mode == 0) k_conv_tc<0><<<g, 128, kConvSmem, st>>>(a);
    else if (mode == 1) k_conv_tc<1><<<g, 128, kConvSmem, st>>>(a);
    else k_conv_tc<2><<<g, 128, kConvSmem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t wgrad(WarmStart &W, const bf16 *x, const bf16 *g, int layer, cudaStream_t st)
{
    WgradArgs a;
    a.nx = W.nx; a.ny = W.ny; a.nz = W.nz; a.ncells = W.ncells;
    a.x = x; a.g = g; a.cells_per_block = W.cells_per_block;
    a.partial_w = W.partial_w; a.partial_b = W.partial_b; a.err = W.err;
    k_wgrad_tc<<<W.wgrad_blocks, 128, kWgradSmem, st>>>(a);
    k_wgrad_reduce<<<blocks(kWElems + 16, 256), 256, 0, st>>>(W.partial_w, W.partial_b,
                                                             W.wgrad_blocks, W.dw[layer], W.db[layer]);
    return cudaGetLastError();
}

cudaError_t forward(WarmStart &W, cudaStream_t st)
{
    cudaError_t e;
    if ((e = conv(W, 0, W.x0, W.w_bf[0], W.b[0], nullptr, W.a1, nullptr, st)) != cudaSuccess) return e;
    if ((e = conv(W, 0, W.a1, W.w_bf[1], W.b[1], nullptr, W.a2, nullptr, st)) != cudaSuccess) return e;
    return conv(W, 1, W.a2, W.w_bf[2], W.b[2], nullptr, nullptr, W.out, st);
}

// gradients of every layer from g3 (the output gradient already in W.g3)
cudaError_t backward(WarmStart &W, cudaStream_t st)
{
    cudaError_t e;
    if ((e = wgrad(W, W.a2, W.g3, 2, st)) != cudaSuccess) return e;
    if ((e = conv(W, 2, W.g3, W.wt_bf[2], nullptr, W.a2, W.g2, nullptr, st)) != cudaSuccess) return e;
    if ((e = wgrad(W, W.a1, W.g2, 1, st)) != cudaSuccess) return e;
    if ((e = conv(W, 2, W.g2, W.wt_bf[1], nullptr, W.a1, W.g1, nullptr, st)) != cudaSuccess) return e;
    return wgrad(W, W.x0, W.g1, 0, st);
}

cudaError_t pack_all(WarmStart &W, cudaStream_t st)
{
    for (int l = 0; l < 3; ++l)
        k_pack<<<blocks(kWElems, 256), 256, 0, st>>>(W.w[l], W.w_bf[l], W.wt_bf[l]);
    return cudaGetLastError();
}

cudaError_t adam_step(WarmStart &W, cudaStream_t st)
{
    W.adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    AdamArgs a;
    a.lr = W.lr; a.b1 = b1; a.b2 = b2; a.eps = 1e-8f;
    a.c1 = 1.0f - std::pow(b1, (float)W.adam_t);
    a.c2 = 1.0f - std::pow(b2, (float)W.adam_t);
    for (int l = 0; l < 3; ++l) {
        a.w = W.w[l]; a.m = W.mw[l]; a.v = W.vw[l]; a.g = W.dw[l]; a.n = kWElems;
        k_adam<<<blocks(kWElems, 256), 256, 0, st>>>(a);
        a.w = W.b[l]; a.m = W.mb[l]; a.v = W.vb[l]; a.g = W.db[l]; a.n = 16;
        k_adam<<<1, 32, 0, st>>>(a);
    }
    return pack_all(W, st);
}

}  // namespace

WarmStart *ws_create(int nx, int ny, int nz, uint64_t seed, int train_solves, bool use_net)
{
    if (!set_attrs()) return nullptr;
    auto *W = new WarmStart();
    W->use_net = use_net;
    W->nx = nx; W->ny = ny; W->nz = nz;
    W->ncells = (unsigned)nx * ny * nz;
    W->train_budget = train_solves;
    const size_t act = (size_t)W->ncells * kCh;
    W->x0 = W->alloc<bf16>(act); W->a1 = W->alloc<bf16>(act); W->a2 = W->alloc<bf16>(act);
    W->g3 = W->alloc<bf16>(act); W->g2 = W->alloc<bf16>(act); W->g1 = W->alloc<bf16>(act);
    W->out = W->alloc<float>(W->ncells);
    W->freec = W->alloc<unsigned char>(W->ncells);
    W->dp_last = W->alloc<float>(W->ncells);
    W->dp_base = W->alloc<double>(W->ncells);
    W->dp_prev = W->alloc<double>(W->ncells);
    W->dp_prev2 = W->alloc<double>(W->ncells);
    W->wpartial = W->alloc<float>(blocks(W->ncells, 256));
    W->sc = W->alloc<Scalars>(1);
    W->err = W->alloc<int>(1);
    // weight-gradient blocks: three per SM, each over a multiple of 64 cells
    {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const unsigned target = std::max(1u, std::min((unsigned)(3 * sms), blocks(W->ncells, kWChunk)));
        W->cells_per_block = blocks(blocks(W->ncells, target), kWChunk) * kWChunk;
        W->wgrad_blocks = blocks(W->ncells, W->cells_per_block);
    }
    W->partial_w = W->alloc<float>((size_t)W->wgrad_blocks * 512 * 16);
    W->partial_b = W->alloc<float>((size_t)W->wgrad_blocks * 16);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    for (int l = 0; l < 3; ++l) {
        W->w[l] = W->alloc<float>(kWElems); W->b[l] = W->alloc<float>(16);
        W->mw[l] = W->alloc<float>(kWElems); W->vw[l] = W->alloc<float>(kWElems);
        W->mb[l] = W->alloc<float>(16); W->vb[l] = W->alloc<float>(16);
        W->dw[l] = W->alloc<float>(kWElems); W->db[l] = W->alloc<float>(16);
        W->w_bf[l] = W->alloc<bf16>(kWElems); W->wt_bf[l] = W->alloc<bf16>(kWElems);
        // He initialisation over the real fan-in; unused channels stay zero
        const int cin = l == 0 ? kInputs : 16, cout = l == 2 ? 1 : 16;
        const float stdv = l == 2 ? 1e-3f : std::sqrt(2.0f / (27.0f * cin));
        std::vector<float> h(kWElems, 0.0f);
        for (int tap = 0; tap < kTaps; ++tap)
            for (int co = 0; co < cout; ++co)
                for (int ci = 0; ci < cin; ++ci) h[(tap * 16 + co) * 16 + ci] = stdv * nd(rng);
        cudaMemcpy(W->w[l], h.data(), kWElems * 4, cudaMemcpyHostToDevice);
    }
    for (void *p : W->allocs)
        if (!p) {
            delete W;
            return nullptr;
        }
    if (pack_all(*W, nullptr) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        delete W;
        return nullptr;
    }
    return W;
}

void ws_destroy(WarmStart *w) { delete w; }

int ws_trained(const WarmStart *w) { return w ? w->trained : 0; }
int ws_predictions(const WarmStart *w) { return w ? w->predictions : 0; }

cudaError_t ws_predict(WarmStart *W, const WSDarcyInputs &in, double *guess, double *guess_base,
                       cudaStream_t st)
{
    const unsigned n = W->ncells;
    cudaError_t e = cudaMemcpyAsync(W->freec, in.free, n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    // clear the per-solve statistics (dp_scale and dp_init persist)
    if ((e = cudaMemsetAsync(W->sc, 0, 16, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(&W->sc->loss, 0, 4, st)) != cudaSuccess) return e;
    k_stats<<<blocks(n, 256), 256, 0, st>>>(W->nx, W->ny, W->nz, in.p, in.dphi, W->freec, W->sc);
    if (W->use_net) {
        k_features<<<blocks(n, 256), 256, 0, st>>>(W->nx, W->ny, W->nz, in.p, in.phi, in.dphi,
                                                  W->dp_last, W->sc, W->x0);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = forward(*W, st)) != cudaSuccess) return e;
    }
    k_compose<<<blocks(n, 256), 256, 0, st>>>(W->nx, W->ny, W->nz, in.p, W->use_net ? W->out : nullptr,
                                             W->dp_base, W->freec, W->sc, guess);
    if (guess_base && W->use_net)
        k_compose<<<blocks(n, 256), 256, 0, st>>>(W->nx, W->ny, W->nz, in.p, nullptr, W->dp_base,
                                                 W->freec, W->sc, guess_base);
    W->last_p_prev = in.p;
    W->predictions += 1;
    return cudaGetLastError();
}

cudaError_t ws_train(WarmStart *W, const double *p_prev, const double *p_star, cudaStream_t st)
{
    const unsigned n = W->ncells;
    cudaError_t e;
    // the running scale, including this solve's change
    k_dpmax<<<blocks(n, 256), 256, 0, st>>>(W->nx, W->ny, W->nz, p_prev, p_star, W->freec, W->sc);
    k_dpscale<<<1, 1, 0, st>>>(W->sc);
    // training (from the second solve on, when an extrapolation exists),
    // towards what the extrapolation the prediction used missed, in units of
    // its running scale
    if (W->use_net && W->solves > 0) {
        k_resmax<<<blocks(n, 256), 256, 0, st>>>(W->nx, W->ny, W->nz, p_prev, p_star, W->dp_base,
                                                 W->freec, W->sc);
        k_resscale<<<1, 1, 0, st>>>(W->sc);
    }
    if (W->use_net && W->solves > 0 && W->trained < W->train_budget) {
        k_weight_partials<<<blocks(n, 256), 256, 0, st>>>(W->nx, W->ny, W->nz, p_prev, W->freec,
                                                          W->sc, W->wpartial);
        k_weight_sum<<<1, 1, 0, st>>>(W->wpartial, blocks(n, 256), W->sc);
        for (int it = 0; it < W->train_iters; ++it) {
            if (it > 0 && (e = forward(*W, st)) != cudaSuccess) return e;
            if ((e = cudaMemsetAsync(&W->sc->loss, 0, 4, st)) != cudaSuccess) return e;
            k_loss_grad<<<blocks(n, 256), 256, 0, st>>>(W->nx, W->ny, W->nz, p_prev, p_star, W->dp_base,
                                                        W->out, W->freec, W->sc, W->g3, nullptr);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            if ((e = backward(*W, st)) != cudaSuccess) return e;
            if ((e = adam_step(*W, st)) != cudaSuccess) return e;
        }
        W->trained += 1;
    }
    // every solve: the change the next prediction extrapolates
    k_dpstore<<<blocks(n, 256), 256, 0, st>>>(W->nx, W->ny, W->nz, p_prev, p_star, W->freec,
                                              W->dp_last, W->dp_base, W->dp_prev, W->dp_prev2);
    W->solves += 1;
    return cudaGetLastError();
}

int ws_error(WarmStart *W, cudaStream_t st)
{
    int v = 0;
    cudaMemcpyAsync(&v, W->err, 4, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return v;
}

float ws_last_loss(WarmStart *W, cudaStream_t st)
{
    float v = 0.0f;
    cudaMemcpyAsync(&v, &W->sc->loss, 4, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return v;
}

// ---- test hooks: the network on host arrays ----

int ws_set_params(WarmStart *W, int layer, const float *w, const float *b)
{
    if (!W || layer < 0 || layer > 2) return -1;
    cudaMemcpy(W->w[layer], w, kWElems * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(W->b[layer], b, 64, cudaMemcpyHostToDevice);
    return pack_all(*W, nullptr) == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

int ws_get_params(WarmStart *W, int layer, float *w, float *b)
{
    if (!W || layer < 0 || layer > 2) return -1;
    cudaMemcpy(w, W->w[layer], kWElems * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(b, W->b[layer], 64, cudaMemcpyDeviceToHost);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

int ws_forward_host(WarmStart *W, const float *x4, float *out)
{
    const unsigned n = W->ncells;
    float *dx = nullptr;
    if (cudaMalloc(&dx, (size_t)n * 16) != cudaSuccess) return -1;
    cudaMemcpy(dx, x4, (size_t)n * 16, cudaMemcpyHostToDevice);
    k_pack_inputs<<<blocks(n, 256), 256>>>(dx, n, W->x0);
    cudaError_t e = forward(*W, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(dx);
    if (e != cudaSuccess) return -1;
    cudaMemcpy(out, W->out, (size_t)n * 4, cudaMemcpyDeviceToHost);
    return ws_error(W, nullptr) ? -2 : 0;
}

int ws_gradients_host(WarmStart *W, const float *x4, const float *target, const unsigned char *freec,
                      float *dw, float *db)
{
    const unsigned n = W->ncells;
    std::vector<float> out(n);
    if (ws_forward_host(W, x4, out.data())) return -1;
    float *dt = nullptr;
    if (cudaMalloc(&dt, (size_t)n * 4) != cudaSuccess) return -1;
    cudaMemcpy(dt, target, (size_t)n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(W->freec, freec, n, cudaMemcpyHostToDevice);
    unsigned nf = 0;
    for (unsigned i = 0; i < n; ++i) nf += freec[i] ? 1u : 0u;
    Scalars s;
    std::memset(&s, 0, sizeof s);
    s.nfree = nf;
    s.dp_scale = 1.0f;
    s.dp_init = 1;
    cudaMemcpy(W->sc, &s, sizeof s, cudaMemcpyHostToDevice);
    k_loss_grad<<<blocks(n, 256), 256>>>(W->nx, W->ny, W->nz, nullptr, nullptr, nullptr, W->out, W->freec,
                                         W->sc, W->g3, dt);
    cudaError_t e = backward(*W, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(dt);
    if (e != cudaSuccess) return -1;
    for (int l = 0; l < 3; ++l) {
        cudaMemcpy(dw + (size_t)l * kWElems, W->dw[l], kWElems * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(db + (size_t)l * 16, W->db[l], 64, cudaMemcpyDeviceToHost);
    }
    return ws_error(W, nullptr) ? -2 : 0;
}

}  // namespace sphb

// ---- C ABI of the network alone (gradient checks against the CPU oracle) ----

struct sph_wsnet {
    sphb::WarmStart *w;
};

extern "C" {

int sph_wsnet_create(int nx, int ny, int nz, uint64_t seed, sph_wsnet **out)
{
    if (!out || nx < 1 || ny < 1 || nz < 1) return -8;
    sphb::WarmStart *w = sphb::ws_create(nx, ny, nz, seed, 0, true);
    if (!w) return -4;
    *out = new sph_wsnet{w};
    return 0;
}

int sph_wsnet_set_params(sph_wsnet *n, int layer, const float *w, const float *b)
{
    return (n && w && b) ? sphb::ws_set_params(n->w, layer, w, b) : -8;
}

int sph_wsnet_get_params(sph_wsnet *n, int layer, float *w, float *b)
{
    return (n && w && b) ? sphb::ws_get_params(n->w, layer, w, b) : -8;
}

int sph_wsnet_forward(sph_wsnet *n, const float *x4, float *out)
{
    return (n && x4 && out) ? sphb::ws_forward_host(n->w, x4, out) : -8;
}

int sph_wsnet_gradients(sph_wsnet *n, const float *x4, const float *target,
                        const unsigned char *free_cells, float *dw, float *db)
{
    return (n && x4 && target && free_cells && dw && db)
               ? sphb::ws_gradients_host(n->w, x4, target, free_cells, dw, db)
               : -8;
}

void sph_wsnet_destroy(sph_wsnet *n)
{
    if (!n) return;
    sphb::ws_destroy(n->w);
    delete n;
}

}  // extern "C"
