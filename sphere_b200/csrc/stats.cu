// Diagnostics computed on the device from the resident state, replacing the
// reference's host-side analysis tools:
//   - energy sums of python/sphere.py:4311-4380 (sim.energy(method));
//   - the porosity profile of DEM::porosity (src/sphere.cpp:487-605, the
//     `porosity` program);
//   - the particle-overlap list of DEM::findOverlaps (src/sphere.cpp:677-725,
//     `sphere --contacts`, behind sim.findOverlaps() and the coordination
//     number), by a cell-grid search instead of the O(N^2) double loop.
//
// Every sum is formed per block in a fixed tree order and then added on the
// host in block order, so results are deterministic; they differ from the
// reference's serial sums only by rounding.  The overlap list is exact: the
// same pairs in the same order, the same FP64 separation arithmetic (this
// file is compiled with -fmad=false).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine_internal.h"

namespace sphb {

namespace {

constexpr int STAT_THREADS = 256;
constexpr int NSUMS = 7;   // pot, kin, rot, es, es_dot, ev, ev_dot

// Math constant of python's math.pi and C's M_PI (both the FP64 value of pi).
constexpr double PI_FULL = 3.141592653589793;

unsigned blocks_of(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// Tree sum of one value per thread; every thread gets the block's sum.
__device__ double block_tree_sum(double v, double *sh)
{
    sh[threadIdx.x] = v;
    __syncthreads();
    for (unsigned s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

// Per-particle energy terms of sim.energy() (python/sphere.py:4327-4358):
// m = 4/3 pi r^3 rho evaluated as (4/3 * pi) * r**3 * rho;
// pot = m |g| z; kin = 1/2 m sqrt(v.v)^2; rot = 1/2 2/5 m r^2 sqrt(w.w)^2.
__global__ void __launch_bounds__(STAT_THREADS) k_energy_partials(DevParams P, DevState S,
                                                                  double *part)
{
    __shared__ double sh[STAT_THREADS];
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    double t[NSUMS] = {0, 0, 0, 0, 0, 0, 0};
    if (k < P.np) {
        const double4 x = S.x[k], v = S.vel[k], w = S.angvel[k];
        const double r = x.w;
        const double m = 4.0 / 3.0 * PI_FULL * pow(r, 3.0) * P.rho;
        const double gabs = sqrt(P.g[0] * P.g[0] + P.g[1] * P.g[1] + P.g[2] * P.g[2]);
        t[0] = m * gabs * x.z;
        const double sv = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
        t[1] = 0.5 * m * (sv * sv);
        const double sw = sqrt(w.x * w.x + w.y * w.y + w.z * w.z);
        t[2] = 0.5 * 2.0 / 5.0 * m * (r * r) * (sw * sw);
        t[3] = S.es[k];
        t[4] = S.es_dot[k];
        t[5] = S.ev[k];
        t[6] = S.ev_dot[k];
    }
    for (int s = 0; s < NSUMS; ++s) {
        double b = block_tree_sum(t[s], sh);
        if (threadIdx.x == 0) part[(size_t)blockIdx.x * NSUMS + s] = b;
    }
}

// Bond energy terms of sim.energy('bondpot') (python/sphere.py:4360-4376):
// R = lambda_bar min(r_i, r_j), A = pi R^2, I = pi R^4 / 4, J = 2 I.
// The reference multiplies each bond's 0.5 A k_t (and 0.5 I k_n) by the norm
// of the WHOLE delta_t (omega_t) array squared, so those two terms are
// formed here as (sum of the per-bond factors) x (sum of squares over all
// bonds).  Sums: [0] 0.5 A k_n dn^2, [1] 0.5 A k_t, [2] |delta_t|^2,
// [3] 0.5 J k_t wn^2, [4] 0.5 I k_n, [5] |omega_t|^2.
__global__ void __launch_bounds__(STAT_THREADS) k_bond_partials(DevParams P, DevState S,
                                                                double *part)
{
    __shared__ double sh[STAT_THREADS];
    const unsigned b = blockIdx.x * blockDim.x + threadIdx.x;
    double t[6] = {0, 0, 0, 0, 0, 0};
    if (b < P.nb0) {
        const uint2 bd = S.bonds[b];
        // a broken bond keeps index nb0 in .x (src/cohesion.cuh:205); the
        // host checked that every index used here is below np
        const double ri = S.x[S.pos_of[bd.x]].w, rj = S.x[S.pos_of[bd.y]].w;
        const double R = P.lambda_bar * fmin(ri, rj);
        const double A = PI_FULL * (R * R);
        const double I = 0.25 * PI_FULL * pow(R, 4.0);
        const double J = I * 2.0;
        const double4 d = S.bonds_delta[b], o = S.bonds_omega[b];
        const double dn = fabs(d.w), wn = fabs(o.w);
        t[0] = 0.5 * A * P.k_n * (dn * dn);
        t[1] = 0.5 * A * P.k_t;
        t[2] = d.x * d.x + d.y * d.y + d.z * d.z;
        t[3] = 0.5 * J * P.k_t * (wn * wn);
        t[4] = 0.5 * I * P.k_n;
        t[5] = o.x * o.x + o.y * o.y + o.z * o.z;
    }
    for (int s = 0; s < 6; ++s) {
        double v = block_tree_sum(t[s], sh);
        if (threadIdx.x == 0) part[(size_t)blockIdx.x * 6 + s] = v;
    }
}

__device__ __forceinline__ double spherical_cap(double h, double r)
{
    return PI_FULL * h * h / 3.0 * (3.0 * r - h);   // src/sphere.cpp:468-471
}

// Solid volume that DEM::porosity subtracts from slice iz = blockIdx.y for
// one particle (src/sphere.cpp:531-589), the same case analysis, including
// the reference's "V_sphere + cap" where the sphere minus the cap outside
// the slice would be the geometric volume.  Slices start at z = 0, not at
// origo.z, as in the reference.
__global__ void __launch_bounds__(STAT_THREADS) k_porosity_partials(DevParams P, DevState S,
                                                                    double h_slice, double *part)
{
    __shared__ double sh[STAT_THREADS];
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned iz = blockIdx.y;
    double sub = 0.0;
    if (k < P.np) {
        const double z_slice_low = (double)iz * h_slice;
        const double z_slice_high = z_slice_low + h_slice;
        const double4 x = S.x[k];
        const double c = x.z, radius = x.w;
        const double lo = c - radius, hi = c + radius;
        const double V_sphere = 4.0 / 3.0 * PI_FULL * radius * radius * radius;
        if (z_slice_low <= lo && hi <= z_slice_high) {
            sub = V_sphere;
        } else {
            if (z_slice_low >= c && z_slice_low <= hi)
                sub += spherical_cap(hi - z_slice_low, radius);
            else if (z_slice_low < c && z_slice_low > lo)
                sub += V_sphere + spherical_cap(z_slice_low - lo, radius);
            if (z_slice_high <= c && z_slice_high >= lo)
                sub += spherical_cap(z_slice_high - lo, radius);
            else if (z_slice_high > c && z_slice_high < hi)
                sub += V_sphere + spherical_cap(hi - z_slice_high, radius);
        }
    }
    double v = block_tree_sum(sub, sh);
    if (threadIdx.x == 0) part[(size_t)iz * gridDim.x + blockIdx.x] = v;
}

// ---- overlap list (src/sphere.cpp:677-725) ----

// Largest radius, as the bit pattern of a positive double (ordered like u64).
__global__ void k_rmax(DevParams P, DevState S, unsigned long long *out)
{
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < P.np) atomicMax(out, (unsigned long long)__double_as_longlong(S.x[k].w));
}

// Cell of each ORIGINAL index from its current position; counts per cell.
// Particles outside the grid are counted in *outside (the engine's error
// flag is left alone).
__global__ void k_ov_hash(DevParams P, DevState S, uint32_t *key, uint32_t *cnt, uint32_t *outside)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np) return;
    const double4 x = S.x[S.pos_of[i]];
    int c[3];
    if (!cell_coord(P, x.x, 0, c[0]) || !cell_coord(P, x.y, 1, c[1]) || !cell_coord(P, x.z, 2, c[2])) {
        atomicAdd(outside, 1u);
        key[i] = 0xffffffffu;
        return;
    }
    const uint32_t kk = ((uint32_t)c[2] * P.num[1] + (uint32_t)c[1]) * P.num[0] + (uint32_t)c[0];
    key[i] = kk;
    atomicAdd(cnt + kk, 1u);
}

// Exclusive scan of n counts by one block (diagnostic sizes; each thread
// owns one contiguous chunk).  out[n] = total.
__global__ void __launch_bounds__(1024) k_scan_1block(const uint32_t *in, uint32_t *out, uint32_t n)
{
    __shared__ uint32_t tot[1024];
    const uint32_t T = blockDim.x, t = threadIdx.x;
    const uint32_t chunk = (n + T - 1) / T;
    const uint32_t b = min(n, t * chunk), e = min(n, b + chunk);
    uint32_t s = 0;
    for (uint32_t i = b; i < e; ++i) s += in[i];
    tot[t] = s;
    __syncthreads();
    if (t == 0) {
        uint32_t run = 0;
        for (uint32_t i = 0; i < T; ++i) {
            uint32_t v = tot[i];
            tot[i] = run;
            run += v;
        }
        out[n] = run;
    }
    __syncthreads();
    uint32_t run = tot[t];
    for (uint32_t i = b; i < e; ++i) {
        uint32_t v = in[i];
        out[i] = run;
        run += v;
    }
}

__global__ void k_ov_fill(DevParams P, const uint32_t *key, const uint32_t *start, uint32_t *fill,
                          uint32_t *list)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np || key[i] == 0xffffffffu) return;
    list[start[key[i]] + atomicAdd(fill + key[i], 1u)] = i;
}

// Pairs (i, j > i) of ORIGINAL indices with negative separation
// |x_j - x_i| - (r_i + r_j) whose fixvel flags are both zero
// (src/sphere.cpp:690-722), among cells within `reach` of i's cell (no
// periodic images, like the reference).  PASS 0 counts, PASS 1 writes the
// pairs of i from out_off[i] on and then orders them by j.
template <int PASS>
__global__ void __launch_bounds__(STAT_THREADS) k_ov_search(DevParams P, DevState S, const uint32_t *key,
                                                             const uint32_t *start, const uint32_t *list,
                                                             int3 reach, uint32_t *count,
                                                             const uint32_t *out_off, uint32_t *out_j,
                                                             double *out_d)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np || key[i] == 0xffffffffu) return;
    const double4 xi = S.x[S.pos_of[i]];
    const double4 vi = S.vel[S.pos_of[i]];
    uint32_t n = 0;
    if (vi.w == 0.0) {
        const uint32_t kk = key[i];
        const int cx = (int)(kk % P.num[0]), cy = (int)((kk / P.num[0]) % P.num[1]),
                  cz = (int)(kk / (P.num[0] * P.num[1]));
        const uint32_t base = PASS ? out_off[i] : 0u;
        for (int z = max(0, cz - reach.z); z <= min((int)P.num[2] - 1, cz + reach.z); ++z)
            for (int y = max(0, cy - reach.y); y <= min((int)P.num[1] - 1, cy + reach.y); ++y)
                for (int x = max(0, cx - reach.x); x <= min((int)P.num[0] - 1, cx + reach.x); ++x) {
                    const uint32_t c = ((uint32_t)z * P.num[1] + (uint32_t)y) * P.num[0] + (uint32_t)x;
                    for (uint32_t q = start[c]; q < start[c + 1]; ++q) {
                        const uint32_t j = list[q];
                        if (j <= i) continue;
                        const uint32_t pj = S.pos_of[j];
                        const double4 xj = S.x[pj];
                        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
                        const double len = sqrt(dx * dx + dy * dy + dz * dz);
                        const double delta = len - (xi.w + xj.w);
                        if (delta < 0.0 && S.vel[pj].w == 0.0) {
                            if (PASS) {
                                out_j[base + n] = j;
                                out_d[base + n] = delta;
                            }
                            ++n;
                        }
                    }
                }
        if (PASS) {
            // insertion sort of this particle's segment by j
            for (uint32_t a = 1; a < n; ++a) {
                const uint32_t jj = out_j[base + a];
                const double dd = out_d[base + a];
                uint32_t b = a;
                while (b > 0 && out_j[base + b - 1] > jj) {
                    out_j[base + b] = out_j[base + b - 1];
                    out_d[base + b] = out_d[base + b - 1];
                    --b;
                }
                out_j[base + b] = jj;
                out_d[base + b] = dd;
            }
        }
    }
    if (!PASS) count[i] = n;
}

// RAII device scratch for one diagnostic call.
struct Scratch {
    std::vector<void *> p;
    template <class T> T *get(size_t n)
    {
        void *q = nullptr;
        if (cudaMalloc(&q, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
        p.push_back(q);
        return (T *)q;
    }
    ~Scratch()
    {
        for (void *q : p) cudaFree(q);
    }
};

}  // namespace

int Engine::energy(const char *method, double *out)
{
    if (!method || !out) return fail(ST_ARG, "energy: null argument");
    static const char *names[NSUMS] = {"pot", "kin", "rot", "shear", "shearrate", "visc_n",
                                       "visc_n_rate"};
    int which = -1;
    for (int s = 0; s < NSUMS; ++s)
        if (std::strcmp(method, names[s]) == 0) which = s;
    const bool bond = std::strcmp(method, "bondpot") == 0;
    if (which < 0 && !bond) return fail(ST_ARG, std::string("Unknown energy() method \"") + method + "\"");
    int rc = poll_errors("energy");
    if (rc < 0 && rc != ST_OUTSIDE && rc != ST_CAPACITY) return rc;
    Scratch sc;
    cudaError_t e = cudaSuccess;
    if (!bond) {
        const unsigned nb = blocks_of(hs.np, STAT_THREADS);
        double *part = sc.get<double>((size_t)nb * NSUMS);
        if (!part) return fail(ST_CUDA, "energy: out of device memory");
        if (nb) k_energy_partials<<<nb, STAT_THREADS, 0, stream>>>(P, S, part);
        std::vector<double> h((size_t)nb * NSUMS);
        e = cudaGetLastError();
        if (e == cudaSuccess && nb)
            e = cudaMemcpyAsync(h.data(), part, h.size() * 8, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "energy");
        double acc = 0.0;
        for (unsigned b = 0; b < nb; ++b) acc += h[(size_t)b * NSUMS + which];
        *out = acc;
        return ST_OK;
    }
    if (hs.nb0 == 0) {
        *out = 0.0;
        return ST_OK;
    }
    // python indexes radius[bonds[:, 0]] and radius[bonds[:, 1]]: an index
    // at or beyond np raises IndexError there, an error here
    std::vector<uint32_t> bonds((size_t)hs.nb0 * 2);
    e = cudaMemcpyAsync(bonds.data(), S.bonds, bonds.size() * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "energy");
    for (uint32_t v : bonds)
        if (v >= hs.np) return fail(ST_ARG, "energy: a bond refers to a particle index beyond np");
    const unsigned nb = blocks_of(hs.nb0, STAT_THREADS);
    double *part = sc.get<double>((size_t)nb * 6);
    if (!part) return fail(ST_CUDA, "energy: out of device memory");
    k_bond_partials<<<nb, STAT_THREADS, 0, stream>>>(P, S, part);
    std::vector<double> h((size_t)nb * 6);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, h.size() * 8, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "energy");
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (unsigned b = 0; b < nb; ++b)
        for (int k = 0; k < 6; ++k) s[k] += h[(size_t)b * 6 + k];
    *out = s[0] + s[1] * s[2] + s[3] + s[4] * s[5];
    return ST_OK;
}

int Engine::porosity_profile(int z_slices, double *z_pos, double *porosity)
{
    if (z_slices < 1 || !z_pos || !porosity) return fail(ST_ARG, "porosity: bad arguments");
    int rc = poll_errors("porosity");
    if (rc < 0 && rc != ST_OUTSIDE && rc != ST_CAPACITY) return rc;
    // top = walls.nx->w (wall 0 position) when there are walls, else L_z
    double top = hs.L[2];
    cudaError_t e = cudaSuccess;
    if (hs.nw > 0) {
        double4 w0;
        e = cudaMemcpyAsync(&w0, S.wnx, sizeof w0, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "porosity");
        top = w0.w;
    }
    const double h_slice = (top - hs.origo[2]) / (double)z_slices;
    // The reference compares with 2 * DEM::r_max(), which returns the radius
    // of the LAST particle (src/sphere.cpp:474-484), not the largest one.
    double r_last = 0.0;
    if (hs.np > 0) {
        uint32_t pos = 0;
        e = cudaMemcpyAsync(&pos, S.pos_of + (hs.np - 1), 4, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        double4 xl{};
        if (e == cudaSuccess) e = cudaMemcpyAsync(&xl, S.x + pos, sizeof xl, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "porosity");
        r_last = xl.w;
    }
    if (h_slice <= r_last * 2.0) return fail(ST_ARG, "Error! The number of z-slices is too high.");
    const double V_slice = h_slice * hs.L[0] * hs.L[1];
    const unsigned nb = blocks_of(hs.np, STAT_THREADS);
    std::vector<double> h((size_t)nb * z_slices);
    Scratch sc;
    if (nb) {
        double *part = sc.get<double>(h.size());
        if (!part) return fail(ST_CUDA, "porosity: out of device memory");
        k_porosity_partials<<<dim3(nb, (unsigned)z_slices), STAT_THREADS, 0, stream>>>(P, S, h_slice, part);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, h.size() * 8, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "porosity");
    }
    for (int iz = 0; iz < z_slices; ++iz) {
        double solid = 0.0;
        for (unsigned b = 0; b < nb; ++b) solid += h[(size_t)iz * nb + b];
        const double z_slice_low = iz * h_slice;
        z_pos[iz] = z_slice_low + 0.5 * h_slice;
        porosity[iz] = (V_slice - solid) / V_slice;
    }
    return ST_OK;
}

int Engine::overlaps(uint32_t *pairs, double *delta, uint64_t cap, uint64_t *count)
{
    if (!count) return fail(ST_ARG, "overlaps: null count");
    *count = 0;
    int rc = poll_errors("overlaps");
    if (rc < 0) return rc;
    const size_t n = hs.np, nc = hs.ncells();
    if (n == 0) return ST_OK;
    Scratch sc;
    unsigned long long *rmax_bits = sc.get<unsigned long long>(1);
    uint32_t *outside = sc.get<uint32_t>(1);
    uint32_t *key = sc.get<uint32_t>(n), *cnt = sc.get<uint32_t>(nc), *start = sc.get<uint32_t>(nc + 1),
             *fill = sc.get<uint32_t>(nc), *list = sc.get<uint32_t>(n), *pc = sc.get<uint32_t>(n),
             *off = sc.get<uint32_t>(n + 1);
    if (!rmax_bits || !outside || !key || !cnt || !start || !fill || !list || !pc || !off)
        return fail(ST_CUDA, "overlaps: out of device memory");
    const unsigned nb = blocks_of(n, STAT_THREADS);
    cudaError_t e = cudaMemsetAsync(rmax_bits, 0, 8, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(outside, 0, 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, nc * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(fill, 0, nc * 4, stream);
    if (e != cudaSuccess) return cuda_fail(e, "overlaps");
    k_rmax<<<nb, STAT_THREADS, 0, stream>>>(P, S, rmax_bits);
    k_ov_hash<<<nb, STAT_THREADS, 0, stream>>>(P, S, key, cnt, outside);
    k_scan_1block<<<1, 1024, 0, stream>>>(cnt, start, (uint32_t)nc);
    k_ov_fill<<<nb, STAT_THREADS, 0, stream>>>(P, key, start, fill, list);
    unsigned long long bits = 0;
    uint32_t nout = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, rmax_bits, 8, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nout, outside, 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "overlaps");
    if (nout) return fail(ST_OUTSIDE, "overlaps: a particle is outside the grid");
    double rmax;
    std::memcpy(&rmax, &bits, 8);
    // overlapping centres are closer than 2 r_max: search that many cells
    int reach[3];
    for (int d = 0; d < 3; ++d) {
        const double w = hs.L[d] / hs.num[d];
        double cells = std::ceil(2.0 * rmax / w);
        reach[d] = (int)std::min<double>(std::max(cells, 1.0), (double)hs.num[d]);
    }
    const int3 r3 = make_int3(reach[0], reach[1], reach[2]);
    k_ov_search<0><<<nb, STAT_THREADS, 0, stream>>>(P, S, key, start, list, r3, pc, nullptr, nullptr,
                                                    nullptr);
    k_scan_1block<<<1, 1024, 0, stream>>>(pc, off, (uint32_t)n);
    uint32_t total = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, off + n, 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "overlaps");
    *count = total;
    if (!pairs && !delta) return ST_OK;
    if (!pairs || !delta || cap < total) return fail(ST_ARG, "overlaps: output buffers hold fewer pairs than found");
    if (total == 0) return ST_OK;
    uint32_t *oj = sc.get<uint32_t>(total);
    double *od = sc.get<double>(total);
    if (!oj || !od) return fail(ST_CUDA, "overlaps: out of device memory");
    k_ov_search<1><<<nb, STAT_THREADS, 0, stream>>>(P, S, key, start, list, r3, nullptr, off, oj, od);
    std::vector<uint32_t> hj(total), hoff(n + 1);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(hj.data(), oj, total * 4ull, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(delta, od, total * 8ull, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hoff.data(), off, (n + 1) * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "overlaps");
    for (size_t i = 0; i < n; ++i)
        for (uint32_t q = hoff[i]; q < hoff[i + 1]; ++q) {
            pairs[2 * (size_t)q] = (uint32_t)i;
            pairs[2 * (size_t)q + 1] = hj[q];
        }
    return ST_OK;
}

}  // namespace sphb
