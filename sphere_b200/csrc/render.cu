// Ray-traced image of the particles: the reference's renderer
// (src/raytracer.cuh: imageInit, rayInitPerspective, rayIntersectSpheres,
// rayIntersectSpheresColormap, DEM::cameraInit, DEM::render;
// src/colorbar.h) as one kernel that writes a host RGBA buffer; the caller
// writes the PPM (DEM::writePPM, src/file_io.cpp:734-757).
//
// Every pixel casts one ray from the eye and tests every sphere in original
// order, keeping the first of equally near hits; a block stages the spheres
// in shared memory in chunks, so the spheres are read once per block rather
// than once per pixel.  The arithmetic is the reference's single precision
// in its order (this file is compiled with -fmad=false; vector lengths and
// normalisation use IEEE sqrtf and division), so the pixels equal a
// host restatement of the same formulas.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine_internal.h"
#include "dem_launch.h"

namespace sphb {

namespace {

constexpr int kRtThreads = 256;

struct F3 {
    float x, y, z;
};
__host__ __device__ inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__host__ __device__ inline F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ inline F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ inline F3 operator-(F3 a) { return f3(-a.x, -a.y, -a.z); }
__host__ __device__ inline F3 operator*(float s, F3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__host__ __device__ inline F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ inline F3 operator*(F3 a, F3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ inline F3 operator/(F3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__host__ __device__ inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline F3 cross(F3 a, F3 b)
{
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ inline float length(F3 v) { return sqrtf(dot(v, v)); }
__host__ __device__ inline F3 normalize(F3 v) { return v * (1.0f / sqrtf(dot(v, v))); }

// the blue-white-red colour map of src/colorbar.h
__device__ inline float cm_red(float r) { return fminf(1.0f, 0.209f * r * r * r - 2.49f * r * r + 3.0f * r + 0.0109f); }
__device__ inline float cm_green(float r) { return fminf(1.0f, -2.44f * r * r + 2.15f * r + 0.369f); }
__device__ inline float cm_blue(float r) { return fminf(1.0f, -2.21f * r * r + 1.61f * r + 0.573f); }

struct Camera {
    F3 u, v, w, eye, light;
    float d;
    float plane[4];   // image plane extent (x0, x1, y0, y1)
    unsigned width, height;
};

// Per-particle render data in ORIGINAL order: position and radius in FP32,
// the colour-map value (FP64) and the fixvel flag.
__global__ void k_render_prep(DevParams P, DevState S, int method, float4 *xr, double *val,
                              float *fixvel)
{
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P.np) return;
    const unsigned o = S.orig_of[k];
    const double4 x = S.x[k];
    xr[o] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)x.w);
    const double4 v = S.vel[k];
    fixvel[o] = (float)v.w;
    double a = 0.0;
    if (method == 1) {
        a = S.p[k];
    } else if (method == 2) {
        a = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    } else if (method == 3) {
        const double4 w = S.angvel[k];
        a = sqrt(w.x * w.x + w.y * w.y + w.z * w.z);
    } else if (method == 4) {
        a = S.xyzsum[k].x;
    } else if (method == 5) {
        const double4 r = S.angpos[k];
        a = sqrt(r.x * r.x + r.y * r.y + r.z * r.z);
    }
    val[o] = a;
}

// One pixel per thread.  method 0: Lambertian shading; 1..5: the colour map
// of val / max_val (fixed particles grey; with lower_cutoff > 0 only free
// particles above the cutoff are hit).
__global__ void __launch_bounds__(kRtThreads) k_render(Camera C, const float4 *xr, const double *val,
                                                     const float *fixvel, unsigned np, int method,
                                                     float max_val, float lower_cutoff, uchar4 *img)
{
    __shared__ float4 sx[kRtThreads];
    __shared__ float sv[kRtThreads], sf[kRtThreads];
    const unsigned pixels = C.width * C.height;
    const unsigned mempos = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = mempos < pixels;
    // rayInitPerspective
    const unsigned i = active ? mempos % C.width : 0u;
    const unsigned j = active ? (unsigned)(int)floorf((float)mempos / C.width) % C.width : 0u;
    const float p_u = C.plane[0] + (C.plane[1] - C.plane[0]) * (i + 0.5f) / C.width;
    const float p_v = C.plane[2] + (C.plane[3] - C.plane[2]) * (j + 0.5f) / C.height;
    const F3 e = C.eye;
    const F3 d = (-C.d) * C.w + p_u * C.u + p_v * C.v;
    float tdist = 1e10f;
    F3 n = f3(0.f, 0.f, 0.f);
    unsigned hitidx = 0;
    const bool cut = lower_cutoff > 0.0;
    for (unsigned base = 0; base < np; base += kRtThreads) {
        const unsigned m = min((unsigned)kRtThreads, np - base);
        __syncthreads();
        if (threadIdx.x < m) {
            sx[threadIdx.x] = xr[base + threadIdx.x];
            if (method != 0) {
                sv[threadIdx.x] = (float)val[base + threadIdx.x];
                sf[threadIdx.x] = fixvel[base + threadIdx.x];
            }
        }
        __syncthreads();
        if (!active) continue;
        for (unsigned q = 0; q < m; ++q) {
            const float4 x = sx[q];
            const F3 c = f3(x.x, x.y, x.z);
            const float R = x.w;
            const F3 ec = e - c;
            const float Delta = (2.0f * dot(d, ec)) * (2.0f * dot(d, ec)) -
                                4.0f * dot(d, d) * (dot(ec, ec) - R * R);
            bool take = Delta > 0.0f;
            if (method != 0 && cut) take = take && sv[q] > lower_cutoff && sf[q] == 0.f;
            if (take) {
                const float t_minus =
                    (dot(-d, ec) - sqrtf(dot(d, ec) * dot(d, ec) - dot(d, d) * (dot(ec, ec) - R * R))) /
                    dot(d, d);
                if (fabsf(t_minus) < tdist) {
                    const F3 p = e + t_minus * d;
                    tdist = fabsf(t_minus);
                    n = normalize(2.0f * (p - c));
                    hitidx = base + q;
                }
            }
        }
    }
    if (!active) return;
    uchar4 out = make_uchar4(255, 255, 255, 255);   // imageInit: white background
    if (tdist < 1e10f) {
        const float dotprod = fmaxf(0.0f, dot(n, C.light));
        const float I_d = 40.0f, k_d = 5.0f, k_a = 10.0f, I_a = 5.0f;
        const float shade = k_d * I_d * dotprod + k_a * I_a;
        if (method == 0) {
            out.x = (unsigned char)(shade * 0.48f);
            out.y = (unsigned char)(shade * 0.41f);
            out.z = (unsigned char)(shade * 0.27f);
        } else {
            float ratio = (float)(val[hitidx] / (double)max_val);
            if (ratio < 0.01f) ratio = 0.01f;
            if (ratio > 0.99f) ratio = 0.99f;
            float r = cm_red(ratio), g = cm_green(ratio), b = cm_blue(ratio);
            if (fixvel[hitidx] > 0.f) r = g = b = 0.5f;
            out.x = (unsigned char)(shade * r);
            out.y = (unsigned char)(shade * g);
            out.z = (unsigned char)(shade * b);
        }
    }
    img[mempos] = out;
}

}  // namespace

int Engine::render(int method, float max_val, float lower_cutoff, unsigned width, unsigned height,
                   unsigned char *rgba)
{
    if (!rgba || width == 0 || height == 0 || method < 0 || method > 5)
        return fail(ST_ARG, "render: bad arguments");
    if ((size_t)width * height > (1u << 26)) return fail(ST_ARG, "render: image too large");
    int rc = poll_errors("render");
    if (rc < 0 && rc != ST_OUTSIDE && rc != ST_CAPACITY) return rc;
    const size_t n = hs.np;
    // camera (DEM::render + DEM::cameraInit): the largest coordinates of the
    // particles (from 0), the reference's eye and look-at points
    std::vector<double> xs(n * 4);
    if (n && (rc = get(SPH_F_X, xs.data(), xs.size() * 8))) return rc;
    double mx = 0.0, my = 0.0, mz = 0.0;
    for (size_t i = 0; i < n; ++i) {
        mx = std::max(mx, xs[4 * i]);
        my = std::max(my, xs[4 * i + 1]);
        mz = std::max(mz, xs[4 * i + 2]);
    }
    Camera C{};
    C.width = width;
    C.height = height;
    const float imgw = (float)(hs.L[0] * 1.35f);
    const F3 lookat = f3((float)mx, (float)my, (float)mz) / 2.0f;
    const F3 eye = f3((float)(hs.L[0] * 2.3f), (float)(hs.L[1] * -5.0f), (float)(hs.L[2] * 1.3f));
    const float hw_ratio = (float)(height / width);   // integer division, as the reference
    C.plane[0] = -0.5f * imgw;
    C.plane[1] = 0.5f * imgw;
    C.plane[2] = -0.5f * imgw * hw_ratio;
    C.plane[3] = 0.5f * imgw * hw_ratio;
    const F3 view = eye - lookat;
    const F3 up = f3(0.0f, 0.0f, 1.0f);
    C.w = -view / length(view);
    C.u = cross(up, C.w) / length(cross(up, C.w));
    C.v = cross(C.w, C.u);
    C.eye = eye;
    C.d = length(view) * 0.8f;
    C.light = normalize(-1.0f * eye * f3(1.0f, 0.2f, 0.6f));

    float4 *xr = nullptr;
    double *val = nullptr;
    float *fixv = nullptr;
    uchar4 *img = nullptr;
    const size_t pixels = (size_t)width * height;
    cudaError_t e = cudaSuccess;
    auto cleanup = [&]() {
        cudaFree(xr);
        cudaFree(val);
        cudaFree(fixv);
        cudaFree(img);
    };
    if ((e = cudaMalloc(&xr, std::max<size_t>(n, 1) * 16)) != cudaSuccess ||
        (e = cudaMalloc(&val, std::max<size_t>(n, 1) * 8)) != cudaSuccess ||
        (e = cudaMalloc(&fixv, std::max<size_t>(n, 1) * 4)) != cudaSuccess ||
        (e = cudaMalloc(&img, pixels * 4)) != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "render");
    }
    if (n) k_render_prep<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(P, S, method, xr, val, fixv);
    k_render<<<(unsigned)((pixels + kRtThreads - 1) / kRtThreads), kRtThreads, 0, stream>>>(
        C, xr, val, fixv, (unsigned)n, method, max_val, lower_cutoff, img);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(rgba, img, pixels * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cleanup();
    if (e != cudaSuccess) return cuda_fail(e, "render");
    return ST_OK;
}

}  // namespace sphb
