/* Self-written stand-in for the vector-operator header the reference
 * downloads at build time (src/CMakeLists.txt:11-13) -- TEST
 * INFRASTRUCTURE ONLY.  Only the operators the host build needs: the int3
 * sum (in ref_shim.h) and the float3 arithmetic of the ray tracer
 * (src/raytracer.cuh), in their host forms (normalisation by one division
 * by the square root). */
#ifndef REF_SHIM_HELPER_MATH_H_
#define REF_SHIM_HELPER_MATH_H_
#include "ref_shim.h"

inline float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
inline float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(float3 v) { return std::sqrt(dot(v, v)); }
inline float3 normalize(float3 v)
{
    float inv = 1.0f / std::sqrt(dot(v, v));
    return v * inv;
}
inline float3 cross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float4 make_float4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
#endif
