// Device helpers shared by the kernels: the counter-based hash, the
// potential, small float3 arithmetic. Mirrors Sources/Gargantua/Shaders/Common.h.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "../../include/gargantua_constants.h"
#include "../../include/gargantua_types.h"

#define GG_PI_F 3.14159265358979323846f

namespace gg {

// pcg4d of Jarzynski and Olano 2020, JCGT 9(3), 20 (Common.h:11-17).
__host__ __device__ __forceinline__ uint4 pcg4d(uint4 v) {
    v.x = v.x * 1664525u + 1013904223u;
    v.y = v.y * 1664525u + 1013904223u;
    v.z = v.z * 1664525u + 1013904223u;
    v.w = v.w * 1664525u + 1013904223u;
    v.x += v.y * v.w;
    v.y += v.z * v.x;
    v.z += v.x * v.y;
    v.w += v.y * v.z;
    v.x ^= v.x >> 16;
    v.y ^= v.y >> 16;
    v.z ^= v.z >> 16;
    v.w ^= v.w >> 16;
    v.x += v.y * v.w;
    v.y += v.z * v.x;
    v.z += v.x * v.y;
    v.w += v.y * v.z;
    return v;
}

// Uniform in [0, 1) from the top 24 bits (Common.h:20-22).
__host__ __device__ __forceinline__ float unit_float(uint32_t x) {
    return (float)(x >> 8) * (1.0f / 16777216.0f);
}

// d Phi / d r (Common.h:32-38).
__device__ __forceinline__ float potential_gradient(float r, uint32_t potential) {
    if (potential == PotentialPaczynskiWiita) {
        float d = fmaxf(r - R_SCHWARZSCHILD, 1e-6f);
        return 1.0f / (d * d);
    }
    return 1.0f / (r * r);
}

__device__ __forceinline__ float circular_speed(float r, uint32_t potential) {
    return sqrtf(r * potential_gradient(r, potential));
}

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float length3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float3 normalize3(float3 a) { return a * (1.0f / length3(a)); }
__device__ __forceinline__ float3 abs3(float3 a) { return f3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }

__device__ __forceinline__ float3 to_f3(simd_float3 v) { return f3(v.x, v.y, v.z); }

// Blackbody table coordinate, log spaced (Common.h:56-59).
__device__ __forceinline__ float blackbody_coordinate(float temperature) {
    float t = fminf(fmaxf(temperature, BLACKBODY_T_MIN), BLACKBODY_T_MAX);
    return (logf(t) - logf(BLACKBODY_T_MIN)) / (logf(BLACKBODY_T_MAX) - logf(BLACKBODY_T_MIN));
}

// Linear, clamp-to-edge lookup of a table of `n` entries at normalized
// coordinate c, texel centres at (i + 0.5) / n, interpolated in FP32.
__device__ __forceinline__ float4 table_lookup4(const float4* table, int n, float c) {
    float x = c * (float)n - 0.5f;
    float fl = floorf(x);
    float f = x - fl;
    int i0 = (int)fl;
    int i1 = i0 + 1;
    i0 = min(max(i0, 0), n - 1);
    i1 = min(max(i1, 0), n - 1);
    float4 a = __ldg(table + i0), b = __ldg(table + i1);
    return make_float4(a.x + (b.x - a.x) * f, a.y + (b.y - a.y) * f, a.z + (b.z - a.z) * f, a.w + (b.w - a.w) * f);
}

__device__ __forceinline__ float table_lookup(const float* table, int n, float c) {
    float x = c * (float)n - 0.5f;
    float fl = floorf(x);
    float f = x - fl;
    int i0 = (int)fl;
    int i1 = i0 + 1;
    i0 = min(max(i0, 0), n - 1);
    i1 = min(max(i1, 0), n - 1);
    float a = __ldg(table + i0), b = __ldg(table + i1);
    return a + (b - a) * f;
}

__device__ __forceinline__ ushort4 pack_half4(float x, float y, float z, float w) {
    return make_ushort4(__half_as_ushort(__float2half_rn(x)), __half_as_ushort(__float2half_rn(y)),
                        __half_as_ushort(__float2half_rn(z)), __half_as_ushort(__float2half_rn(w)));
}

}  // namespace gg
