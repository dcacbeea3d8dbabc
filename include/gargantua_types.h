/*
 * Structs shared by the host and the sm_100a kernels.
 *
 * Every struct here is byte-identical to gargantua's ShaderTypes.h
 * (Sources/ShaderTypes/include/ShaderTypes.h:14-162), the C header its Swift
 * host and Metal shaders share, so a host that fills ShaderTypes structs can
 * hand them to this library unchanged. Field names, order, sizes and
 * alignments are kept; the static assertions at the end pin every size and
 * offset the host relies on.
 *
 * Apple's <simd/simd.h> vector types decide the layout: simd_float3 is 16
 * bytes with 16-byte alignment, simd_float2 and simd_uint2 are 8 bytes with
 * 8-byte alignment, simd_float4 is 16/16 and simd_float4x4 is 64/16. On
 * Apple platforms the real header is used; elsewhere the shim below gives
 * structs of exactly those sizes and alignments.
 *
 * A host that has already included its own ShaderTypes.h (its include
 * guard GARGANTUA_SHADER_TYPES_H is defined) keeps its types: the
 * definitions below are skipped, the library's entry points take the host's
 * structs by the same names, and the layout pins at the end check the
 * host's header instead. A Swift host importing both its ShaderTypes module
 * and this library's module then sees one set of types.
 */
#ifndef GARGANTUA_TYPES_H
#define GARGANTUA_TYPES_H

#include <stddef.h>
#include <stdint.h>

#ifndef GARGANTUA_SHADER_TYPES_H

#if defined(__APPLE__) && !defined(GG_FORCE_SIMD_SHIM)
#include <simd/simd.h>
#else
#if defined(_MSC_VER)
#define GG_ALIGNED(n) __declspec(align(n))
#else
#define GG_ALIGNED(n) __attribute__((aligned(n)))
#endif
typedef struct GG_ALIGNED(8) { float x, y; } simd_float2;
typedef struct GG_ALIGNED(16) { float x, y, z, pad_w; } simd_float3;
typedef struct GG_ALIGNED(16) { float x, y, z, w; } simd_float4;
typedef struct GG_ALIGNED(8) { uint32_t x, y; } simd_uint2;
typedef struct GG_ALIGNED(16) { simd_float4 columns[4]; } simd_float4x4;
#endif

/* ShaderTypes.h:8-12: a tightly packed three-float vector, 12 bytes. */
typedef struct { float x, y, z; } packed3;

/* ShaderTypes.h:14-20. One test particle, 32 bytes. */
typedef struct {
    packed3 position;
    packed3 velocity;
    float temperature;
    uint32_t respawns;
} Particle;

/* ShaderTypes.h:22-25. */
enum {
    PotentialNewtonian = 0,
    PotentialPaczynskiWiita = 1
};

/* ShaderTypes.h:27-36. */
typedef struct {
    simd_uint2 seed;
    uint32_t particleCount;
    uint32_t potential;
    uint32_t inverseCdfCount;
    float dt;
    float alpha;
    /* Peak temperature divided by the unnormalized profile at its peak. */
    float temperatureScale;
} SimUniforms;

/* ShaderTypes.h:38-48. Kept for layout compatibility; no kernel reads it. */
typedef struct {
    simd_float4x4 viewProjection;
    simd_float2 viewport;
    float pixelsPerUnit;
    float spriteRadius;
    float exposure;
    float peakTemperature;
    float padding0;
    float padding1;
} SpriteUniforms;

/* ShaderTypes.h:50-57. */
typedef struct {
    simd_float4 hudRect;
    float exposure;
    uint32_t hudVisible;
    uint32_t debugView;
    float driftBudget;
} PresentUniforms;

/* ShaderTypes.h:59-70. Geodesic integration policy. */
typedef struct {
    float stepFactor;
    float stepMin;
    float stepMax;
    float captureRadius;
    float escapeRadius;
    uint32_t stepCap;
    float emptyStepFactor;
    float emptyStepMax;
} GeodesicSettings;

/* ShaderTypes.h:72-76. */
enum {
    RayCaptured = 0,
    RayEscaped = 1,
    RayExhausted = 2
};

/* ShaderTypes.h:78-82. One ray integrated outside the image path. */
typedef struct {
    packed3 origin;
    packed3 direction;
} RayProbe;

/* ShaderTypes.h:84-92. */
typedef struct {
    packed3 position;
    packed3 direction;
    float drift;
    uint32_t outcome;
    uint32_t steps;
    float energy;
    float angularMomentum;
} RayProbeResult;

/* ShaderTypes.h:94-106. */
typedef struct {
    uint32_t volumeSize;
    uint32_t particleCount;
    float halfExtent;
    float peakTemperature;
    float emissionScale;
    /* Changes every frame; salts the stochastic deposit. */
    uint32_t frame;
    /* 1: all eight cloud-in-cell corners; 0: one corner picked per particle. */
    uint32_t exactDeposit;
    simd_uint2 seed;
} SplatUniforms;

/* ShaderTypes.h:108-144. */
typedef struct {
    simd_float3 cameraPosition;
    simd_float3 cameraRight;
    simd_float3 cameraUp;
    simd_float3 cameraForward;
    simd_float2 tanHalfFov;
    simd_uint2 resolution;
    simd_uint2 tileOrigin;
    float volumeHalfExtent;
    float opacityScale;
    float starBrightness;
    float driftBudget;
    uint32_t starSeed;
    uint32_t redshift;
    float bakeSpacing;
    uint32_t bakeCapacity;
    float sphereRadius;
    float cameraRadius;
    float sphereMaxB;
    float sphereTableMaxB;
    float cameraMaxB;
    float skyMinB;
    float skyMaxB;
    float spin;
    simd_float2 jitter;
    GeodesicSettings geodesic;
} MarchUniforms;

/* ShaderTypes.h:146-154. One baked ray's header. */
typedef struct {
    uint32_t count;
    uint32_t fallsIn;
    uint32_t directionXY;
    uint32_t directionZDepth;
} BakedRay;

/* ShaderTypes.h:156-162. Per-frame ray statistics. */
typedef struct {
    uint32_t rays;
    uint32_t overDriftBudget;
    uint32_t exhausted;
    uint32_t captured;
} MarchCounters;

#endif /* GARGANTUA_SHADER_TYPES_H */

/* Layout pins, the sizes and offsets ShaderTypes.h produces under Apple's
 * simd alignment rules. */
#if defined(__cplusplus)
#define GG_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define GG_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif
GG_STATIC_ASSERT(sizeof(packed3) == 12, "packed3");
GG_STATIC_ASSERT(sizeof(Particle) == 32, "Particle");
GG_STATIC_ASSERT(offsetof(Particle, temperature) == 24, "Particle.temperature");
GG_STATIC_ASSERT(sizeof(SimUniforms) == 32, "SimUniforms");
GG_STATIC_ASSERT(offsetof(SimUniforms, temperatureScale) == 28, "SimUniforms.temperatureScale");
GG_STATIC_ASSERT(sizeof(SpriteUniforms) == 96, "SpriteUniforms");
GG_STATIC_ASSERT(sizeof(PresentUniforms) == 32, "PresentUniforms");
GG_STATIC_ASSERT(sizeof(GeodesicSettings) == 32, "GeodesicSettings");
GG_STATIC_ASSERT(sizeof(RayProbe) == 24, "RayProbe");
GG_STATIC_ASSERT(sizeof(RayProbeResult) == 44, "RayProbeResult");
GG_STATIC_ASSERT(sizeof(SplatUniforms) == 40, "SplatUniforms");
GG_STATIC_ASSERT(offsetof(SplatUniforms, seed) == 32, "SplatUniforms.seed");
GG_STATIC_ASSERT(sizeof(MarchUniforms) == 192, "MarchUniforms");
GG_STATIC_ASSERT(offsetof(MarchUniforms, cameraRight) == 16, "MarchUniforms.cameraRight");
GG_STATIC_ASSERT(offsetof(MarchUniforms, cameraForward) == 48, "MarchUniforms.cameraForward");
GG_STATIC_ASSERT(offsetof(MarchUniforms, tanHalfFov) == 64, "MarchUniforms.tanHalfFov");
GG_STATIC_ASSERT(offsetof(MarchUniforms, resolution) == 72, "MarchUniforms.resolution");
GG_STATIC_ASSERT(offsetof(MarchUniforms, tileOrigin) == 80, "MarchUniforms.tileOrigin");
GG_STATIC_ASSERT(offsetof(MarchUniforms, volumeHalfExtent) == 88, "MarchUniforms.volumeHalfExtent");
GG_STATIC_ASSERT(offsetof(MarchUniforms, spin) == 148, "MarchUniforms.spin");
GG_STATIC_ASSERT(offsetof(MarchUniforms, jitter) == 152, "MarchUniforms.jitter");
GG_STATIC_ASSERT(offsetof(MarchUniforms, geodesic) == 160, "MarchUniforms.geodesic");
GG_STATIC_ASSERT(sizeof(BakedRay) == 16, "BakedRay");
GG_STATIC_ASSERT(sizeof(MarchCounters) == 16, "MarchCounters");

#endif
