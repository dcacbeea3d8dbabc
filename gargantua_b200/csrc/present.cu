// Present, reduced to its arithmetic (present.metal:22-58): exposure, the
// Khronos PBR Neutral tone curve, sRGB encoding into a headless 8-bit RGBA
// buffer, or the drift heat map of the debug target. Also the blackbody
// colour table the kernels sample and the host PNG writer that stands in for
// Capture.writePNG.
#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "runtime.h"

namespace gg {

int blackbody_init(gg_context* ctx) {
    // Blackbody.table in FP64, stored as half like the reference's rgba16f
    // table (ParticleSystem.swift:28-47), widened to float4 for FP32 lookups.
    std::vector<double> rgb(3 * BLACKBODY_TABLE_SIZE);
    blackbody_table(BLACKBODY_TABLE_SIZE, BLACKBODY_T_MIN, BLACKBODY_T_MAX, rgb.data());
    std::vector<float4> table(BLACKBODY_TABLE_SIZE);
    for (uint32_t k = 0; k < BLACKBODY_TABLE_SIZE; ++k) {
        table[k] = make_float4(__half2float(__double2half(rgb[3 * k + 0])), __half2float(__double2half(rgb[3 * k + 1])),
                               __half2float(__double2half(rgb[3 * k + 2])), 1.0f);
    }
    GG_CHECK(device_alloc(ctx, BLACKBODY_TABLE_SIZE * sizeof(float4), (void**)&ctx->blackbody, "blackbody table"));
    GG_CUDA(cudaMemcpyAsync(ctx->blackbody, table.data(), table.size() * sizeof(float4), cudaMemcpyHostToDevice,
                            ctx->stream),
            "blackbody table upload");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "blackbody table upload");
    return GG_OK;
}

// Khronos PBR Neutral tone mapper (Khronos Group 2024, PBR Neutral Tone
// Mapper Specification; present.metal:22-35).
__device__ __forceinline__ float3 pbr_neutral(float3 c) {
    const float start = 0.8f - 0.04f;
    const float desat = 0.15f;
    float x = fminf(c.x, fminf(c.y, c.z));
    float offset = x < 0.08f ? x - 6.25f * x * x : 0.04f;
    c = make_float3(c.x - offset, c.y - offset, c.z - offset);
    float peak = fmaxf(c.x, fmaxf(c.y, c.z));
    if (peak < start) return c;
    const float d = 1.0f - start;
    float np = 1.0f - d * d / (peak + d - start);
    float s = np / peak;
    c = make_float3(c.x * s, c.y * s, c.z * s);
    float g = 1.0f - 1.0f / (desat * (peak - np) + 1.0f);
    return make_float3(c.x + (np - c.x) * g, c.y + (np - c.y) * g, c.z + (np - c.z) * g);
}

// Drift heat map (present.metal:40-46).
__device__ __forceinline__ float3 drift_heat(float4 d, float budget) {
    float t = fminf(fmaxf(d.x / budget, 0.0f), 2.0f) * 0.5f;
    float3 heat = make_float3(t, 1.0f - fabsf(t - 0.5f) * 2.0f, 1.0f - t);
    float shade = 0.2f + 0.8f * fminf(fmaxf(d.y / (float)STEP_CAP_INTERACTIVE, 0.0f), 1.0f);
    if (d.z < 0.5f) shade *= 0.35f;
    return make_float3(heat.x * shade, heat.y * shade, heat.z * shade);
}

// Linear to 8-bit sRGB (IEC 61966-2-1 transfer function), as the
// bgra8Unorm_srgb drawable encodes on store (Renderer.swift:66).
__device__ __forceinline__ uint8_t srgb8(float v) {
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    float e = v <= 0.0031308f ? 12.92f * v : 1.055f * powf(v, 1.0f / 2.4f) - 0.055f;
    return (uint8_t)__float2int_rn(e * 255.0f);
}

__device__ __forceinline__ float4 unpack4(ushort4 h) {
    return make_float4(__half2float(__ushort_as_half(h.x)), __half2float(__ushort_as_half(h.y)),
                       __half2float(__ushort_as_half(h.z)), __half2float(__ushort_as_half(h.w)));
}

__device__ __forceinline__ float half_round(float x) { return __half2float(__float2half_rn(x)); }

__global__ void tonemap_kernel(const ushort4* __restrict__ hdr, const ushort4* __restrict__ debug, PresentUniforms u,
                               uint32_t count, uchar4* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float3 c;
    if (u.debugView != 0u) {
        c = drift_heat(unpack4(debug[i]), u.driftBudget);
    } else {
        float4 h = unpack4(hdr[i]);
        c = pbr_neutral(make_float3(fmaxf(h.x * u.exposure, 0.0f), fmaxf(h.y * u.exposure, 0.0f),
                                    fmaxf(h.z * u.exposure, 0.0f)));
    }
    // The fragment returns half4 before the store encodes it.
    out[i] = make_uchar4(srgb8(half_round(c.x)), srgb8(half_round(c.y)), srgb8(half_round(c.z)), 255);
}

}  // namespace gg

using namespace gg;

static void put32(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back((uint8_t)(x >> 24));
    v.push_back((uint8_t)(x >> 16));
    v.push_back((uint8_t)(x >> 8));
    v.push_back((uint8_t)x);
}

static void chunk(std::vector<uint8_t>& png, const char* type, const uint8_t* data, uint32_t n) {
    put32(png, n);
    size_t start = png.size();
    png.insert(png.end(), type, type + 4);
    png.insert(png.end(), data, data + n);
    uLong crc = crc32(0L, png.data() + start, (uInt)(n + 4));
    put32(png, (uint32_t)crc);
}

extern "C" {

GG_API int gg_tonemap(gg_targets* t, const PresentUniforms* u, uint8_t* rgba8) {
    gg::Range range("gg_tonemap");
    if (!t || !u || !rgba8) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_tonemap needs targets, uniforms and an output.");
    gg_context* ctx = t->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint32_t count = t->width * t->height;
    // The 8-bit image's device buffer stays with the targets (freed with
    // them), so a frame loop's tone maps allocate nothing after the first.
    if (!t->srgb) GG_CHECK(gg::device_alloc(ctx, (uint64_t)count * 4u, (void**)&t->srgb, "tone-mapped image"));
    tonemap_kernel<<<(count + 255u) / 256u, 256, 0, ctx->stream>>>(t->color, t->debug, *u, count, t->srgb);
    GG_CHECK(gg::launch_status("tone map"));
    GG_CUDA(cudaMemcpyAsync(rgba8, t->srgb, (size_t)count * 4u, cudaMemcpyDeviceToHost, ctx->stream),
            "tone map readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "tone map");
    return GG_OK;
}

GG_API int gg_write_png(const char* path, const uint8_t* rgba8, uint32_t width, uint32_t height) {
    if (!path || !rgba8 || width == 0 || height == 0)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_write_png needs a path, pixels and a size.");
    std::vector<uint8_t> raw;
    raw.reserve((size_t)height * (1 + 4 * (size_t)width));
    for (uint32_t y = 0; y < height; ++y) {
        raw.push_back(0);  // filter: none
        const uint8_t* row = rgba8 + (size_t)y * width * 4u;
        raw.insert(raw.end(), row, row + (size_t)width * 4u);
    }
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<uint8_t> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK)
        return gg::fail(GG_ERR_OUT_OF_MEMORY, "PNG compression failed.");
    std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    uint8_t ihdr[13];
    std::vector<uint8_t> tmp;
    put32(tmp, width);
    put32(tmp, height);
    for (int i = 0; i < 8; ++i) ihdr[i] = tmp[i];
    ihdr[8] = 8;   // bit depth
    ihdr[9] = 6;   // RGBA
    ihdr[10] = 0;  // deflate
    ihdr[11] = 0;  // adaptive filtering
    ihdr[12] = 0;  // no interlace
    chunk(png, "IHDR", ihdr, 13);
    uint8_t srgb = 0;  // sRGB chunk, perceptual intent
    chunk(png, "sRGB", &srgb, 1);
    chunk(png, "IDAT", z.data(), (uint32_t)zlen);
    chunk(png, "IEND", nullptr, 0);
    FILE* f = std::fopen(path, "wb");
    if (!f) return gg::fail(GG_ERR_INVALID_ARGUMENT, "Could not open %s for writing.", path);
    size_t w = std::fwrite(png.data(), 1, png.size(), f);
    int closed = std::fclose(f);
    if (w != png.size() || closed != 0) return gg::fail(GG_ERR_DEVICE, "Could not write the PNG to %s.", path);
    return GG_OK;
}

GG_API int gg_context_blackbody(gg_context* ctx, float* rgba, uint32_t count) {
    if (!ctx || !rgba || count != BLACKBODY_TABLE_SIZE)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_context_blackbody needs %u float4 entries.", BLACKBODY_TABLE_SIZE);
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    GG_CUDA(cudaMemcpyAsync(rgba, ctx->blackbody, count * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream),
            "blackbody readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "blackbody readback");
    return GG_OK;
}

}  // extern "C"
