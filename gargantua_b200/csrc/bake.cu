// Bake strategy (bake.metal:1-144, BakePass.swift:8-102): for a camera that
// holds still each ray's in-slab sample points are integrated once and stored
// as half4 (position, path length since the previous stored sample), at
// least bakeSpacing apart and at most bakeCapacity per ray, with a 16-byte
// header; each later frame walks the stored samples through the current
// volume.
//
// Sample layout: ray-major, BAKE_SAMPLES half4 per ray, ray index
// y * width + x (BakePass.swift:35). A ray's samples are one contiguous
// 768-byte run that the walk streams front to back.
#include "march.cuh"
#include "runtime.h"

namespace gg {

__device__ __forceinline__ uint32_t pack_half2(float a, float b) {
    return (uint32_t)__half_as_ushort(__float2half_rn(a)) | ((uint32_t)__half_as_ushort(__float2half_rn(b)) << 16);
}

__device__ __forceinline__ float2 unpack_half2(uint32_t v) {
    return make_float2(__half2float(__ushort_as_half((unsigned short)(v & 0xffffu))),
                       __half2float(__ushort_as_half((unsigned short)(v >> 16))));
}

struct BakeArgs {
    MarchParams p;
    ushort4* samples;
    BakedRay* headers;
    uint32_t* overflow;
    uint32_t rows;
    // Optional (NULL: not kept): [0] += RK4 steps, [5] += rays that ran out
    // of steps, [6] += captured rays (a served request's counter words).
    unsigned long long* stats;
};

// bakeRays (bake.metal:17-92).
__global__ void __launch_bounds__(64) bake_kernel(BakeArgs a) {
    const MarchUniforms& u = a.p.u;
    const uint32_t gx = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gy >= a.rows) return;
    const uint32_t px = u.tileOrigin.x + gx, py = u.tileOrigin.y + gy;
    if (px >= u.resolution.x || py >= u.resolution.y) return;
    const uint32_t index = py * u.resolution.x + px;
    ushort4* slot = a.samples + (uint64_t)index * u.bakeCapacity;
    // Pixel centre, no jitter (bake.metal:30-33).
    float sx = (float)px + 0.5f, sy = (float)py + 0.5f;
    float nx = (2.0f * sx / (float)u.resolution.x - 1.0f) * u.tanHalfFov.x;
    float ny = (1.0f - 2.0f * sy / (float)u.resolution.y) * u.tanHalfFov.y;
    float3 dir = normalize3(to_f3(u.cameraForward) + nx * to_f3(u.cameraRight) + ny * to_f3(u.cameraUp));
    PreparedRay<float> prepared = prepare_ray(to_v3<float>(to_f3(u.cameraPosition)), to_v3<float>(dir), u, a.p.tables);
    uint32_t steps = 0;
    uint32_t outcome = RayEscaped;
    // Per-warp sums of the served request's counters, taken by the threads
    // still running (sky-only rays count as escaped with no steps).
    auto count = [&] {
        if (!a.stats) return;
        const unsigned mask = __activemask();
        const uint32_t s = __reduce_add_sync(mask, steps);
        const uint32_t e = __reduce_add_sync(mask, outcome == RayExhausted ? 1u : 0u);
        const uint32_t c = __reduce_add_sync(mask, outcome == RayCaptured ? 1u : 0u);
        if ((uint32_t)(__ffs(mask) - 1) == (threadIdx.x + threadIdx.y * blockDim.x) % 32u) {
            if (s) atomicAdd(&a.stats[0], (unsigned long long)s);
            if (e) atomicAdd(&a.stats[5], (unsigned long long)e);
            if (c) atomicAdd(&a.stats[6], (unsigned long long)c);
        }
    };
    if (prepared.skyOnly) {
        BakedRay h;
        h.count = 0u;
        h.fallsIn = 0u;
        h.directionXY = pack_half2(prepared.sky.x, prepared.sky.y);
        h.directionZDepth = pack_half2(prepared.sky.z, 1.0f);
        a.headers[index] = h;
        count();
        return;
    }
    PlaneRay<float> ray = prepared.ray;
    const GeodesicSettings& g = u.geodesic;
    V3<float> previous = ray_position(ray);
    float since = 0.0f, travelled = 0.0f, first_depth = -1.0f;
    uint32_t stored = 0;
    bool overflowed = false, left_sphere = false;
    outcome = RayExhausted;
    const float sphere = u.sphereRadius;
    for (uint32_t k = 0; k < STEP_CAP_STILL; ++k) {
        if (k >= g.stepCap) break;
        float h = ray_step_length(previous.z, ray.s.r, g);
        RayState<float> before = ray.s;
        ray.s = ray_step(ray.s, h);
        steps += 1u;
        if (sphere > 0.0f && ray.s.r >= sphere && ray.s.rDot > 0.0f && before.r < sphere)
            ray.s = ray_step(before, h * (sphere - before.r) / (ray.s.r - before.r));
        V3<float> position = ray_position(ray);
        float path = length(position - previous);
        since += path;
        travelled += path;
        previous = position;
        if (ray.s.r <= g.captureRadius) {
            outcome = RayCaptured;
            break;
        }
        float3 pf = to_float3(position);
        if (in_slab(pf, u.volumeHalfExtent) && since >= u.bakeSpacing) {
            if (stored < u.bakeCapacity) {
                slot[stored] = pack_half4(pf.x, pf.y, pf.z, since);
                stored += 1u;
                if (first_depth < 0.0f) first_depth = travelled;
            } else {
                overflowed = true;
            }
            since = 0.0f;
        }
        if (sphere > 0.0f && ray.s.r >= sphere && ray.s.rDot > 0.0f) {
            outcome = RayEscaped;
            left_sphere = true;
            break;
        }
        if (ray.s.r >= g.escapeRadius) {
            outcome = RayEscaped;
            break;
        }
    }
    bool falls_in = ray_falls_in(ray, outcome);
    V3<float> fin = left_sphere ? sphere_exit_direction(ray, u, a.p.tables) : ray_direction(ray);
    float depth = first_depth >= 0.0f ? first_depth : travelled;
    BakedRay hd;
    hd.count = stored;
    hd.fallsIn = falls_in ? 1u : 0u;
    hd.directionXY = pack_half2(fin.x, fin.y);
    hd.directionZDepth = pack_half2(fin.z, fminf(depth / (2.0f * R_ESCAPE), 1.0f));
    a.headers[index] = hd;
    if (overflowed) atomicAdd(a.overflow, 1u);
    count();
}

struct WalkArgs {
    MarchParams p;
    const ushort4* samples;
    const BakedRay* headers;
};

__device__ __forceinline__ float half_bits(unsigned short b) { return __half2float(__ushort_as_half(b)); }

// walkRays (bake.metal:94-144): front-to-back compositing over the stored
// samples with the redshift factor, then the starfield for rays that do not
// fall in.
__global__ void __launch_bounds__(64) walk_kernel(WalkArgs a) {
    const MarchUniforms& u = a.p.u;
    const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= u.resolution.x || py >= u.resolution.y) return;
    const uint32_t index = py * u.resolution.x + px;
    BakedRay header = a.headers[index];
    const ushort4* slot = a.samples + (uint64_t)index * u.bakeCapacity;
    float3 color = make_float3(0.0f, 0.0f, 0.0f);
    float transmittance = 1.0f;
    float3 previous = to_f3(u.cameraPosition);
    const bool gas = a.p.emission != 0;
    const float inv = 1.0f / (2.0f * u.volumeHalfExtent);
    for (uint32_t k = 0; k < BAKE_SAMPLES; ++k) {
        if (k >= header.count || k >= u.bakeCapacity || transmittance <= 0.004f) break;
        ushort4 stored = slot[k];
        float3 position = make_float3(half_bits(stored.x), half_bits(stored.y), half_bits(stored.z));
        float path = half_bits(stored.w);
        if (gas) {
            float ux = (position.x + u.volumeHalfExtent) * inv, uy = (position.y + u.volumeHalfExtent) * inv,
                  uz = (position.z + u.volumeHalfExtent) * inv;
            float4 e = tex3D<float4>(a.p.emission, ux, uy, uz);
            if (e.w > 0.0f) {
                float3 direction = normalize3(position - previous);
                float g3 = 1.0f;
                if (u.redshift != 0u) {
                    float4 v = tex3D<float4>(a.p.velocity, ux, uy, uz);
                    float g = redshift_factor(1.0f - R_SCHWARZSCHILD / length3(position), direction,
                                              make_float3(v.x, v.y, v.z));
                    g3 = g * g * g;
                }
                float alpha = 1.0f - expf(-u.opacityScale * e.w * path);
                float kk = transmittance * g3 * path;
                color = color + make_float3(e.x * kk, e.y * kk, e.z * kk);
                transmittance *= 1.0f - alpha;
            }
        }
        previous = position;
    }
    if (header.fallsIn == 0u && u.starBrightness > 0.0f) {
        float2 xy = unpack_half2(header.directionXY);
        float2 zd = unpack_half2(header.directionZDepth);
        float3 d = normalize3(make_float3(xy.x, xy.y, zd.x));
        color = color + starfield(d, u.starSeed, a.p.blackbody) * (transmittance * u.starBrightness);
    }
    a.p.color[index] = pack_half4(color.x, color.y, color.z, 1.0f);
    if (a.p.depth) a.p.depth[index] = unpack_half2(header.directionZDepth).y;
    if (a.p.motion) a.p.motion[index] = make_ushort2(0, 0);
}

MarchParams make_params(gg_context* ctx, const gg_volume* vol, const MarchUniforms& u, const gg_sweep* sweep);
int check_uniforms(gg_context* ctx, const MarchUniforms* u, const char* what);

// A served bake request (the server's GG_REQUEST_BAKE): every row baked with
// `bake` (its tables, spacing and capacity set), then walked through
// `walk`'s volume into walk.color, on `stream`. stats: the request's
// counter words (see BakeArgs), or NULL.
int launch_bake_walk(const MarchParams& bake, const MarchParams& walk, ushort4* samples, BakedRay* headers,
                     uint32_t* overflow, unsigned long long* stats, cudaStream_t stream) {
    BakeArgs b{};
    b.p = bake;
    b.p.u.tileOrigin.x = 0;
    b.p.u.tileOrigin.y = 0;
    b.samples = samples;
    b.headers = headers;
    b.overflow = overflow;
    b.rows = bake.u.resolution.y;
    b.stats = stats;
    dim3 block(MARCH_THREADGROUP_WIDTH, MARCH_THREADGROUP_HEIGHT);
    dim3 grid((bake.u.resolution.x + block.x - 1) / block.x, (b.rows + block.y - 1) / block.y);
    bake_kernel<<<grid, block, 0, stream>>>(b);
    GG_CHECK(launch_status("served bake"));
    WalkArgs w{};
    w.p = walk;
    w.samples = samples;
    w.headers = headers;
    walk_kernel<<<grid, block, 0, stream>>>(w);
    return launch_status("served walk");
}

}  // namespace gg

using namespace gg;

extern "C" {

GG_API int gg_bake_create(gg_context* ctx, uint32_t width, uint32_t height, gg_bake** out) {
    if (!ctx || !out) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_bake_create needs a context and an output.");
    *out = nullptr;
    if (width == 0 || height == 0 || width > 16384 || height > 16384)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Bake size %ux%u is outside 1..16384.", width, height);
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t px = (uint64_t)width * height;
    gg_bake* b = new gg_bake();
    b->ctx = ctx;
    b->width = width;
    b->height = height;
    int s = gg::device_alloc(ctx, px * BAKE_SAMPLES * 8u, (void**)&b->samples, "bake samples");
    if (s == GG_OK) s = gg::device_alloc(ctx, px * 16u, (void**)&b->headers, "bake headers");
    if (s == GG_OK) s = gg::device_alloc(ctx, 4u, (void**)&b->overflow, "bake overflow");
    if (s == GG_OK) s = gg::cuda_status(cudaMemsetAsync(b->overflow, 0, 4u, ctx->stream), "bake overflow reset");
    if (s == GG_OK) s = gg::cuda_status(cudaMemsetAsync(b->headers, 0, px * 16u, ctx->stream), "bake header reset");
    b->bytes = px * BAKE_SAMPLES * 8u + px * 16u + 4u;
    if (s != GG_OK) {
        gg_bake_destroy(b);
        return s;
    }
    *out = b;
    return GG_OK;
}

GG_API void gg_bake_destroy(gg_bake* b) {
    if (!b) return;
    gg_context* ctx = b->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    const uint64_t px = (uint64_t)b->width * b->height;
    gg::device_free(ctx, b->samples, px * BAKE_SAMPLES * 8u);
    gg::device_free(ctx, b->headers, px * 16u);
    gg::device_free(ctx, b->overflow, 4u);
    delete b;
}

GG_API int gg_bake_rows(gg_bake* b, const MarchUniforms* u, uint32_t row_begin, uint32_t row_end) {
    gg::Range range("gg_bake_rows");
    if (!b) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_bake_rows needs a bake.");
    gg_context* ctx = b->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    GG_CHECK(gg::check_uniforms(ctx, u, "gg_bake_rows"));
    if (u->spin != 0.0f)
        return gg::fail(GG_ERR_UNSUPPORTED, "The bake strategy is Schwarzschild only; spin %g was given.", (double)u->spin);
    if (u->resolution.x != b->width || u->resolution.y != b->height)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Uniforms give %ux%u but the bake is %ux%u.", u->resolution.x,
                        u->resolution.y, b->width, b->height);
    if (u->bakeCapacity > BAKE_SAMPLES || u->bakeCapacity == 0)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Bake capacity %u is outside 1..%u.", u->bakeCapacity, BAKE_SAMPLES);
    if (row_begin >= row_end || row_end > b->height)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Bake rows [%u, %u) are not inside 0..%u.", row_begin, row_end, b->height);
    BakeArgs a{};
    a.p = gg::make_params(ctx, nullptr, *u, &ctx->sweep);
    a.p.u.tileOrigin.x = 0;
    a.p.u.tileOrigin.y = row_begin;
    a.samples = b->samples;
    a.headers = b->headers;
    a.overflow = b->overflow;
    a.rows = row_end - row_begin;
    dim3 block(MARCH_THREADGROUP_WIDTH, MARCH_THREADGROUP_HEIGHT);
    dim3 grid((b->width + block.x - 1) / block.x, (a.rows + block.y - 1) / block.y);
    bake_kernel<<<grid, block, 0, ctx->stream>>>(a);
    return gg::launch_status("bake rows");
}

GG_API int gg_bake_overflow(gg_bake* b, uint32_t* count, int reset) {
    if (!b || !count) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_bake_overflow needs a bake and an output.");
    gg_context* ctx = b->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    GG_CUDA(cudaMemcpyAsync(count, b->overflow, 4u, cudaMemcpyDeviceToHost, ctx->stream), "overflow readback");
    if (reset) GG_CUDA(cudaMemsetAsync(b->overflow, 0, 4u, ctx->stream), "overflow reset");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "overflow readback");
    return GG_OK;
}

GG_API int gg_walk(gg_bake* b, const gg_volume* vol, const MarchUniforms* u, gg_targets* targets) {
    gg::Range range("gg_walk");
    if (!b || !u || !targets) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_walk needs a bake, uniforms and targets.");
    gg_context* ctx = b->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (targets->width != b->width || targets->height != b->height || u->resolution.x != b->width ||
        u->resolution.y != b->height)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_walk: targets, uniforms and bake must share one size.");
    if (u->bakeCapacity > BAKE_SAMPLES)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Bake capacity %u exceeds %u.", u->bakeCapacity, BAKE_SAMPLES);
    WalkArgs a{};
    a.p = gg::make_params(ctx, vol, *u, nullptr);
    a.p.color = targets->color;
    a.p.depth = targets->depth;
    a.p.motion = targets->motion;
    a.samples = b->samples;
    a.headers = b->headers;
    dim3 block(MARCH_THREADGROUP_WIDTH, MARCH_THREADGROUP_HEIGHT);
    dim3 grid((b->width + block.x - 1) / block.x, (b->height + block.y - 1) / block.y);
    walk_kernel<<<grid, block, 0, ctx->stream>>>(a);
    return gg::launch_status("walk");
}

GG_API int gg_bake_read(gg_bake* b, uint16_t* samples_half4, BakedRay* headers) {
    if (!b) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_bake_read needs a bake.");
    gg_context* ctx = b->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t px = (uint64_t)b->width * b->height;
    if (samples_half4)
        GG_CUDA(cudaMemcpyAsync(samples_half4, b->samples, px * BAKE_SAMPLES * 8u, cudaMemcpyDeviceToHost, ctx->stream),
                "bake readback");
    if (headers) GG_CUDA(cudaMemcpyAsync(headers, b->headers, px * 16u, cudaMemcpyDeviceToHost, ctx->stream), "bake readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "bake readback");
    return GG_OK;
}

}  // extern "C"
