// Image march and probe kernels (march.metal:194-341) and their entry points.
//
// The image kernel is one thread per pixel in 8x8 blocks, the shape of the
// reference's dispatch (MarchPass.swift:101); it is the plain per-request
// path. With GG_PRECISION_COMPENSATED the state update is TwoSum-compensated
// and rays left over the drift budget after passing inside r = 4 go onto a
// list that a second kernel re-integrates in FP64.
#include <vector>

#include "lanes.cuh"
#include "runtime.h"

namespace gg {

// Mode: GG_PRECISION_PLAIN, _COMPENSATED, _PLAIN_AS_WRITTEN or _RENORMALISED.
template <int Mode>
__global__ void __launch_bounds__(256) march_image_kernel(MarchParams p) {
    constexpr bool Comp = Mode == GG_PRECISION_COMPENSATED || Mode == GG_PRECISION_RENORMALISED;
    const uint32_t gx = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gy = blockIdx.y * blockDim.y + threadIdx.y;
    const uint32_t px = p.u.tileOrigin.x + gx, py = p.u.tileOrigin.y + gy;
    const bool inside = gx < p.target_width && gy < p.target_height;
    const bool active = inside && px < p.u.resolution.x && py < p.u.resolution.y;
    PixelResult r{};
    r.outcome = RayEscaped;
    if (active) {
        if constexpr (Mode == GG_PRECISION_COMPENSATED) r = shade_pixel_compensated(p, px, py);
        else if constexpr (Mode == GG_PRECISION_RENORMALISED) r = shade_pixel_renormalised(p, px, py);
        else if constexpr (Mode == GG_PRECISION_PLAIN) r = shade_pixel_plain(p, px, py);
        else r = shade_pixel<float, false>(p, px, py);
        const uint32_t local = gy * p.target_width + gx;
        write_pixel(p, local, r);
        if (Comp && p.flagged && needs_fp64(p.u, r, p.fp64_all != 0u)) {
            uint32_t slot = atomicAdd(p.flagged_count, 1u);
            if (slot < p.flagged_capacity) p.flagged[slot] = local;
        }
    }
    // Per-frame counters: a warp sum, one atomic per warp (march.metal:274-287).
    uint32_t over = (active && r.drift > p.u.driftBudget) ? 1u : 0u;
    uint32_t exhausted = (active && r.outcome == RayExhausted) ? 1u : 0u;
    uint32_t captured = (active && r.outcome == RayCaptured) ? 1u : 0u;
    const unsigned mask = __activemask();
    uint32_t sr = __reduce_add_sync(mask, active ? 1u : 0u);
    uint32_t so = __reduce_add_sync(mask, over);
    uint32_t se = __reduce_add_sync(mask, exhausted);
    uint32_t sc = __reduce_add_sync(mask, captured);
    uint32_t ssteps = __reduce_add_sync(mask, active ? r.steps : 0u);
    uint32_t ssamples = __reduce_add_sync(mask, active ? r.samples : 0u);
    if ((threadIdx.x + threadIdx.y * blockDim.x) % 32u == 0u && p.counters) {
        if (sr) atomicAdd(&p.counters->rays, sr);
        if (so) atomicAdd(&p.counters->overDriftBudget, so);
        if (se) atomicAdd(&p.counters->exhausted, se);
        if (sc) atomicAdd(&p.counters->captured, sc);
        if (ssteps) atomicAdd(&p.stats[0], (unsigned long long)ssteps);
        if (ssamples) atomicAdd(&p.stats[1], (unsigned long long)ssamples);
    }
}

// FP64 re-integration of the flagged pixels; the grid strides over a list
// whose length is only known on the device.
__global__ void __launch_bounds__(128) reintegrate_kernel(MarchParams p) {
    const uint32_t n = min(*p.flagged_count, p.flagged_capacity);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t local = p.flagged[i];
        const uint32_t gx = local % p.target_width, gy = local / p.target_width;
        PixelResult r = shade_pixel_lane<double>(p, p.u.tileOrigin.x + gx, p.u.tileOrigin.y + gy);
        write_pixel(p, local, r);
        atomicAdd(&p.stats[2], 1ull);
    }
}

// probeRays (march.metal:290-341).
template <typename R, bool Comp>
__device__ RayProbeResult probe_one(const MarchParams& p, const RayProbe& q, float* min_r_out) {
    const MarchUniforms& u = p.u;
    V3<R> origin = v3<R>(R(q.origin.x), R(q.origin.y), R(q.origin.z));
    V3<R> direction = v3<R>(R(q.direction.x), R(q.direction.y), R(q.direction.z));
    RayProbeResult out;
    if (u.spin > 0.0f) {
        const R a = R(u.spin);
        KerrState<R> kray;
        MarchResult m = march_ray_kerr<R, Comp>(kerr_launch(a, origin, direction), p, false, kray);
        V3<R> pos = kerr_position(a, kray), dir = kerr_direction(a, kray);
        out.position = {(float)pos.x, (float)pos.y, (float)pos.z};
        out.direction = {(float)dir.x, (float)dir.y, (float)dir.z};
        out.drift = m.drift;
        out.outcome = m.outcome;
        out.steps = m.steps;
        out.energy = (float)kray.energy;
        out.angularMomentum = (float)kray.angularMomentum;
        *min_r_out = m.min_r;
        return out;
    }
    PreparedRay<R> prepared = prepare_ray(origin, direction, u, p.tables);
    if (prepared.skyOnly) {
        V3<R> pos = ray_position(prepared.ray);
        out.position = {(float)pos.x, (float)pos.y, (float)pos.z};
        out.direction = {(float)prepared.sky.x, (float)prepared.sky.y, (float)prepared.sky.z};
        out.drift = 0.0f;
        out.outcome = RayEscaped;
        out.steps = 0;
        out.energy = (float)prepared.ray.energy;
        out.angularMomentum = (float)prepared.ray.angularMomentum;
        *min_r_out = (float)prepared.ray.s.r;
        return out;
    }
    PlaneRay<R> ray;
    MarchResult m = march_ray<R, Comp>(prepared.ray, p, false, ray);
    V3<R> pos = ray_position(ray);
    V3<R> dir = (m.outcome == RayEscaped && !ray_falls_in(ray, m.outcome)) ? sky_direction(ray, m, u, p.tables)
                                                                           : ray_direction(ray);
    out.position = {(float)pos.x, (float)pos.y, (float)pos.z};
    out.direction = {(float)dir.x, (float)dir.y, (float)dir.z};
    out.drift = m.drift;
    out.outcome = m.outcome;
    out.steps = m.steps;
    out.energy = (float)ray_energy(ray.s);
    out.angularMomentum = (float)ray_angular_momentum(ray.s);
    *min_r_out = m.min_r;
    return out;
}

// One probe through the lane code (the image kernels' arithmetic): plain,
// compensated or renormalised FP32, or FP64.
template <typename R, bool Comp, bool Project = false>
__device__ RayProbeResult probe_lane(const MarchParams& p, const RayProbe& q, float* min_r) {
    const MarchUniforms& u = p.u;
    float3 origin = make_float3(q.origin.x, q.origin.y, q.origin.z);
    float3 dir = make_float3(q.direction.x, q.direction.y, q.direction.z);
    if (u.spin > 0.0f) {
        KLane<R> l;
        k_init(l, origin, dir, u);
        for (uint32_t k = 0; k <= STEP_CAP_STILL; ++k)
            if (k_step<R, Comp, Project>(l, u, 0, 0, false)) break;
        *min_r = l.min_r;
        return k_probe_result(l);
    }
    SLane<R> l;
    float3 sky;
    if (s_init(l, origin, dir, u, p.tables, &sky))
        return probe_one<float, false>(p, q, min_r);  // sky-only: no integration either way
    for (uint32_t k = 0; k <= STEP_CAP_STILL; ++k)
        if (s_step<R, Comp, Project>(l, u, 0, 0, false)) break;
    *min_r = l.min_r;
    return s_probe_result(l, u, p.tables);
}

template <int Mode>
__global__ void __launch_bounds__(64) probe_kernel(MarchParams p, const RayProbe* __restrict__ probes,
                                                   RayProbeResult* __restrict__ results, uint32_t count) {
    constexpr bool Comp = Mode == GG_PRECISION_COMPENSATED || Mode == GG_PRECISION_RENORMALISED;
    constexpr bool Project = Mode == GG_PRECISION_RENORMALISED;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    RayProbe q = probes[i];
    float min_r = 0.0f;
    RayProbeResult r;
    if constexpr (Mode == GG_PRECISION_PLAIN_AS_WRITTEN) {
        r = probe_one<float, false>(p, q, &min_r);
    } else {
        r = probe_lane<float, Comp, Project>(p, q, &min_r);
        PixelResult pr{};
        pr.drift = r.drift;
        pr.min_r = min_r;
        pr.outcome = r.outcome;
        if (Comp && needs_fp64(p.u, pr, p.fp64_all != 0u)) r = probe_lane<double, false>(p, q, &min_r);
    }
    results[i] = r;
}

// One FP64 ray per thread along the family origin -> base + t axis, t at
// the centres of `count` equal cells of [lo, hi]; its outcome (RayOutcome).
struct BoundaryArgs {
    double origin[3], base[3], axis[3];
    double lo, hi;
    uint32_t count;
    uint32_t* outcome;
};

__global__ void __launch_bounds__(128) boundary_kernel(MarchParams p, BoundaryArgs a) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.count) return;
    const double t = a.lo + (a.hi - a.lo) * ((double)k + 0.5) / (double)a.count;
    V3<double> o = v3<double>(a.origin[0], a.origin[1], a.origin[2]);
    V3<double> d = v3<double>(fma(t, a.axis[0], a.base[0]), fma(t, a.axis[1], a.base[1]), fma(t, a.axis[2], a.base[2]));
    uint32_t outcome;
    if (p.u.spin > 0.0f) {
        KLane<double> l;
        k_init(l, o, d, p.u);
        for (uint32_t s = 0; s <= STEP_CAP_STILL; ++s)
            if (k_step<double, false>(l, p.u, 0, 0, false)) break;
        outcome = l.outcome;
    } else {
        SLane<double> l;
        float3 sky;
        if (s_init(l, o, d, p.u, p.tables, &sky)) {
            outcome = RayEscaped;
        } else {
            for (uint32_t s = 0; s <= STEP_CAP_STILL; ++s)
                if (s_step<double, false>(l, p.u, 0, 0, false)) break;
            outcome = l.outcome;
        }
    }
    a.outcome[k] = outcome;
}

MarchParams make_params(gg_context* ctx, const gg_volume* vol, const MarchUniforms& u, const gg_sweep* sweep) {
    MarchParams p{};
    p.u = u;
    p.tables.sphere = ctx->sphere_table;
    p.tables.camera = sweep ? sweep->camera : nullptr;
    p.tables.sky = sweep ? sweep->sky : nullptr;
    p.emission = vol ? vol->emission_tex : 0;
    p.velocity = vol ? vol->velocity_tex : 0;
    p.blackbody = ctx->blackbody;
    p.fp64_all = ctx->fp64_policy == GG_FP64_ALL_FLAGGED ? 1u : 0u;
    p.block_w = ctx->march_block_w;
    p.block_h = ctx->march_block_h;
    return p;
}

// The compensated image march and its FP64 pass, given a parameter block
// whose flagged list and counter are already set (p.flagged, p.flagged_count
// zeroed by the caller, p.flagged_capacity entries).
int launch_compensated_image(const MarchParams& p, cudaStream_t stream, int sm_count) {
    dim3 block(p.block_w, p.block_h);
    dim3 grid((p.target_width + block.x - 1) / block.x, (p.target_height + block.y - 1) / block.y);
    march_image_kernel<GG_PRECISION_COMPENSATED><<<grid, block, 0, stream>>>(p);
    GG_CHECK(launch_status("compensated march"));
    reintegrate_kernel<<<sm_count, 128, 0, stream>>>(p);
    return launch_status("FP64 re-integration");
}

int launch_plain_image(const MarchParams& p, cudaStream_t stream, bool as_written) {
    dim3 block(p.block_w, p.block_h);
    dim3 grid((p.target_width + block.x - 1) / block.x, (p.target_height + block.y - 1) / block.y);
    if (as_written) march_image_kernel<GG_PRECISION_PLAIN_AS_WRITTEN><<<grid, block, 0, stream>>>(p);
    else march_image_kernel<GG_PRECISION_PLAIN><<<grid, block, 0, stream>>>(p);
    return launch_status("plain march");
}

static bool known_precision(int precision) {
    return precision == GG_PRECISION_PLAIN || precision == GG_PRECISION_COMPENSATED ||
           precision == GG_PRECISION_PLAIN_AS_WRITTEN || precision == GG_PRECISION_RENORMALISED;
}

// The tables the uniforms enable must exist: sphereRadius > 0 means the
// caller applied gg_tables_update for u->cameraRadius.
int check_uniforms(gg_context* ctx, const MarchUniforms* u, const char* what) {
    if (!u) return fail(GG_ERR_INVALID_ARGUMENT, "%s needs uniforms.", what);
    if (u->geodesic.stepCap > STEP_CAP_STILL)
        return fail(GG_ERR_INVALID_ARGUMENT, "%s: step cap %u exceeds STEP_CAP_STILL (%u).", what, u->geodesic.stepCap,
                    STEP_CAP_STILL);
    if (u->spin < 0.0f || u->spin >= 1.0f)
        return fail(GG_ERR_INVALID_ARGUMENT, "%s: spin %g is outside [0, 1).", what, (double)u->spin);
    if (u->sphereRadius > 0.0f && u->spin == 0.0f) {
        if (!ctx->sweep.camera || std::fabs((double)u->cameraRadius - ctx->sweep.camera_radius) > 1e-3)
            return fail(GG_ERR_INVALID_ARGUMENT,
                        "%s: the uniforms enable the sphere jump for camera radius %g but the tables were built for %g; "
                        "call gg_tables_update first.",
                        what, (double)u->cameraRadius, ctx->sweep.camera_radius);
    }
    return GG_OK;
}

}  // namespace gg

using namespace gg;

extern "C" {

GG_API int gg_targets_create(gg_context* ctx, uint32_t width, uint32_t height, gg_targets** out) {
    if (!ctx || !out) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_targets_create needs a context and an output.");
    *out = nullptr;
    if (width == 0 || height == 0 || width > 16384 || height > 16384)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Target size %ux%u is outside 1..16384.", width, height);
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t px = (uint64_t)width * height;
    gg_targets* t = new gg_targets();
    t->ctx = ctx;
    t->width = width;
    t->height = height;
    int s = gg::device_alloc(ctx, px * 8u, (void**)&t->color, "march target");
    if (s == GG_OK) s = gg::device_alloc(ctx, px * 8u, (void**)&t->debug, "debug target");
    if (s == GG_OK) s = gg::device_alloc(ctx, px * 4u, (void**)&t->depth, "depth target");
    if (s == GG_OK) s = gg::device_alloc(ctx, px * 4u, (void**)&t->motion, "motion target");
    t->bytes = px * 24u;
    if (s != GG_OK) {
        gg_targets_destroy(t);
        return s;
    }
    *out = t;
    return GG_OK;
}

GG_API void gg_targets_destroy(gg_targets* t) {
    if (!t) return;
    gg_context* ctx = t->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    const uint64_t px = (uint64_t)t->width * t->height;
    gg::device_free(ctx, t->color, px * 8u);
    gg::device_free(ctx, t->debug, px * 8u);
    gg::device_free(ctx, t->depth, px * 4u);
    gg::device_free(ctx, t->motion, px * 4u);
    if (t->srgb) gg::device_free(ctx, t->srgb, px * 4u);
    delete t;
}

GG_API int gg_targets_read(gg_targets* t, uint16_t* color, uint16_t* debug, float* depth, uint16_t* motion) {
    if (!t) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_targets_read needs targets.");
    gg_context* ctx = t->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t px = (uint64_t)t->width * t->height;
    if (color) GG_CUDA(cudaMemcpyAsync(color, t->color, px * 8u, cudaMemcpyDeviceToHost, ctx->stream), "target readback");
    if (debug) GG_CUDA(cudaMemcpyAsync(debug, t->debug, px * 8u, cudaMemcpyDeviceToHost, ctx->stream), "target readback");
    if (depth) GG_CUDA(cudaMemcpyAsync(depth, t->depth, px * 4u, cudaMemcpyDeviceToHost, ctx->stream), "target readback");
    if (motion) GG_CUDA(cudaMemcpyAsync(motion, t->motion, px * 4u, cudaMemcpyDeviceToHost, ctx->stream), "target readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "target readback");
    return GG_OK;
}

GG_API int gg_context_set_march_block(gg_context* ctx, uint32_t width, uint32_t height) {
    const uint32_t threads = width * height;
    if (!ctx || width == 0 || height == 0 || width > 256 || height > 256 || threads < 32 || threads > 256 ||
        threads % 32u != 0)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "March block %ux%u is not 32..256 threads in whole warps.", width,
                        height);
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ctx->march_block_w = width;
    ctx->march_block_h = height;
    return GG_OK;
}

GG_API int gg_context_set_fp64_policy(gg_context* ctx, int policy) {
    if (!ctx || (policy != GG_FP64_ESCAPING && policy != GG_FP64_ALL_FLAGGED))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_context_set_fp64_policy needs a context and a known policy.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    ctx->fp64_policy = policy;
    return GG_OK;
}

GG_API int gg_targets_write(gg_targets* t, const uint16_t* color, const uint16_t* debug) {
    if (!t || (!color && !debug)) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_targets_write needs targets and pixels.");
    gg_context* ctx = t->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t px = (uint64_t)t->width * t->height;
    if (color) GG_CUDA(cudaMemcpyAsync(t->color, color, px * 8u, cudaMemcpyHostToDevice, ctx->stream), "target upload");
    if (debug) GG_CUDA(cudaMemcpyAsync(t->debug, debug, px * 8u, cudaMemcpyHostToDevice, ctx->stream), "target upload");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "target upload");
    return GG_OK;
}

GG_API int gg_march(gg_context* ctx, const gg_volume* vol, const MarchUniforms* u, gg_targets* targets, int precision,
                    MarchCounters* counters) {
    gg::Range range("gg_march");
    if (!ctx || !targets) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_march needs a context and targets.");
    if (!gg::known_precision(precision))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Unknown precision policy %d.", precision);
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    GG_CHECK(gg::check_uniforms(ctx, u, "gg_march"));
    if (vol && vol->ctx != ctx) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_march: volume from another context.");
    MarchParams p = gg::make_params(ctx, vol, *u, &ctx->sweep);
    p.color = targets->color;
    p.debug = targets->debug;
    p.depth = targets->depth;
    p.motion = targets->motion;
    p.target_width = targets->width;
    p.target_height = targets->height;
    p.counters = ctx->counters;
    p.stats = ctx->stats;
    GG_CUDA(cudaMemsetAsync(ctx->counters, 0, sizeof(MarchCounters), ctx->stream), "counter reset");
    GG_CUDA(cudaMemsetAsync(ctx->stats, 0, 4 * sizeof(unsigned long long), ctx->stream), "stats reset");
    const bool comp = precision == GG_PRECISION_COMPENSATED || precision == GG_PRECISION_RENORMALISED;
    if (comp) {
        // Scratch: the flagged-pixel list (one entry per target pixel at most)
        // and its counter, in one buffer.
        const uint64_t entries = (uint64_t)targets->width * targets->height;
        GG_CHECK(gg::ensure_capacity(ctx, (void**)&ctx->flagged, &ctx->flagged_capacity, (entries + 1u) * 4u,
                                     "re-integration list"));
        p.flagged_count = ctx->flagged;
        p.flagged = ctx->flagged + 1;
        p.flagged_capacity = (uint32_t)entries;
        GG_CUDA(cudaMemsetAsync(ctx->flagged, 0, 4u, ctx->stream), "re-integration list reset");
    }
    dim3 block(p.block_w, p.block_h);
    dim3 grid((targets->width + block.x - 1) / block.x, (targets->height + block.y - 1) / block.y);
    if (comp) {
        if (precision == GG_PRECISION_RENORMALISED)
            march_image_kernel<GG_PRECISION_RENORMALISED><<<grid, block, 0, ctx->stream>>>(p);
        else
            march_image_kernel<GG_PRECISION_COMPENSATED><<<grid, block, 0, ctx->stream>>>(p);
        GG_CHECK(gg::launch_status("march"));
        reintegrate_kernel<<<ctx->sm_count, 128, 0, ctx->stream>>>(p);
    } else if (precision == GG_PRECISION_PLAIN) {
        march_image_kernel<GG_PRECISION_PLAIN><<<grid, block, 0, ctx->stream>>>(p);
    } else {
        march_image_kernel<GG_PRECISION_PLAIN_AS_WRITTEN><<<grid, block, 0, ctx->stream>>>(p);
    }
    GG_CHECK(gg::launch_status("march"));
    if (counters) {
        GG_CUDA(cudaMemcpyAsync(counters, ctx->counters, sizeof(MarchCounters), cudaMemcpyDeviceToHost, ctx->stream),
                "counter readback");
        GG_CUDA(cudaStreamSynchronize(ctx->stream), "march");
    }
    return GG_OK;
}

GG_API int gg_march_stats(gg_context* ctx, uint64_t* ray_steps, uint64_t* samples, uint64_t* fp64_rays) {
    if (!ctx) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_march_stats needs a context.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    unsigned long long host[4];
    GG_CUDA(cudaMemcpyAsync(host, ctx->stats, sizeof host, cudaMemcpyDeviceToHost, ctx->stream), "stats readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "stats readback");
    if (ray_steps) *ray_steps = host[0];
    if (samples) *samples = host[1];
    if (fp64_rays) *fp64_rays = host[2];
    return GG_OK;
}

GG_API int gg_capture_boundary(gg_context* ctx, const MarchUniforms* u, const double origin[3], const double base[3],
                               const double axis[3], double lo, double hi, uint32_t rays_per_round, uint32_t rounds,
                               double* t_out) {
    if (!ctx || !origin || !base || !axis || !t_out)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_capture_boundary needs a context, three vectors and an output.");
    if (!(hi > lo) || rays_per_round < 2 || rays_per_round > (1u << 20) || rounds == 0 || rounds > 64)
        return gg::fail(GG_ERR_INVALID_ARGUMENT,
                        "gg_capture_boundary needs lo < hi, 2..1048576 rays per round and 1..64 rounds.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    GG_CHECK(gg::check_uniforms(ctx, u, "gg_capture_boundary"));
    GG_CHECK(gg::ensure_capacity(ctx, &ctx->probe_buffer, &ctx->probe_capacity, 4ull * rays_per_round,
                                 "boundary outcomes"));
    MarchParams p = gg::make_params(ctx, nullptr, *u, &ctx->sweep);
    BoundaryArgs a;
    for (int c = 0; c < 3; ++c) {
        a.origin[c] = origin[c];
        a.base[c] = base[c];
        a.axis[c] = axis[c];
    }
    a.count = rays_per_round;
    a.outcome = static_cast<uint32_t*>(ctx->probe_buffer);
    std::vector<uint32_t> out(rays_per_round);
    for (uint32_t round = 0; round < rounds; ++round) {
        a.lo = lo;
        a.hi = hi;
        boundary_kernel<<<(rays_per_round + 127u) / 128u, 128, 0, ctx->stream>>>(p, a);
        GG_CHECK(gg::launch_status("capture boundary"));
        GG_CUDA(cudaMemcpyAsync(out.data(), a.outcome, 4ull * rays_per_round, cudaMemcpyDeviceToHost, ctx->stream),
                "boundary readback");
        GG_CUDA(cudaStreamSynchronize(ctx->stream), "capture boundary");
        auto t_of = [&](uint32_t k) { return lo + (hi - lo) * ((double)k + 0.5) / (double)rays_per_round; };
        // The edge follows the last ray whose fate matches the first ray's:
        // a ray deep on the captured side that a step carries across the
        // horizon can come out as a spurious escape (the reference's
        // integrator does the same), so earlier changes are not the edge.
        const bool first_captured = out[0] == RayCaptured;
        uint32_t last = rays_per_round;
        for (uint32_t k = rays_per_round; k-- > 0;)
            if ((out[k] == RayCaptured) == first_captured) {
                last = k;
                break;
            }
        const uint32_t k = last + 1;
        if (k >= rays_per_round) {
            if (round == 0)
                return gg::fail(GG_ERR_INVALID_ARGUMENT, "Every ray in [%g, %g] is %s: no capture boundary inside.", lo,
                                hi, first_captured ? "captured" : "escaping");
            break;  // the boundary lies between two cells of the last round
        }
        // A ray at the edge that orbits until the step cap sits on the
        // boundary and ends the search (Validate.swift:125-150).
        if (out[k] == RayExhausted) {
            *t_out = t_of(k);
            return GG_OK;
        }
        const double nlo = t_of(k - 1), nhi = t_of(k);
        lo = nlo;
        hi = nhi;
    }
    *t_out = 0.5 * (lo + hi);
    return GG_OK;
}

GG_API int gg_probe(gg_context* ctx, const MarchUniforms* u, const RayProbe* probes, RayProbeResult* results,
                    uint32_t count, int precision) {
    gg::Range range("gg_probe");
    if (!ctx || (!probes && count) || (!results && count))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_probe needs a context and probe arrays.");
    if (!gg::known_precision(precision))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Unknown precision policy %d.", precision);
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    GG_CHECK(gg::check_uniforms(ctx, u, "gg_probe"));
    if (count == 0) return GG_OK;
    const uint64_t in_bytes = (uint64_t)count * sizeof(RayProbe);
    const uint64_t out_bytes = (uint64_t)count * sizeof(RayProbeResult);
    const uint64_t out_offset = (in_bytes + 255u) & ~255ull;
    GG_CHECK(gg::ensure_capacity(ctx, &ctx->probe_buffer, &ctx->probe_capacity, out_offset + out_bytes, "probe buffers"));
    RayProbe* d_in = (RayProbe*)ctx->probe_buffer;
    RayProbeResult* d_out = (RayProbeResult*)((char*)ctx->probe_buffer + out_offset);
    GG_CUDA(cudaMemcpyAsync(d_in, probes, in_bytes, cudaMemcpyHostToDevice, ctx->stream), "probe upload");
    MarchParams p = gg::make_params(ctx, nullptr, *u, &ctx->sweep);
    const unsigned blocks = (count + 63u) / 64u;
    if (precision == GG_PRECISION_COMPENSATED)
        probe_kernel<GG_PRECISION_COMPENSATED><<<blocks, 64, 0, ctx->stream>>>(p, d_in, d_out, count);
    else if (precision == GG_PRECISION_RENORMALISED)
        probe_kernel<GG_PRECISION_RENORMALISED><<<blocks, 64, 0, ctx->stream>>>(p, d_in, d_out, count);
    else if (precision == GG_PRECISION_PLAIN)
        probe_kernel<GG_PRECISION_PLAIN><<<blocks, 64, 0, ctx->stream>>>(p, d_in, d_out, count);
    else
        probe_kernel<GG_PRECISION_PLAIN_AS_WRITTEN><<<blocks, 64, 0, ctx->stream>>>(p, d_in, d_out, count);
    GG_CHECK(gg::launch_status("probe rays"));
    GG_CUDA(cudaMemcpyAsync(results, d_out, out_bytes, cudaMemcpyDeviceToHost, ctx->stream), "probe readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "probe rays");
    return GG_OK;
}

}  // extern "C"
