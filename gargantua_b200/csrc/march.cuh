// Per-ray march shared by the image, probe, bake and served kernels
// (march.metal:29-288). Templated on the real type R (float for the march,
// double for the FP64 re-integration) and on Comp, which accumulates the RK4
// state update with TwoSum compensation (Knuth 1969, TAOCP vol. 2, 4.2.2):
// the rounding error of every state += increment is carried in a second
// word and added back on the next step, which removes the random walk of
// per-step rounding that dominates FP32 drift over thousands of steps.
#pragma once

#include "geodesic.cuh"
#include "kerr.cuh"

namespace gg {

struct MarchParams {
    MarchUniforms u;
    SweepTables tables;
    cudaTextureObject_t emission;  // 0: no gas to gather
    cudaTextureObject_t velocity;
    const float4* blackbody;
    ushort4* color;
    ushort4* debug;
    float* depth;
    ushort2* motion;
    uint32_t target_width;
    uint32_t target_height;
    MarchCounters* counters;
    unsigned long long* stats;  // ray steps, gather samples, FP64 re-integrated rays
    uint32_t* flagged;        // FP64 re-integration list (target-local pixel indices)
    uint32_t* flagged_count;  // its length, a device counter
    uint32_t flagged_capacity;
    uint32_t fp64_all;        // GG_FP64_ALL_FLAGGED: captured rays are re-integrated too
    uint32_t block_w, block_h;  // image kernel block shape
};

struct MarchResult {
    float3 color;
    float transmittance;
    float drift;
    uint32_t steps;
    uint32_t outcome;
    bool leftSphere;
    float depth;
    float min_r;
    uint32_t samples;  // in-slab gather evaluations
};

// x += y with the error word e carried: Fast2Sum(x, y + e). The error word
// is exact when |x| >= |y + e|, which holds for every state word except in
// the step where a momentum or angle crosses zero; there the sum is still
// correctly rounded and only that step's error word is approximate.
__device__ __forceinline__ void comp_add(float& x, float& e, float y) {
    float b = __fadd_rn(y, e);
    float t = __fadd_rn(x, b);
    e = __fsub_rn(b, __fsub_rn(t, x));
    x = t;
}

template <typename R, bool Comp>
__device__ __forceinline__ void advance(RayState<R>& s, RayState<R>& c, R h) {
    RayState<R> inc = ray_increment(s, h);
    if constexpr (Comp) {
        comp_add(s.v, c.v, inc.v);
        comp_add(s.r, c.r, inc.r);
        comp_add(s.phi, c.phi, inc.phi);
        comp_add(s.vDot, c.vDot, inc.vDot);
        comp_add(s.rDot, c.rDot, inc.rDot);
        comp_add(s.phiDot, c.phiDot, inc.phiDot);
    } else {
        s = ray_add(s, inc);
    }
}

// Reciprocal: FP32 within one ulp (PTX rcp.approx); FP64 from the
// approximate reciprocal refined by two Newton steps y += y (1 - x y).
__device__ __forceinline__ float rcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ double rcp(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

// Square root for lengths that feed only path lengths and sample positions:
// FP32 from sqrt.approx (relative error below 2^-22), FP64 exact.
__device__ __forceinline__ float asqrt(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ double asqrt(double x) { return sqrt(x); }

struct GatherView {
    cudaTextureObject_t emission;
    cudaTextureObject_t velocity;
    float half_extent;
    float opacity;
    uint32_t redshift;
};

__device__ __forceinline__ GatherView gather_view(const MarchUniforms& u, cudaTextureObject_t em, cudaTextureObject_t vel) {
    return GatherView{em, vel, u.volumeHalfExtent, u.opacityScale, u.redshift};
}

// Gather one in-slab sample into the running colour (march.metal:81-102).
// The photon's direction is needed only for the redshift of a sample that
// holds gas, so it is passed as a function evaluated there.
//
// Fast (the lanes: served, plain and compensated marches) evaluates the
// redshift and opacity with hardware approximations where the reference's
// kernel calls precise functions: tanh from one exponential, tanh x = 1 -
// 2 / (e^2x + 1) (absolute error near 1e-7), the exponentials, reciprocals
// and square roots approximate (relative errors of a few 1e-7). Without
// Fast (the per-request kernel as written) the arithmetic is the
// reference's. The texture coordinates are the reference's in both.
template <bool Fast, typename Direction>
__device__ __forceinline__ void gather_sample_with(const GatherView& gv, float3 position, float f, Direction direction,
                                                   float path, float travelled, float3& color, float& transmittance,
                                                   float& weighted_depth, float& depth_weight, uint32_t& samples) {
    samples += 1u;
    // sampleVolume (march.metal:15-27); the velocity texel is fetched only
    // where the redshift reads it (gas present, redshift on).
    const float3 c = volume_coordinates(position, gv.half_extent);
    const float4 e = tex3D<float4>(gv.emission, c.x, c.y, c.z);
    Sample s;
    s.emission = make_float3(e.x, e.y, e.z);
    s.density = e.w;
    if (s.density > 0.0f) {
        float g3 = 1.0f;
        if (gv.redshift != 0u) {
            const float4 v = tex3D<float4>(gv.velocity, c.x, c.y, c.z);
            s.velocity = make_float3(v.x, v.y, v.z);
            float g, gravity, bulk;
            if constexpr (Fast) {
                // redshiftFactor (Geodesic.h:225-236) as redshift_factor below.
                const float3 gas = s.velocity;
                const float magnitude = asqrt(dot3(gas, gas));
                const float speed = fminf(magnitude, 8.0f);
                const float beta =
                    GAS_SPEED_CEILING * (1.0f - 2.0f * rcp(__expf(speed * (2.0f / GAS_SPEED_CEILING)) + 1.0f));
                const float scale = magnitude > 0.0f ? beta * rcp(magnitude) : 0.0f;
                gravity = asqrt(fmaxf(f, 0.0f));
                g = gravity * asqrt(1.0f - beta * beta) * rcp(fmaf(dot3(direction(), gas), scale, 1.0f));
                bulk = fminf(s.density * (1.0f / BEAMING_DENSITY_FLOOR), 1.0f);
            } else {
                g = redshift_factor(f, direction(), s.velocity);
                gravity = sqrtf(fmaxf(f, 0.0f));
                bulk = fminf(s.density / BEAMING_DENSITY_FLOOR, 1.0f);
            }
            float gr3 = gravity * gravity * gravity;
            g3 = gr3 + (g * g * g - gr3) * bulk;
        }
        float extinction = -gv.opacity * s.density * path;
        float alpha = 1.0f - (Fast ? __expf(extinction) : expf(extinction));
        float k = transmittance * g3 * path;
        float3 contribution = make_float3(s.emission.x * k, s.emission.y * k, s.emission.z * k);
        color = color + contribution;
        float weight = dot3(contribution, make_float3(0.2126f, 0.7152f, 0.0722f));
        weighted_depth += weight * travelled;
        depth_weight += weight;
        transmittance *= 1.0f - alpha;
    }
}

__device__ __forceinline__ void gather_sample(const GatherView& gv, float3 position, float f, float3 direction,
                                              float path, float travelled, float3& color, float& transmittance,
                                              float& weighted_depth, float& depth_weight, uint32_t& samples) {
    gather_sample_with<false>(gv, position, f, [&] { return direction; }, path, travelled, color, transmittance,
                              weighted_depth, depth_weight, samples);
}

__device__ __forceinline__ bool in_slab(float3 q, float half_extent) {
    return fabsf(q.z) < DISK_SLAB_HALF_HEIGHT && fabsf(q.x) < half_extent && fabsf(q.y) < half_extent;
}

// The Schwarzschild integration loop (march.metal:51-117).
template <typename R, bool Comp>
__device__ MarchResult march_ray(const PlaneRay<R>& launched, const MarchParams& p, bool gather, PlaneRay<R>& out) {
    const MarchUniforms& u = p.u;
    const GeodesicSettings& g = u.geodesic;
    PlaneRay<R> ray = launched;
    RayState<R> comp{};
    float3 color = make_float3(0.0f, 0.0f, 0.0f);
    float transmittance = 1.0f;
    V3<R> previous = ray_position(ray);
    uint32_t outcome = RayExhausted;
    bool left_sphere = false;
    uint32_t steps = 0;
    float travelled = 0.0f, weighted_depth = 0.0f, depth_weight = 0.0f;
    uint32_t samples = 0;
    float min_r = (float)ray.s.r;
    const R sphere = R(u.sphereRadius);
    for (uint32_t k = 0; k < STEP_CAP_STILL; ++k) {
        if (k >= g.stepCap) break;
        R h = ray_step_length(previous.z, ray.s.r, g);
        RayState<R> before = ray.s;
        RayState<R> before_c = comp;
        advance<R, Comp>(ray.s, comp, h);
        steps = k + 1u;
        if (u.sphereRadius > 0.0f && ray.s.r >= sphere && ray.s.rDot > R(0) && before.r < sphere) {
            // Land on the sphere, where the sweep table is exact (march.metal:71-76).
            R frac = (sphere - before.r) / (ray.s.r - before.r);
            ray.s = before;
            comp = before_c;
            advance<R, Comp>(ray.s, comp, h * frac);
        }
        V3<R> position = ray_position(ray);
        float path = (float)length(position - previous);
        travelled += path;
        min_r = fminf(min_r, (float)ray.s.r);
        if (ray.s.r <= R(g.captureRadius)) {
            outcome = RayCaptured;
            break;
        }
        float3 pf = to_float3(position);
        if (gather && in_slab(pf, u.volumeHalfExtent) && transmittance > 0.004f) {
            float f = (float)schwarzschild_f(ray.s.r);
            float3 dir = to_float3(ray_direction(ray));
            gather_sample(gather_view(u, p.emission, p.velocity), pf, f, dir, path, travelled, color, transmittance, weighted_depth,
                          depth_weight, samples);
        }
        previous = position;
        if (u.sphereRadius > 0.0f && ray.s.r >= sphere && ray.s.rDot > R(0)) {
            outcome = RayEscaped;
            left_sphere = true;
            break;
        }
        if (ray.s.r >= R(g.escapeRadius)) {
            outcome = RayEscaped;
            break;
        }
    }
    out = ray;
    MarchResult m;
    m.color = color;
    m.transmittance = transmittance;
    if constexpr (Comp) {
        // Drift of the compensated state, evaluated in double from value +
        // error word against the launch values evaluated the same way.
        double r = (double)ray.s.r + (double)comp.r;
        double e = (1.0 - 2.0 / r) * ((double)ray.s.vDot + (double)comp.vDot) - ((double)ray.s.rDot + (double)comp.rDot);
        double l = r * r * ((double)ray.s.phiDot + (double)comp.phiDot);
        double r0 = (double)launched.s.r;
        double e0 = (1.0 - 2.0 / r0) * (double)launched.s.vDot - (double)launched.s.rDot;
        double l0 = r0 * r0 * (double)launched.s.phiDot;
        double ed = fabs(e - e0) / fabs(e0);
        double ld = fabs(l - l0) / fmax(fabs(l0), 1e-3);
        m.drift = (float)fmax(ed, ld);
    } else {
        m.drift = (float)ray_drift(ray);
    }
    m.steps = steps;
    m.outcome = outcome;
    m.leftSphere = left_sphere;
    m.depth = depth_weight > 0.0f ? weighted_depth / depth_weight : travelled;
    m.min_r = min_r;
    m.samples = samples;
    return m;
}

template <typename R, bool Comp>
__device__ __forceinline__ void kerr_advance(R a, KerrState<R>& s, KerrVec<R>& c, R h) {
    KerrVec<R> inc = kerr_increment(a, s, h);
    if constexpr (Comp) {
        comp_add(s.r, c.r, inc.r);
        comp_add(s.theta, c.theta, inc.theta);
        comp_add(s.phi, c.phi, inc.phi);
        comp_add(s.pr, c.pr, inc.pr);
        comp_add(s.ptheta, c.ptheta, inc.ptheta);
    } else {
        s.r += inc.r;
        s.theta += inc.theta;
        s.phi += inc.phi;
        s.pr += inc.pr;
        s.ptheta += inc.ptheta;
    }
}

// The Kerr twin of march_ray (march.metal:123-184): no sweep-table jump,
// capture at the outer horizon plus KERR_CAPTURE_MARGIN, drift = max over
// steps of the Carter-constant and null-residual gauges.
template <typename R, bool Comp>
__device__ MarchResult march_ray_kerr(const KerrState<R>& launched, const MarchParams& p, bool gather, KerrState<R>& out) {
    const MarchUniforms& u = p.u;
    const GeodesicSettings& g = u.geodesic;
    const R a = R(u.spin);
    KerrState<R> ray = launched;
    KerrVec<R> comp{};
    R carter0 = kerr_carter(a, launched);
    R scale = gmax(gabs(carter0), launched.energy * launched.energy);
    R capture = kerr_outer_horizon(a) + R(KERR_CAPTURE_MARGIN);
    float3 color = make_float3(0.0f, 0.0f, 0.0f);
    float transmittance = 1.0f;
    V3<R> previous = kerr_position(a, ray);
    uint32_t outcome = RayExhausted;
    uint32_t steps = 0;
    float travelled = 0.0f, weighted_depth = 0.0f, depth_weight = 0.0f;
    uint32_t samples = 0;
    R drift = R(0);
    float min_r = (float)ray.r;
    for (uint32_t k = 0; k < STEP_CAP_STILL; ++k) {
        if (k >= g.stepCap) break;
        kerr_advance<R, Comp>(a, ray, comp, kerr_step_length(a, ray, g));
        steps = k + 1u;
        V3<R> position = kerr_position(a, ray);
        float path = (float)length(position - previous);
        travelled += path;
        R cd = gabs(kerr_carter(a, ray) - carter0) / scale;
        R nd = gabs(kerr_null_residual(a, ray)) / (scale * gmax(ray.r * ray.r, R(1)));
        drift = gmax(drift, gmax(cd, nd));
        min_r = fminf(min_r, (float)ray.r);
        if (ray.r <= capture) {
            outcome = RayCaptured;
            break;
        }
        float3 pf = to_float3(position);
        if (gather && in_slab(pf, u.volumeHalfExtent) && transmittance > 0.004f) {
            R st, ct;
            gsincos(ray.theta, &st, &ct);
            float sigma = (float)(ray.r * ray.r + a * a * ct * ct);
            float fk = 1.0f - 2.0f * (float)ray.r / sigma;
            float3 dir = to_float3(kerr_direction(a, ray));
            gather_sample(gather_view(u, p.emission, p.velocity), pf, fmaxf(fk, 0.0f), dir, path, travelled, color,
                          transmittance, weighted_depth, depth_weight, samples);
        }
        previous = position;
        if (ray.r >= R(g.escapeRadius)) {
            outcome = RayEscaped;
            break;
        }
    }
    out = ray;
    MarchResult m;
    m.color = color;
    m.transmittance = transmittance;
    m.drift = (float)drift;
    m.steps = steps;
    m.outcome = outcome;
    m.leftSphere = false;
    m.depth = depth_weight > 0.0f ? weighted_depth / depth_weight : travelled;
    m.min_r = min_r;
    m.samples = samples;
    return m;
}

// Falls into the hole: captured, or out of steps moving inward with impact
// parameter below 3 sqrt 3 (march.metal:44-47).
template <typename R> __device__ __forceinline__ bool ray_falls_in(const PlaneRay<R>& ray, uint32_t outcome) {
    return outcome == RayCaptured ||
           (outcome == RayExhausted && ray.s.rDot < R(0) && gabs(ray.angularMomentum) < R(B_CRITICAL) * ray.energy);
}

template <typename R>
__device__ __forceinline__ V3<R> sky_direction(const PlaneRay<R>& ray, const MarchResult& m, const MarchUniforms& u,
                                               const SweepTables& t) {
    return m.leftSphere ? sphere_exit_direction(ray, u, t) : ray_direction(ray);
}

struct PixelResult {
    float3 color;
    float drift;
    uint32_t steps;
    uint32_t outcome;
    float depth;
    float min_r;
    uint32_t samples;
};

// Camera ray through a pixel centre plus jitter (march.metal:215-218).
__device__ __forceinline__ float3 camera_direction(const MarchUniforms& u, uint32_t px, uint32_t py) {
    float sx = (float)px + 0.5f + u.jitter.x;
    float sy = (float)py + 0.5f + u.jitter.y;
    float nx = (2.0f * sx / (float)u.resolution.x - 1.0f) * u.tanHalfFov.x;
    float ny = (1.0f - 2.0f * sy / (float)u.resolution.y) * u.tanHalfFov.y;
    return normalize3(to_f3(u.cameraForward) + nx * to_f3(u.cameraRight) + ny * to_f3(u.cameraUp));
}

// One pixel of marchImage (march.metal:207-273), up to the output writes.
template <typename R, bool Comp>
__device__ PixelResult shade_pixel(const MarchParams& p, uint32_t px, uint32_t py) {
    const MarchUniforms& u = p.u;
    const bool gather = p.emission != 0;
    float3 dirf = camera_direction(u, px, py);
    V3<R> origin = to_v3<R>(to_f3(u.cameraPosition));
    V3<R> direction = to_v3<R>(dirf);
    PixelResult r;
    if (u.spin > 0.0f) {
        KerrState<R> kray;
        MarchResult m = march_ray_kerr<R, Comp>(kerr_launch(R(u.spin), origin, direction), p, gather, kray);
        r.color = m.color;
        r.drift = m.drift;
        r.steps = m.steps;
        r.outcome = m.outcome;
        r.depth = m.depth;
        r.min_r = m.min_r;
        r.samples = m.samples;
        bool falls_in = m.outcome == RayCaptured || (m.outcome == RayExhausted && kray.pr < R(0));
        if (!falls_in && u.starBrightness > 0.0f) {
            float3 star = starfield(to_float3(kerr_direction(R(u.spin), kray)), u.starSeed, p.blackbody);
            r.color = r.color + star * (m.transmittance * u.starBrightness);
        }
        return r;
    }
    PreparedRay<R> prepared = prepare_ray(origin, direction, u, p.tables);
    r.drift = 0.0f;
    r.steps = 0;
    r.outcome = RayEscaped;
    r.depth = 2.0f * R_ESCAPE;
    r.min_r = (float)prepared.ray.s.r;
    r.samples = 0;
    if (prepared.skyOnly) {
        r.color = u.starBrightness > 0.0f ? starfield(to_float3(prepared.sky), u.starSeed, p.blackbody) * u.starBrightness
                                          : make_float3(0.0f, 0.0f, 0.0f);
        return r;
    }
    PlaneRay<R> ray;
    MarchResult m = march_ray<R, Comp>(prepared.ray, p, gather, ray);
    r.color = m.color;
    r.drift = m.drift;
    r.steps = m.steps;
    r.outcome = m.outcome;
    r.depth = m.depth;
    r.min_r = m.min_r;
    r.samples = m.samples;
    if (!ray_falls_in(ray, m.outcome) && u.starBrightness > 0.0f) {
        float3 star = starfield(to_float3(sky_direction(ray, m, u, p.tables)), u.starSeed, p.blackbody);
        r.color = r.color + star * (m.transmittance * u.starBrightness);
    }
    return r;
}

__device__ __forceinline__ void write_pixel(const MarchParams& p, uint32_t local, const PixelResult& r) {
    p.color[local] = pack_half4(r.color.x, r.color.y, r.color.z, 1.0f);
    if (p.debug) p.debug[local] = pack_half4(r.drift, (float)r.steps, (float)r.outcome, 1.0f);
    if (p.depth) p.depth[local] = fminf(r.depth / (2.0f * R_ESCAPE), 1.0f);
    if (p.motion) p.motion[local] = make_ushort2(0, 0);
}

// A ray the compensated FP32 march flags for FP64 re-integration: over the
// drift budget after passing inside r = 4.
// FP64 re-integration: over the drift budget after passing inside r < 4,
// and (unless every flagged ray is asked for) not captured.
__device__ __forceinline__ bool needs_fp64(const MarchUniforms& u, const PixelResult& r, bool all) {
    return r.drift > u.driftBudget && r.min_r < 4.0f && (all || r.outcome != RayCaptured);
}

}  // namespace gg
