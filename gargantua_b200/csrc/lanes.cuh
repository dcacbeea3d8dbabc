// The compensated FP32 march as a per-lane state machine: init from a camera
// ray, advance one RK4 step at a time, finish with the starfield. The served
// persistent kernel refills lanes between steps; the compensated image and
// probe kernels run one lane to completion. Both therefore execute exactly
// the same arithmetic, which the goldens check through gg_probe.
//
// Arithmetic, against the reference's march (march.metal:51-184):
//  - the same RK4 steps, step policy, capture/escape/sphere-exit logic and
//    gather, so ray-step counts are the reference's;
//  - each state += increment is TwoSum-compensated (march.cuh comp_add);
//  - one reciprocal per Schwarzschild derivative instead of four divides,
//    using vDotDot = r phiDot^2 - vDot^2/r^2 appearing inside rDotDot;
//    the Kerr derivative uses four reciprocals instead of eleven divides;
//  - sin and cos from a Cody-Waite reduction by pi/2 and the Taylor series
//    through r^9 / r^10 on |r| <= pi/4 (relative error below 2e-9 before
//    float rounding) instead of the library's slow-path-capable sincosf;
//  - the Eddington-Finkelstein time v, which nothing downstream reads, is
//    not integrated.
#pragma once

#include "march.cuh"

namespace gg {

// sin and cos of a float angle of moderate size (|x| < 1e5).
__device__ __forceinline__ void fast_sincos(float x, float* s_out, float* c_out) {
    const float two_over_pi = 0.636619772367581f;
    // pi/2 = hi + lo (hi holds 21 significant bits)
    const float pio2_hi = 1.57079601287841796875f;
    const float pio2_lo = 3.13916478650481e-07f;
    float k = rintf(x * two_over_pi);
    float r = fmaf(-k, pio2_hi, x);
    r = fmaf(-k, pio2_lo, r);
    float r2 = r * r;
    // sin r = r + r^3 (-1/3! + r^2 (1/5! + r^2 (-1/7! + r^2 / 9!)))
    float ps = fmaf(r2, 2.75573192239859e-06f, -1.98412698412698e-04f);
    ps = fmaf(r2, ps, 8.33333333333333e-03f);
    ps = fmaf(r2, ps, -1.66666666666667e-01f);
    float sr = fmaf(r * r2, ps, r);
    // cos r = 1 + r^2 (-1/2 + r^2 (1/4! + r^2 (-1/6! + r^2 (1/8! - r^2/10!))))
    float pc = fmaf(r2, -2.75573192239859e-07f, 2.48015873015873e-05f);
    pc = fmaf(r2, pc, -1.38888888888889e-03f);
    pc = fmaf(r2, pc, 4.16666666666667e-02f);
    pc = fmaf(r2, pc, -0.5f);
    float cr = fmaf(r2, pc, 1.0f);
    int q = (int)k;
    float s = (q & 1) ? cr : sr;
    float c = (q & 1) ? sr : cr;
    if (q & 2) s = -s;
    if ((q + 1) & 2) c = -c;
    *s_out = s;
    *c_out = c;
}

// Reciprocal to within one ulp (PTX rcp.approx: max error 1 ulp).
__device__ __forceinline__ float rcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// ------------------------------------------------------------ Schwarzschild

struct SState {
    float r, phi, vd, rd, pd;
};

// Geodesic equations (Geodesic.h:42-49) with one reciprocal.
__device__ __forceinline__ SState s_derivative(const SState& s) {
    float inv_r = rcp(s.r);
    float inv_r2 = inv_r * inv_r;
    float vdd = s.r * (s.pd * s.pd) - (s.vd * s.vd) * inv_r2;
    float f = fmaf(-2.0f, inv_r, 1.0f);
    float rdd = fmaf(f, vdd, 2.0f * (s.rd * s.vd) * inv_r2);
    float pdd = -2.0f * (s.rd * s.pd) * inv_r;
    return SState{s.rd, s.pd, vdd, rdd, pdd};
}

__device__ __forceinline__ SState s_offset(const SState& s, const SState& k, float w) {
    return SState{fmaf(k.r, w, s.r), fmaf(k.phi, w, s.phi), fmaf(k.vd, w, s.vd), fmaf(k.rd, w, s.rd), fmaf(k.pd, w, s.pd)};
}

// The RK4 increment (k1 + 2 k2 + 2 k3 + k4) h / 6 (Geodesic.h:52-59).
__device__ __forceinline__ SState s_increment(const SState& s, float h) {
    const float hh = 0.5f * h;
    SState k1 = s_derivative(s);
    SState k2 = s_derivative(s_offset(s, k1, hh));
    SState k3 = s_derivative(s_offset(s, k2, hh));
    SState k4 = s_derivative(s_offset(s, k3, h));
    const float w = h * (1.0f / 6.0f);
    SState inc;
    inc.r = (k1.r + 2.0f * k2.r + (2.0f * k3.r + k4.r)) * w;
    inc.phi = (k1.phi + 2.0f * k2.phi + (2.0f * k3.phi + k4.phi)) * w;
    inc.vd = (k1.vd + 2.0f * k2.vd + (2.0f * k3.vd + k4.vd)) * w;
    inc.rd = (k1.rd + 2.0f * k2.rd + (2.0f * k3.rd + k4.rd)) * w;
    inc.pd = (k1.pd + 2.0f * k2.pd + (2.0f * k3.pd + k4.pd)) * w;
    return inc;
}

struct SLane {
    SState s, c;  // value and TwoSum error word
    float3 e1, e2;
    float energy, angular_momentum;  // launch values (the reference's ray.energy, ray.angularMomentum)
    float e0, l0;                    // launch values of the integrated state, evaluated in double
    float3 color;
    float transmittance, travelled, weighted_depth, depth_weight;
    float3 previous;
    uint32_t steps, samples, outcome;
    float min_r;
    bool left_sphere;
};

__device__ __forceinline__ float3 s_position(const SLane& l, float* sn, float* cs) {
    fast_sincos(l.s.phi, sn, cs);
    return make_float3(l.s.r * fmaf(*cs, l.e1.x, *sn * l.e2.x), l.s.r * fmaf(*cs, l.e1.y, *sn * l.e2.y),
                       l.s.r * fmaf(*cs, l.e1.z, *sn * l.e2.z));
}

// Static-observer direction at the ray's radius (Geodesic.h:94-100).
__device__ __forceinline__ float3 s_direction(const SLane& l, float sn, float cs) {
    float3 radial = make_float3(fmaf(cs, l.e1.x, sn * l.e2.x), fmaf(cs, l.e1.y, sn * l.e2.y), fmaf(cs, l.e1.z, sn * l.e2.z));
    float3 tang = make_float3(fmaf(-sn, l.e1.x, cs * l.e2.x), fmaf(-sn, l.e1.y, cs * l.e2.y), fmaf(-sn, l.e1.z, cs * l.e2.z));
    float a = l.s.rd * rsqrtf(fmaxf(1.0f - 2.0f * rcp(l.s.r), 1e-6f));
    float b = l.s.r * l.s.pd;
    float3 local = make_float3(fmaf(a, radial.x, b * tang.x), fmaf(a, radial.y, b * tang.y), fmaf(a, radial.z, b * tang.z));
    float len2 = dot3(local, local);
    return len2 > 0.0f ? local * rsqrtf(len2) : radial;
}

// prepareRay (Geodesic.h:130-163) into a lane. Returns true when the ray is
// sky-only; then *sky holds its asymptotic direction.
__device__ __forceinline__ bool s_init(SLane& l, float3 origin, float3 direction, const MarchUniforms& u,
                                       const SweepTables& t, float3* sky) {
    PreparedRay<float> p = prepare_ray(to_v3<float>(origin), to_v3<float>(direction), u, t);
    l.e1 = to_float3(p.ray.e1);
    l.e2 = to_float3(p.ray.e2);
    l.energy = p.ray.energy;
    l.angular_momentum = p.ray.angularMomentum;
    if (p.skyOnly) {
        *sky = to_float3(p.sky);
        return true;
    }
    l.s = SState{p.ray.s.r, p.ray.s.phi, p.ray.s.vDot, p.ray.s.rDot, p.ray.s.phiDot};
    l.c = SState{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    double r0 = (double)l.s.r;
    l.e0 = (float)((1.0 - 2.0 / r0) * (double)l.s.vd - (double)l.s.rd);
    l.l0 = (float)(r0 * r0 * (double)l.s.pd);
    l.color = make_float3(0.0f, 0.0f, 0.0f);
    l.transmittance = 1.0f;
    l.travelled = l.weighted_depth = l.depth_weight = 0.0f;
    float sn, cs;
    l.previous = s_position(l, &sn, &cs);
    l.steps = l.samples = 0;
    l.outcome = RayExhausted;
    l.min_r = l.s.r;
    l.left_sphere = false;
    return false;
}

__device__ __forceinline__ void s_advance(SState& s, SState& c, float h) {
    SState inc = s_increment(s, h);
    comp_add(s.r, c.r, inc.r);
    comp_add(s.phi, c.phi, inc.phi);
    comp_add(s.vd, c.vd, inc.vd);
    comp_add(s.rd, c.rd, inc.rd);
    comp_add(s.pd, c.pd, inc.pd);
}

// One iteration of marchRay's loop (march.metal:65-106). Returns true when
// the ray ended (captured, escaped, left the sphere or hit the step cap).
__device__ __forceinline__ bool s_step(SLane& l, const MarchUniforms& u, cudaTextureObject_t em, cudaTextureObject_t vel,
                                       bool gather) {
    const GeodesicSettings& g = u.geodesic;
    if (l.steps >= g.stepCap) return true;
    float h = ray_step_length(l.previous.z, l.s.r, g);
    const float sphere = u.sphereRadius;
    SState before = l.s, before_c = l.c;
    s_advance(l.s, l.c, h);
    l.steps += 1u;
    if (sphere > 0.0f && l.s.r >= sphere && l.s.rd > 0.0f && before.r < sphere) {
        float frac = (sphere - before.r) / (l.s.r - before.r);
        l.s = before;
        l.c = before_c;
        s_advance(l.s, l.c, h * frac);
    }
    float sn, cs;
    float3 position = s_position(l, &sn, &cs);
    float3 d = position - l.previous;
    float path = sqrtf(dot3(d, d));
    l.travelled += path;
    l.min_r = fminf(l.min_r, l.s.r);
    if (l.s.r <= g.captureRadius) {
        l.outcome = RayCaptured;
        return true;
    }
    if (gather && in_slab(position, u.volumeHalfExtent) && l.transmittance > 0.004f) {
        float f = fmaf(-2.0f, rcp(l.s.r), 1.0f);
        float3 dir = s_direction(l, sn, cs);
        gather_sample(gather_view(u, em, vel), position, f, dir, path, l.travelled, l.color, l.transmittance,
                      l.weighted_depth, l.depth_weight, l.samples);
    }
    l.previous = position;
    if (sphere > 0.0f && l.s.r >= sphere && l.s.rd > 0.0f) {
        l.outcome = RayEscaped;
        l.left_sphere = true;
        return true;
    }
    if (l.s.r >= g.escapeRadius) {
        l.outcome = RayEscaped;
        return true;
    }
    return false;
}

// Drift of the compensated state against its launch values (Geodesic.h:
// 184-188), evaluated in double from value plus error word.
__device__ __forceinline__ float s_drift(const SLane& l) {
    double r = (double)l.s.r + (double)l.c.r;
    double e = (1.0 - 2.0 / r) * ((double)l.s.vd + (double)l.c.vd) - ((double)l.s.rd + (double)l.c.rd);
    double lm = r * r * ((double)l.s.pd + (double)l.c.pd);
    double ed = fabs(e - (double)l.e0) / fabs((double)l.e0);
    double ld = fabs(lm - (double)l.l0) / fmax(fabs((double)l.l0), 1e-3);
    return (float)fmax(ed, ld);
}

__device__ __forceinline__ bool s_falls_in(const SLane& l) {
    return l.outcome == RayCaptured ||
           (l.outcome == RayExhausted && l.s.rd < 0.0f && fabsf(l.angular_momentum) < B_CRITICAL * l.energy);
}

// Final sky direction: the sphere-exit asymptote or the last direction.
__device__ __forceinline__ float3 s_sky(const SLane& l, const MarchUniforms& u, const SweepTables& t) {
    float sn, cs;
    if (l.left_sphere) {
        float b = fabsf(l.angular_momentum) / l.energy;
        float sweep = sweep_lookup(t.sphere, 0.0f, u.sphereTableMaxB, b);
        fast_sincos(l.s.phi + sweep, &sn, &cs);
        return make_float3(fmaf(cs, l.e1.x, sn * l.e2.x), fmaf(cs, l.e1.y, sn * l.e2.y), fmaf(cs, l.e1.z, sn * l.e2.z));
    }
    fast_sincos(l.s.phi, &sn, &cs);
    return s_direction(l, sn, cs);
}

__device__ __forceinline__ PixelResult s_finish(const SLane& l, const MarchUniforms& u, const SweepTables& t,
                                                const float4* blackbody) {
    PixelResult r;
    r.color = l.color;
    r.drift = s_drift(l);
    r.steps = l.steps;
    r.outcome = l.outcome;
    r.depth = l.depth_weight > 0.0f ? l.weighted_depth / l.depth_weight : l.travelled;
    r.min_r = l.min_r;
    r.samples = l.samples;
    if (!s_falls_in(l) && u.starBrightness > 0.0f) {
        float3 star = starfield(s_sky(l, u, t), u.starSeed, blackbody);
        r.color = r.color + star * (l.transmittance * u.starBrightness);
    }
    return r;
}

__device__ __forceinline__ PixelResult sky_only_result(float3 sky, const MarchUniforms& u, const float4* blackbody) {
    PixelResult r;
    r.color = u.starBrightness > 0.0f ? starfield(sky, u.starSeed, blackbody) * u.starBrightness
                                      : make_float3(0.0f, 0.0f, 0.0f);
    r.drift = 0.0f;
    r.steps = 0;
    r.outcome = RayEscaped;
    r.depth = 2.0f * R_ESCAPE;
    r.min_r = 1e30f;
    r.samples = 0;
    return r;
}

// --------------------------------------------------------------------- Kerr

struct KState {
    float r, th, ph, pr, pt;
};

struct KConst {
    float a, a2, E, L, aE, aL, L2, a2E2, two_aEL;
};

__device__ __forceinline__ KConst k_const(float a, float E, float L) {
    KConst k;
    k.a = a;
    k.a2 = a * a;
    k.E = E;
    k.L = L;
    k.aE = a * E;
    k.aL = a * L;
    k.L2 = L * L;
    k.a2E2 = k.a2 * E * E;
    k.two_aEL = 2.0f * a * E * L;
    return k;
}

// Hamilton's equations with the off-shell Sigma terms (Kerr.h:63-90).
__device__ __forceinline__ KState k_derivative(const KConst& k, const KState& s) {
    float st, ct;
    fast_sincos(s.th, &st, &ct);
    float r = s.r;
    float r2 = r * r;
    float delta = r2 - 2.0f * r + k.a2;
    float sigma = fmaf(k.a2, ct * ct, r2);
    float inv_sigma = rcp(sigma);
    float inv_delta = rcp(delta);
    float sin2 = fmaxf(st * st, 1e-8f);
    float inv_sin2 = rcp(sin2);
    float p = fmaf(r2 + k.a2, k.E, -k.aL);
    float g = fmaf(k.a2E2, sin2, fmaf(k.L2, inv_sin2, -k.two_aEL));
    float pr2 = s.pr * s.pr;
    float p2d = p * p * inv_delta;
    float F = fmaf(delta, pr2, fmaf(s.pt, s.pt, g - p2d));
    float ham = 0.5f * F * inv_sigma;
    float dprime = 2.0f * r - 2.0f;
    float fr = fmaf(dprime, pr2, inv_delta * (p2d * dprime - 4.0f * r * k.E * p));
    float fth = 2.0f * ct * fmaf(k.a2E2, st, -k.L2 * inv_sin2 * rcp(fmaxf(st, 1e-4f)));
    KState o;
    o.r = delta * s.pr * inv_sigma;
    o.th = s.pt * inv_sigma;
    o.ph = (fmaf(k.a, p * inv_delta, k.L * inv_sin2) - k.aE) * inv_sigma;
    o.pr = (2.0f * r * ham - 0.5f * fr) * inv_sigma;
    o.pt = (-2.0f * k.a2 * st * ct * ham - 0.5f * fth) * inv_sigma;
    return o;
}

__device__ __forceinline__ KState k_offset(const KState& s, const KState& d, float w) {
    return KState{fmaf(d.r, w, s.r), fmaf(d.th, w, s.th), fmaf(d.ph, w, s.ph), fmaf(d.pr, w, s.pr), fmaf(d.pt, w, s.pt)};
}

__device__ __forceinline__ KState k_increment(const KConst& k, const KState& s, float h) {
    const float hh = 0.5f * h;
    KState k1 = k_derivative(k, s);
    KState k2 = k_derivative(k, k_offset(s, k1, hh));
    KState k3 = k_derivative(k, k_offset(s, k2, hh));
    KState k4 = k_derivative(k, k_offset(s, k3, h));
    const float w = h * (1.0f / 6.0f);
    KState inc;
    inc.r = (k1.r + 2.0f * k2.r + (2.0f * k3.r + k4.r)) * w;
    inc.th = (k1.th + 2.0f * k2.th + (2.0f * k3.th + k4.th)) * w;
    inc.ph = (k1.ph + 2.0f * k2.ph + (2.0f * k3.ph + k4.ph)) * w;
    inc.pr = (k1.pr + 2.0f * k2.pr + (2.0f * k3.pr + k4.pr)) * w;
    inc.pt = (k1.pt + 2.0f * k2.pt + (2.0f * k3.pt + k4.pt)) * w;
    return inc;
}

struct KLane {
    KState s, c;
    KConst k;
    float carter0, scale, capture, drift;
    float3 color;
    float transmittance, travelled, weighted_depth, depth_weight;
    float3 previous;
    uint32_t steps, samples, outcome;
    float min_r;
};

// Carter constant and null residual (Kerr.h:39-50) from the state.
__device__ __forceinline__ void k_gauges(const KLane& l, float st, float ct, float* carter, float* residual) {
    const KConst& k = l.k;
    float sin2 = fmaxf(st * st, 1e-8f);
    float inv_sin2 = rcp(sin2);
    *carter = fmaf(ct * ct, fmaf(k.L2, inv_sin2, -k.a2E2), l.s.pt * l.s.pt);
    float r = l.s.r;
    float delta = r * r - 2.0f * r + k.a2;
    float p = fmaf(r * r + k.a2, k.E, -k.aL);
    float g = fmaf(k.a2E2, sin2, fmaf(k.L2, inv_sin2, -k.two_aEL));
    *residual = fmaf(delta, l.s.pr * l.s.pr, fmaf(l.s.pt, l.s.pt, g - p * p * rcp(delta)));
}

__device__ __forceinline__ float3 k_position(const KLane& l, float st, float ct) {
    float sp, cp;
    fast_sincos(l.s.ph, &sp, &cp);
    float radial = sqrtf(fmaf(l.s.r, l.s.r, l.k.a2));
    return make_float3(radial * st * cp, radial * st * sp, l.s.r * ct);
}

// kerrLaunch (Kerr.h:110-148) into a lane.
__device__ __forceinline__ void k_init(KLane& l, float3 origin, float3 direction, const MarchUniforms& u) {
    const float a = u.spin;
    KerrState<float> s0 = kerr_launch(a, to_v3<float>(origin), to_v3<float>(direction));
    l.s = KState{s0.r, s0.theta, s0.phi, s0.pr, s0.ptheta};
    l.c = KState{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    l.k = k_const(a, s0.energy, s0.angularMomentum);
    l.carter0 = kerr_carter(a, s0);
    l.scale = fmaxf(fabsf(l.carter0), s0.energy * s0.energy);
    l.capture = kerr_outer_horizon(a) + KERR_CAPTURE_MARGIN;
    l.drift = 0.0f;
    l.color = make_float3(0.0f, 0.0f, 0.0f);
    l.transmittance = 1.0f;
    l.travelled = l.weighted_depth = l.depth_weight = 0.0f;
    float st, ct;
    fast_sincos(l.s.th, &st, &ct);
    l.previous = k_position(l, st, ct);
    l.steps = l.samples = 0;
    l.outcome = RayExhausted;
    l.min_r = l.s.r;
}

// One iteration of marchRayKerr's loop (march.metal:140-173).
__device__ __forceinline__ bool k_step(KLane& l, const MarchUniforms& u, cudaTextureObject_t em, cudaTextureObject_t vel,
                                       bool gather) {
    const GeodesicSettings& g = u.geodesic;
    if (l.steps >= g.stepCap) return true;
    // kerrStepLength (Kerr.h:177-186)
    float st0, ct0;
    fast_sincos(l.s.th, &st0, &ct0);
    float above = l.s.r - (l.capture - KERR_CAPTURE_MARGIN);
    float pole = fminf(fmaxf(st0 * (1.0f / 0.08f), 0.05f), 1.0f);
    float h = fminf(fmaxf(fminf(g.stepFactor * l.s.r, 0.2f * above) * pole, 0.002f), g.stepMax);
    KState inc = k_increment(l.k, l.s, h);
    comp_add(l.s.r, l.c.r, inc.r);
    comp_add(l.s.th, l.c.th, inc.th);
    comp_add(l.s.ph, l.c.ph, inc.ph);
    comp_add(l.s.pr, l.c.pr, inc.pr);
    comp_add(l.s.pt, l.c.pt, inc.pt);
    l.steps += 1u;
    float st, ct;
    fast_sincos(l.s.th, &st, &ct);
    float3 position = k_position(l, st, ct);
    float3 d = position - l.previous;
    float path = sqrtf(dot3(d, d));
    l.travelled += path;
    float carter, residual;
    k_gauges(l, st, ct, &carter, &residual);
    float cd = fabsf(carter - l.carter0) / l.scale;
    float nd = fabsf(residual) / (l.scale * fmaxf(l.s.r * l.s.r, 1.0f));
    l.drift = fmaxf(l.drift, fmaxf(cd, nd));
    l.min_r = fminf(l.min_r, l.s.r);
    if (l.s.r <= l.capture) {
        l.outcome = RayCaptured;
        return true;
    }
    if (gather && in_slab(position, u.volumeHalfExtent) && l.transmittance > 0.004f) {
        float sigma = fmaf(l.k.a2, ct * ct, l.s.r * l.s.r);
        float fk = 1.0f - 2.0f * l.s.r / sigma;
        KerrState<float> ks{l.s.r, l.s.th, l.s.ph, l.s.pr, l.s.pt, l.k.E, l.k.L};
        float3 dir = to_float3(kerr_direction(l.k.a, ks));
        gather_sample(gather_view(u, em, vel), position, fmaxf(fk, 0.0f), dir, path, l.travelled, l.color,
                      l.transmittance, l.weighted_depth, l.depth_weight, l.samples);
    }
    l.previous = position;
    if (l.s.r >= g.escapeRadius) {
        l.outcome = RayEscaped;
        return true;
    }
    return false;
}

__device__ __forceinline__ PixelResult k_finish(const KLane& l, const MarchUniforms& u, const float4* blackbody) {
    PixelResult r;
    r.color = l.color;
    r.drift = l.drift;
    r.steps = l.steps;
    r.outcome = l.outcome;
    r.depth = l.depth_weight > 0.0f ? l.weighted_depth / l.depth_weight : l.travelled;
    r.min_r = l.min_r;
    r.samples = l.samples;
    bool falls_in = l.outcome == RayCaptured || (l.outcome == RayExhausted && l.s.pr < 0.0f);
    if (!falls_in && u.starBrightness > 0.0f) {
        KerrState<float> ks{l.s.r, l.s.th, l.s.ph, l.s.pr, l.s.pt, l.k.E, l.k.L};
        float3 star = starfield(to_float3(kerr_direction(l.k.a, ks)), u.starSeed, blackbody);
        r.color = r.color + star * (l.transmittance * u.starBrightness);
    }
    return r;
}

// probeRays' result fields (march.metal:303-340) from a finished lane.
__device__ inline RayProbeResult s_probe_result(const SLane& l, const MarchUniforms& u, const SweepTables& t) {
    RayProbeResult out;
    float sn, cs;
    float3 pos = s_position(l, &sn, &cs);
    float3 dir = (l.outcome == RayEscaped && !s_falls_in(l)) ? s_sky(l, u, t) : s_direction(l, sn, cs);
    out.position = {pos.x, pos.y, pos.z};
    out.direction = {dir.x, dir.y, dir.z};
    out.drift = s_drift(l);
    out.outcome = l.outcome;
    out.steps = l.steps;
    double r = (double)l.s.r + (double)l.c.r;
    out.energy = (float)((1.0 - 2.0 / r) * ((double)l.s.vd + (double)l.c.vd) - ((double)l.s.rd + (double)l.c.rd));
    out.angularMomentum = (float)(r * r * ((double)l.s.pd + (double)l.c.pd));
    return out;
}

__device__ inline RayProbeResult k_probe_result(const KLane& l) {
    RayProbeResult out;
    float st, ct;
    fast_sincos(l.s.th, &st, &ct);
    float3 pos = k_position(l, st, ct);
    KerrState<float> ks{l.s.r, l.s.th, l.s.ph, l.s.pr, l.s.pt, l.k.E, l.k.L};
    float3 dir = to_float3(kerr_direction(l.k.a, ks));
    out.position = {pos.x, pos.y, pos.z};
    out.direction = {dir.x, dir.y, dir.z};
    out.drift = l.drift;
    out.outcome = l.outcome;
    out.steps = l.steps;
    out.energy = l.k.E;
    out.angularMomentum = l.k.L;
    return out;
}

// One pixel through the compensated path, run to completion.
__device__ inline PixelResult shade_pixel_compensated(const MarchParams& p, uint32_t px, uint32_t py) {
    const MarchUniforms& u = p.u;
    const bool gather = p.emission != 0;
    float3 dir = camera_direction(u, px, py);
    float3 origin = to_f3(u.cameraPosition);
    if (u.spin > 0.0f) {
        KLane l;
        k_init(l, origin, dir, u);
        for (uint32_t k = 0; k <= STEP_CAP_STILL; ++k)
            if (k_step(l, u, p.emission, p.velocity, gather)) break;
        return k_finish(l, u, p.blackbody);
    }
    SLane l;
    float3 sky;
    if (s_init(l, origin, dir, u, p.tables, &sky)) return sky_only_result(sky, u, p.blackbody);
    for (uint32_t k = 0; k <= STEP_CAP_STILL; ++k)
        if (s_step(l, u, p.emission, p.velocity, gather)) break;
    return s_finish(l, u, p.tables, p.blackbody);
}

}  // namespace gg
