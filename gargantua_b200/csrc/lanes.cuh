// The compensated march as a per-lane state machine: init from a camera
// ray, advance one RK4 step at a time, finish with the starfield. The served
// persistent kernels refill lanes between steps; the compensated image and
// probe kernels run one lane to completion; the FP64 re-integration runs the
// same code in double. All therefore execute the same algorithm, and the
// goldens check the FP32 instantiation through gg_probe.
//
// Against the reference's march (march.metal:51-184):
//  - the same RK4 steps, step policy, capture/escape/sphere-exit logic and
//    gather, so ray-step counts are the reference's;
//  - in FP32 each state += increment is TwoSum-compensated (comp_add);
//  - one reciprocal per Schwarzschild derivative instead of four divides,
//    using vDotDot = r phiDot^2 - vDot^2/r^2 appearing inside rDotDot; the
//    Kerr derivative uses three reciprocals instead of eleven divides;
//  - the four RK4 stages are written as a loop and unrolled: the stage
//    weights and offsets become constants and the stage branches go (on
//    the served stream 15 % faster than the loop kept rolled);
//  - sin and cos from a Cody-Waite reduction by pi/2 and Taylor series on
//    |r| <= pi/4 (through r^9 / r^10 in FP32, r^17 / r^18 in FP64), and
//    reciprocals from rcp.approx (FP32: within one ulp; FP64: refined by
//    two Newton steps to full precision), instead of library calls with slow
//    paths; the sine and cosine of the polar angle at the start of a Kerr
//    step are carried over from the end of the previous one;
//  - the Eddington-Finkelstein time v, which nothing downstream reads, is
//    not integrated.
#pragma once

#include "march.cuh"

namespace gg {

// ----------------------------------------------------------------- math

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
    float ps = fmaf(r2, (float)(1.0 / 362880.0), (float)(-1.0 / 5040.0));
    ps = fmaf(r2, ps, (float)(1.0 / 120.0));
    ps = fmaf(r2, ps, (float)(-1.0 / 6.0));
    float sr = fmaf(r * r2, ps, r);
    // cos r = 1 + r^2 (-1/2 + r^2 (1/4! + r^2 (-1/6! + r^2 (1/8! - r^2/10!))))
    float pc = fmaf(r2, (float)(-1.0 / 3628800.0), (float)(1.0 / 40320.0));
    pc = fmaf(r2, pc, (float)(-1.0 / 720.0));
    pc = fmaf(r2, pc, (float)(1.0 / 24.0));
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

// sin and cos of a double angle of moderate size: the same reduction with
// pi/2 in three parts and the series through r^17 and r^18.
__device__ __forceinline__ void fast_sincos(double x, double* s_out, double* c_out) {
    const double two_over_pi = 6.36619772367581382433e-01;
    const double pio2_hi = 1.57079601287841796875e+00;
    const double pio2_mid = 3.13916478650481311129e-07;
    const double pio2_lo = 1.05629990669874276403e-23;
    double k = rint(x * two_over_pi);
    double r = fma(-k, pio2_hi, x);
    r = fma(-k, pio2_mid, r);
    r = fma(-k, pio2_lo, r);
    double r2 = r * r;
    double ps = fma(r2, 1.0 / 355687428096000.0, -1.0 / 1307674368000.0);
    ps = fma(r2, ps, 1.0 / 6227020800.0);
    ps = fma(r2, ps, -1.0 / 39916800.0);
    ps = fma(r2, ps, 1.0 / 362880.0);
    ps = fma(r2, ps, -1.0 / 5040.0);
    ps = fma(r2, ps, 1.0 / 120.0);
    ps = fma(r2, ps, -1.0 / 6.0);
    double sr = fma(r * r2, ps, r);
    double pc = fma(r2, 1.0 / 6402373705728000.0, -1.0 / 20922789888000.0);
    pc = fma(r2, pc, 1.0 / 87178291200.0);
    pc = fma(r2, pc, -1.0 / 479001600.0);
    pc = fma(r2, pc, 1.0 / 3628800.0);
    pc = fma(r2, pc, -1.0 / 40320.0);
    pc = fma(r2, pc, 1.0 / 720.0);
    pc = fma(r2, pc, -1.0 / 24.0);
    pc = fma(r2, pc, 0.5);
    double cr = fma(-r2, pc, 1.0);
    long long q = (long long)k;
    double s = (q & 1) ? cr : sr;
    double c = (q & 1) ? sr : cr;
    if (q & 2) s = -s;
    if ((q + 1) & 2) c = -c;
    *s_out = s;
    *c_out = c;
}

__device__ __forceinline__ float fmaT(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float rsqrtT(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrtT(double x) { return rcp(sqrt(x)); }


// x += y. Compensated FP32 carries the rounding error in e (TwoSum,
// march.cuh); plain FP32 and FP64 add directly and leave e at zero.
template <bool Comp> __device__ __forceinline__ void comp_addT(float& x, float& e, float y) {
    if constexpr (Comp) {
        comp_add(x, e, y);
    } else {
        x += y;
    }
}
template <bool Comp> __device__ __forceinline__ void comp_addT(double& x, double& e, double y) { x += y; }

template <typename R> __device__ __forceinline__ V3<R> v3_of(float3 a) { return v3<R>(R(a.x), R(a.y), R(a.z)); }

// ------------------------------------------------------------ Schwarzschild

template <typename R> struct SState {
    R r, phi, vd, rd, pd;
};

// Geodesic equations (Geodesic.h:42-49) with one reciprocal.
template <typename R> __device__ __forceinline__ SState<R> s_derivative(const SState<R>& s) {
    R inv_r = rcp(s.r);
    R inv_r2 = inv_r * inv_r;
    R vdd = s.r * (s.pd * s.pd) - (s.vd * s.vd) * inv_r2;
    R f = fmaT(R(-2), inv_r, R(1));
    R rdd = fmaT(f, vdd, R(2) * (s.rd * s.vd) * inv_r2);
    R pdd = R(-2) * (s.rd * s.pd) * inv_r;
    return SState<R>{s.rd, s.pd, vdd, rdd, pdd};
}

template <typename R> __device__ __forceinline__ SState<R> s_offset(const SState<R>& s, const SState<R>& k, R w) {
    return SState<R>{fmaT(k.r, w, s.r), fmaT(k.phi, w, s.phi), fmaT(k.vd, w, s.vd), fmaT(k.rd, w, s.rd),
                     fmaT(k.pd, w, s.pd)};
}

// The RK4 increment (k1 + 2 k2 + 2 k3 + k4) h / 6 (Geodesic.h:52-59).
template <typename R> __device__ __forceinline__ SState<R> s_increment(const SState<R>& s, R h) {
    SState<R> acc{R(0), R(0), R(0), R(0), R(0)};
    SState<R> x = s;
#pragma unroll
    for (int stage = 0; stage < 4; ++stage) {
        SState<R> k = s_derivative(x);
        R wk = (stage == 0 || stage == 3) ? R(1) : R(2);
        acc = s_offset(acc, k, wk);
        x = s_offset(s, k, stage < 2 ? R(0.5) * h : h);
    }
    const R w = h * (R(1) / R(6));
    return SState<R>{acc.r * w, acc.phi * w, acc.vd * w, acc.rd * w, acc.pd * w};
}

template <typename R> struct SLane {
    SState<R> s, c;  // value and TwoSum error word (FP32)
    V3<R> e1, e2;
    R energy, angular_momentum;  // launch values (the reference's ray.energy, ray.angularMomentum)
    double e0, l0;               // E and L of the state integration starts from, in double
    float pre_drift;             // renormalised lanes: max over steps of the drift before projection
    float3 color;
    float transmittance, travelled, weighted_depth, depth_weight;
    V3<R> previous;
    uint32_t steps, samples, outcome;
    float min_r;
    bool left_sphere;
};

template <typename R> __device__ __forceinline__ V3<R> s_position(const SLane<R>& l, R* sn, R* cs) {
    fast_sincos(l.s.phi, sn, cs);
    return v3<R>(l.s.r * fmaT(*cs, l.e1.x, *sn * l.e2.x), l.s.r * fmaT(*cs, l.e1.y, *sn * l.e2.y),
                 l.s.r * fmaT(*cs, l.e1.z, *sn * l.e2.z));
}

// Static-observer direction at the ray's radius (Geodesic.h:94-100).
template <typename R> __device__ __forceinline__ V3<R> s_direction(const SLane<R>& l, R sn, R cs) {
    V3<R> radial = v3<R>(fmaT(cs, l.e1.x, sn * l.e2.x), fmaT(cs, l.e1.y, sn * l.e2.y), fmaT(cs, l.e1.z, sn * l.e2.z));
    V3<R> tang = v3<R>(fmaT(-sn, l.e1.x, cs * l.e2.x), fmaT(-sn, l.e1.y, cs * l.e2.y), fmaT(-sn, l.e1.z, cs * l.e2.z));
    R a = l.s.rd * rsqrtT(gmax(R(1) - R(2) * rcp(l.s.r), R(1e-6)));
    R b = l.s.r * l.s.pd;
    V3<R> local = v3<R>(fmaT(a, radial.x, b * tang.x), fmaT(a, radial.y, b * tang.y), fmaT(a, radial.z, b * tang.z));
    R len2 = dot(local, local);
    return len2 > R(0) ? local * rsqrtT(len2) : radial;
}

// prepareRay (Geodesic.h:130-163) into a lane. Returns true when the ray is
// sky-only; then *sky holds its asymptotic direction.
template <typename R>
__device__ __forceinline__ bool s_init(SLane<R>& l, V3<R> origin, V3<R> direction, const MarchUniforms& u,
                                       const SweepTables& t, float3* sky) {
    PreparedRay<R> p = prepare_ray(origin, direction, u, t);
    l.e1 = p.ray.e1;
    l.e2 = p.ray.e2;
    l.energy = p.ray.energy;
    l.angular_momentum = p.ray.angularMomentum;
    if (p.skyOnly) {
        *sky = to_float3(p.sky);
        return true;
    }
    l.s = SState<R>{p.ray.s.r, p.ray.s.phi, p.ray.s.vDot, p.ray.s.rDot, p.ray.s.phiDot};
    l.c = SState<R>{R(0), R(0), R(0), R(0), R(0)};
    double r0 = (double)l.s.r;
    l.e0 = (1.0 - 2.0 / r0) * (double)l.s.vd - (double)l.s.rd;
    l.l0 = r0 * r0 * (double)l.s.pd;
    l.pre_drift = 0.0f;
    l.color = make_float3(0.0f, 0.0f, 0.0f);
    l.transmittance = 1.0f;
    l.travelled = l.weighted_depth = l.depth_weight = 0.0f;
    R sn, cs;
    l.previous = s_position(l, &sn, &cs);
    l.steps = l.samples = 0;
    l.outcome = RayExhausted;
    l.min_r = (float)l.s.r;
    l.left_sphere = false;
    return false;
}

template <typename R>
__device__ __forceinline__ bool s_init(SLane<R>& l, float3 origin, float3 direction, const MarchUniforms& u,
                                       const SweepTables& t, float3* sky) {
    return s_init(l, v3_of<R>(origin), v3_of<R>(direction), u, t, sky);
}

template <typename R, bool Comp> __device__ __forceinline__ void s_advance(SState<R>& s, SState<R>& c, R h) {
    SState<R> inc = s_increment(s, h);
    comp_addT<Comp>(s.r, c.r, inc.r);
    comp_addT<Comp>(s.phi, c.phi, inc.phi);
    comp_addT<Comp>(s.vd, c.vd, inc.vd);
    comp_addT<Comp>(s.rd, c.rd, inc.rd);
    comp_addT<Comp>(s.pd, c.pd, inc.pd);
}

// value + error word of a compensated component, set from a double.
__device__ __forceinline__ void set_pair(float& x, float& e, double v) {
    x = (float)v;
    e = (float)(v - (double)x);
}
__device__ __forceinline__ void set_pair(double& x, double& e, double v) {
    x = v;
    e = 0.0;
}

// Hamiltonian-constraint renormalisation of a Schwarzschild state (the
// constraint of Schwarzschild.swift:115-117): with L0 and E0 the values the
// integration started from, set phiDot = L0 / r^2 and rDot, vDot on the
// null cone -f vDot^2 + 2 vDot rDot + r^2 phiDot^2 = 0 with E = f vDot -
// rDot = E0: rDot = sign(rDot) sqrt(E0^2 - f L0^2 / r^2), and vDot = (E0 +
// rDot) / f, written as (L0^2 / r^2) / (E0 - rDot) for an ingoing ray so
// that nothing cancels near the horizon. rDot is only replaced when the root
// is real and within kProjectLimit of |rDot|: near a radial turning point
// (rDot ~ 0) a small error in the root is a large change of direction, and
// projecting there moved endpoints away from the FP64 integration; there
// rDot is kept and vDot follows from E0. Evaluated in double from value
// plus error word. Before projecting, the state's drift against E0, L0
// joins the lane's running maximum, so the reported drift is the
// integrator's own per-step error, not the roundoff the projection leaves.
constexpr double kProjectLimit = 1e-3;

template <typename R> __device__ __forceinline__ void s_project(SLane<R>& l) {
    const double r = (double)l.s.r + (double)l.c.r;
    const double f = 1.0 - 2.0 / r;
    const double vd = (double)l.s.vd + (double)l.c.vd, rd = (double)l.s.rd + (double)l.c.rd;
    const double pd = (double)l.s.pd + (double)l.c.pd;
    const double pre = fmax(fabs(f * vd - rd - l.e0) / fabs(l.e0), fabs(r * r * pd - l.l0) / fmax(fabs(l.l0), 1e-3));
    l.pre_drift = fmaxf(l.pre_drift, (float)pre);
    const double inv_r2 = 1.0 / (r * r);
    const double l2 = l.l0 * l.l0 * inv_r2;
    const double disc = l.e0 * l.e0 - f * l2;
    double rd_new = rd, vd_new = (l.e0 + rd) / f;
    if (disc > 0.0) {
        const double root = sqrt(disc);
        if (fabs(root - fabs(rd)) <= kProjectLimit * fabs(rd)) {
            rd_new = rd < 0.0 ? -root : root;
            vd_new = rd < 0.0 ? l2 / (l.e0 + root) : (l.e0 + root) / f;
        }
    }
    set_pair(l.s.pd, l.c.pd, l.l0 * inv_r2);
    set_pair(l.s.rd, l.c.rd, rd_new);
    set_pair(l.s.vd, l.c.vd, vd_new);
}

// One iteration of marchRay's loop (march.metal:65-106). Returns true when
// the ray ended (captured, escaped, left the sphere or hit the step cap).
// Project: renormalise the state after each step (s_project).
template <typename R, bool Comp = true, bool Project = false>
__device__ __forceinline__ bool s_step(SLane<R>& l, const MarchUniforms& u, cudaTextureObject_t em,
                                       cudaTextureObject_t vel, bool gather) {
    const GeodesicSettings& g = u.geodesic;
    if (l.steps >= g.stepCap) return true;
    R h = ray_step_length(l.previous.z, l.s.r, g);
    const R sphere = R(u.sphereRadius);
    SState<R> before = l.s, before_c = l.c;
    s_advance<R, Comp>(l.s, l.c, h);
    l.steps += 1u;
    if (u.sphereRadius > 0.0f && l.s.r >= sphere && l.s.rd > R(0) && before.r < sphere) {
        R frac = (sphere - before.r) / (l.s.r - before.r);
        l.s = before;
        l.c = before_c;
        s_advance<R, Comp>(l.s, l.c, h * frac);
    }
    if constexpr (Project) s_project(l);
    R sn, cs;
    V3<R> position = s_position(l, &sn, &cs);
    V3<R> d = position - l.previous;
    float path = (float)asqrt(dot(d, d));
    l.travelled += path;
    l.min_r = fminf(l.min_r, (float)l.s.r);
    if (l.s.r <= R(g.captureRadius)) {
        l.outcome = RayCaptured;
        return true;
    }
    float3 pf = to_float3(position);
    if (gather && in_slab(pf, u.volumeHalfExtent) && l.transmittance > 0.004f) {
        float f = (float)fmaT(R(-2), rcp(l.s.r), R(1));
        gather_sample_with<true>(gather_view(u, em, vel), pf, f, [&] { return to_float3(s_direction(l, sn, cs)); }, path,
                           l.travelled, l.color, l.transmittance, l.weighted_depth, l.depth_weight, l.samples);
    }
    l.previous = position;
    if (u.sphereRadius > 0.0f && l.s.r >= sphere && l.s.rd > R(0)) {
        l.outcome = RayEscaped;
        l.left_sphere = true;
        return true;
    }
    if (l.s.r >= R(g.escapeRadius)) {
        l.outcome = RayEscaped;
        return true;
    }
    return false;
}

// Drift against the launch values (Geodesic.h:184-188), evaluated in double
// from value plus error word.
template <typename R> __device__ __forceinline__ float s_drift(const SLane<R>& l) {
    double r = (double)l.s.r + (double)l.c.r;
    double e = (1.0 - 2.0 / r) * ((double)l.s.vd + (double)l.c.vd) - ((double)l.s.rd + (double)l.c.rd);
    double lm = r * r * ((double)l.s.pd + (double)l.c.pd);
    double ed = fabs(e - l.e0) / fabs(l.e0);
    double ld = fabs(lm - l.l0) / fmax(fabs(l.l0), 1e-3);
    return fmaxf(l.pre_drift, (float)fmax(ed, ld));
}

template <typename R> __device__ __forceinline__ bool s_falls_in(const SLane<R>& l) {
    return l.outcome == RayCaptured ||
           (l.outcome == RayExhausted && l.s.rd < R(0) && gabs(l.angular_momentum) < R(B_CRITICAL) * l.energy);
}

// Final sky direction: the sphere-exit asymptote or the last direction.
template <typename R>
__device__ __forceinline__ V3<R> s_sky(const SLane<R>& l, const MarchUniforms& u, const SweepTables& t) {
    R sn, cs;
    if (l.left_sphere) {
        float b = (float)(gabs(l.angular_momentum) / l.energy);
        float sweep = sweep_lookup(t.sphere, 0.0f, u.sphereTableMaxB, b);
        fast_sincos(l.s.phi + R(sweep), &sn, &cs);
        return v3<R>(fmaT(cs, l.e1.x, sn * l.e2.x), fmaT(cs, l.e1.y, sn * l.e2.y), fmaT(cs, l.e1.z, sn * l.e2.z));
    }
    fast_sincos(l.s.phi, &sn, &cs);
    return s_direction(l, sn, cs);
}

template <typename R>
__device__ __forceinline__ PixelResult s_finish(const SLane<R>& l, const MarchUniforms& u, const SweepTables& t,
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
        float3 star = starfield(to_float3(s_sky(l, u, t)), u.starSeed, blackbody);
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

template <typename R> struct KState {
    R r, th, ph, pr, pt;
};

template <typename R> struct KConst {
    R a, a2, E, L, aE, aL, L2, a2E2, two_aEL, four_E;
};

template <typename R> __device__ __forceinline__ KConst<R> k_const(R a, R E, R L) {
    KConst<R> k;
    k.a = a;
    k.a2 = a * a;
    k.E = E;
    k.L = L;
    k.aE = a * E;
    k.aL = a * L;
    k.L2 = L * L;
    k.a2E2 = k.a2 * E * E;
    k.two_aEL = R(2) * a * E * L;
    k.four_E = R(4) * E;
    return k;
}

// 1/max(sin^2, floor) and 1/max(sin, floor) (Kerr.h:32, :78). In FP32 the
// floors are 1e-8 = (1e-4)^2 and 1e-4, so one reciprocal of max(|sin|,
// 1e-4) gives both; the FP64 floors are the oracle's 1e-12 and 1e-9.
template <typename R> __device__ __forceinline__ void k_sin_inverses(R st, R* inv_sin2, R* inv_sin_clamped) {
    if constexpr (sizeof(R) == 4) {
        R inv = rcp(fmaxf(fabsf(st), 1e-4f));
        *inv_sin2 = inv * inv;
        *inv_sin_clamped = st > 0.0f ? inv : 1e4f;
    } else {
        *inv_sin2 = rcp(fmax(st * st, 1e-12));
        *inv_sin_clamped = rcp(fmax(st, 1e-9));
    }
}

template <typename R> __device__ __forceinline__ R k_sin2(R st) { return gmax(st * st, R(sizeof(R) == 4 ? 1e-8 : 1e-12)); }

// Hamilton's equations with the off-shell Sigma terms (Kerr.h:63-90), at a
// polar angle whose sine and cosine are given, returned as Sigma times the
// derivative (every component carries the factor 1/Sigma, which the caller
// folds into its RK4 weights) with 1/Sigma in *inv_sigma_out. Also returns
// F = 2 Sigma H, the null residual of the state (Kerr.h:44-50), and
// 1/sin^2.
template <typename R>
__device__ __forceinline__ KState<R> k_derivative(const KConst<R>& k, const KState<R>& s, R st, R ct, R* F_out,
                                                  R* inv_sin2_out, R* inv_sigma_out) {
    const R r = s.r;
    const R r2 = r * r;
    const R delta = fmaT(r, r - R(2), k.a2);  // r^2 - 2r + a^2
    const R sigma = fmaT(k.a2, ct * ct, r2);
    const R inv_sigma = rcp(sigma);
    const R inv_delta = rcp(delta);
    const R sin2 = k_sin2(st);
    R inv_sin2, inv_sc;
    k_sin_inverses(st, &inv_sin2, &inv_sc);
    const R p = fmaT(r2 + k.a2, k.E, -k.aL);
    const R g = fmaT(k.a2E2, sin2, fmaT(k.L2, inv_sin2, -k.two_aEL));
    const R pr2 = s.pr * s.pr;
    const R p2d = p * p * inv_delta;
    const R F = fmaT(delta, pr2, fmaT(s.pt, s.pt, g - p2d));
    *F_out = F;
    *inv_sin2_out = inv_sin2;
    // With 2H = F / Sigma: dp_r = (2 r H - fr / 2) / Sigma, and
    // dp_theta = (-2 a^2 sin cos H - fth / 2) / Sigma where
    // fth / 2 = cos (a^2 E^2 sin - L^2 / (sin^2 |sin|)).
    const R two_h = F * inv_sigma;
    const R dprime = fmaT(R(2), r, R(-2));
    const R fr = fmaT(dprime, pr2, inv_delta * fmaT(p2d, dprime, -k.four_E * r * p));
    *inv_sigma_out = inv_sigma;
    KState<R> o;
    o.r = delta * s.pr;
    o.th = s.pt;
    o.ph = fmaT(k.a, p * inv_delta, k.L * inv_sin2) - k.aE;
    o.pr = fmaT(r, two_h, R(-0.5) * fr);
    o.pt = -ct * fmaT(k.a2 * st, two_h, fmaT(k.a2E2, st, -k.L2 * inv_sin2 * inv_sc));
    return o;
}

template <typename R> __device__ __forceinline__ KState<R> k_offset(const KState<R>& s, const KState<R>& d, R w) {
    return KState<R>{fmaT(d.r, w, s.r), fmaT(d.th, w, s.th), fmaT(d.ph, w, s.ph), fmaT(d.pr, w, s.pr),
                     fmaT(d.pt, w, s.pt)};
}

// sin and cos of theta0 + delta from those of theta0, for |delta| <= 0.35:
// the angle-addition formulas with Taylor polynomials of sin delta (through
// delta^7, remainder below 2.2e-10) and cos delta (through delta^8,
// remainder below 8e-12); for |delta| <= 0.02, the usual size of a stage's
// offset, through delta^3 and delta^4 (remainders below 2.7e-11 and 9e-14).
// False (nothing written) for larger |delta|.
__device__ __forceinline__ bool sincos_shift(float st0, float ct0, float delta, float* st, float* ct) {
    if (!(fabsf(delta) <= 0.35f)) return false;
    float d2 = delta * delta;
    if (fabsf(delta) <= 0.02f) {
        float sd = fmaf(delta * d2, (float)(-1.0 / 6.0), delta);
        float cd = fmaf(d2, fmaf(d2, (float)(1.0 / 24.0), -0.5f), 1.0f);
        *st = fmaf(st0, cd, ct0 * sd);
        *ct = fmaf(ct0, cd, -(st0 * sd));
        return true;
    }
    float ps = fmaf(d2, (float)(-1.0 / 5040.0), (float)(1.0 / 120.0));
    ps = fmaf(d2, ps, (float)(-1.0 / 6.0));
    float sd = fmaf(delta * d2, ps, delta);
    float pc = fmaf(d2, (float)(1.0 / 40320.0), (float)(-1.0 / 720.0));
    pc = fmaf(d2, pc, (float)(1.0 / 24.0));
    pc = fmaf(d2, pc, -0.5f);
    float cd = fmaf(d2, pc, 1.0f);
    *st = fmaf(st0, cd, ct0 * sd);
    *ct = fmaf(ct0, cd, -(st0 * sd));
    return true;
}

// The conserved-quantity gauge of a state, before the division by
// max(|Q0|, E^2) (Kerr.h:39-50; march.metal:160-163): the larger of
// |Q - Q0| and |2 Sigma H| / max(r^2, 1).
template <typename R> __device__ __forceinline__ R k_gauge(const KConst<R>& k, const KState<R>& s, R ct, R F,
                                                           R inv_sin2, R carter0) {
    R carter = fmaT(ct * ct, fmaT(k.L2, inv_sin2, -k.a2E2), s.pt * s.pt);
    return gmax(gabs(carter - carter0), gabs(F) * rcp(gmax(s.r * s.r, R(1))));
}

// RK4 increment (Kerr.h:92-99); (st0, ct0) are sin and cos of s.th. The
// first stage's derivative is evaluated at s itself, so it also yields the
// gauge of s: when `gauged`, *gauge becomes the larger of itself and it.
// The later stages take sin and cos of their polar angle by rotating
// (st0, ct0) through the stage's offset, which is small except near the
// poles; there the full reduction runs.
template <typename R>
__device__ __forceinline__ KState<R> k_increment(const KConst<R>& k, const KState<R>& s, R h, R st0, R ct0,
                                                 bool gauged, R carter0, R* gauge) {
    KState<R> acc{R(0), R(0), R(0), R(0), R(0)};
    KState<R> x = s;
    R st = st0, ct = ct0;
    R shift = R(0);
#pragma unroll
    for (int stage = 0; stage < 4; ++stage) {
        if (stage > 0) {
            if constexpr (sizeof(R) == 4) {
                if (!sincos_shift(st0, ct0, shift, &st, &ct)) fast_sincos(x.th, &st, &ct);
            } else {
                fast_sincos(x.th, &st, &ct);
            }
        }
        R F, inv_sin2, inv_sigma;
        KState<R> d = k_derivative(k, x, st, ct, &F, &inv_sin2, &inv_sigma);  // Sigma times the derivative
        if (stage == 0 && gauged) *gauge = gmax(*gauge, k_gauge(k, s, ct, F, inv_sin2, carter0));
        R wk = (stage == 0 || stage == 3) ? R(1) : R(2);
        acc = k_offset(acc, d, wk * inv_sigma);
        if (stage == 3) break;
        const R wx = (stage < 2 ? R(0.5) * h : h) * inv_sigma;
        x = k_offset(s, d, wx);
        shift = d.th * wx;
    }
    const R w = h * (R(1) / R(6));
    return KState<R>{acc.r * w, acc.th * w, acc.ph * w, acc.pr * w, acc.pt * w};
}

template <typename R> struct KLane {
    KState<R> s, c;
    KConst<R> k;
    R st, ct;  // sin and cos of s.th
    R sp, cp;  // sin and cos of s.ph (FP32: carried between steps, see k_step)
    R carter0, scale, capture;
    R gauge;  // max of k_gauge over the states after steps 1 .. steps-1
    float3 color;
    float transmittance, travelled, weighted_depth, depth_weight;
    V3<R> previous;
    uint32_t steps, samples, outcome;
    float min_r;
};

// Carter constant and null residual (Kerr.h:39-50) of the lane's state.
template <typename R> __device__ __forceinline__ void k_gauges(const KLane<R>& l, R* carter, R* residual) {
    const KConst<R>& k = l.k;
    R sin2 = k_sin2(l.st);
    R inv_sin2, inv_sc;
    k_sin_inverses(l.st, &inv_sin2, &inv_sc);
    *carter = fmaT(l.ct * l.ct, fmaT(k.L2, inv_sin2, -k.a2E2), l.s.pt * l.s.pt);
    R r = l.s.r;
    R delta = r * r - R(2) * r + k.a2;
    R p = fmaT(r * r + k.a2, k.E, -k.aL);
    R g = fmaT(k.a2E2, sin2, fmaT(k.L2, inv_sin2, -k.two_aEL));
    *residual = fmaT(delta, l.s.pr * l.s.pr, fmaT(l.s.pt, l.s.pt, g - p * p * rcp(delta)));
}

// The ray's drift (march.metal:160-163: the maximum over the states after
// every step): the steps' gauges so far and that of the final state,
// divided by max(|Q0|, E^2).
template <typename R> __device__ __forceinline__ float k_drift(const KLane<R>& l) {
    if (l.steps == 0u) return 0.0f;
    R carter, residual;
    k_gauges(l, &carter, &residual);
    R last = gmax(gabs(carter - l.carter0), gabs(residual) * rcp(gmax(l.s.r * l.s.r, R(1))));
    return (float)(gmax(l.gauge, last) / l.scale);
}

template <typename R> __device__ __forceinline__ V3<R> k_position(const KLane<R>& l, R* sp_out = nullptr,
                                                                 R* cp_out = nullptr) {
    R sp, cp;
    fast_sincos(l.s.ph, &sp, &cp);
    if (sp_out) *sp_out = sp;
    if (cp_out) *cp_out = cp;
    R radial = asqrt(fmaT(l.s.r, l.s.r, l.k.a2));
    return v3<R>(radial * l.st * cp, radial * l.st * sp, l.s.r * l.ct);
}

// The position from the lane's carried sin and cos of the azimuth.
template <typename R> __device__ __forceinline__ V3<R> k_position_carried(const KLane<R>& l) {
    R radial = asqrt(fmaT(l.s.r, l.s.r, l.k.a2));
    return v3<R>(radial * l.st * l.cp, radial * l.st * l.sp, l.s.r * l.ct);
}

// Direction of travel against the spherical frame (Kerr.h:158-173) from the
// lane's state, with the sines and cosines the step already has and
// reciprocals in place of the divides.
template <typename R> __device__ __forceinline__ V3<R> k_direction(const KLane<R>& l, R sp, R cp) {
    const KConst<R>& k = l.k;
    const R r = l.s.r, st = l.st, ct = l.ct;
    const R delta = fmaT(r, r - R(2), k.a2);
    const R inv_sigma = rcp(fmaT(k.a2, ct * ct, r * r));
    R inv_sin2, inv_sc;
    k_sin_inverses(st, &inv_sin2, &inv_sc);
    const R p = fmaT(r * r + k.a2, k.E, -k.aL);
    const R rdot = delta * l.s.pr * inv_sigma;
    const R r_thdot = r * l.s.pt * inv_sigma;
    const R r_st_phdot = r * st * ((fmaT(k.a, p * rcp(delta), k.L * inv_sin2) - k.aE) * inv_sigma);
    // rdot rhat + r thdot thhat + r sin phdot phhat, with rhat = (st cp, st sp, ct),
    // thhat = (ct cp, ct sp, -st), phhat = (-sp, cp, 0).
    const R in_plane = fmaT(rdot, st, r_thdot * ct);  // along (cp, sp, 0)
    V3<R> local = v3<R>(fmaT(in_plane, cp, -r_st_phdot * sp), fmaT(in_plane, sp, r_st_phdot * cp),
                        fmaT(rdot, ct, -r_thdot * st));
    R len2 = dot(local, local);
    return len2 > R(0) ? local * rsqrtT(len2) : v3<R>(st * cp, st * sp, ct);
}

// kerrLaunch (Kerr.h:110-148) into a lane.
template <typename R>
__device__ __forceinline__ void k_init(KLane<R>& l, V3<R> origin, V3<R> direction, const MarchUniforms& u) {
    const R a = R(u.spin);
    KerrState<R> s0 = kerr_launch(a, origin, direction);
    l.s = KState<R>{s0.r, s0.theta, s0.phi, s0.pr, s0.ptheta};
    l.c = KState<R>{R(0), R(0), R(0), R(0), R(0)};
    l.k = k_const(a, s0.energy, s0.angularMomentum);
    l.carter0 = kerr_carter(a, s0);
    l.scale = gmax(gabs(l.carter0), s0.energy * s0.energy);
    l.capture = kerr_outer_horizon(a) + R(KERR_CAPTURE_MARGIN);
    l.gauge = R(0);
    l.color = make_float3(0.0f, 0.0f, 0.0f);
    l.transmittance = 1.0f;
    l.travelled = l.weighted_depth = l.depth_weight = 0.0f;
    fast_sincos(l.s.th, &l.st, &l.ct);
    l.previous = k_position(l, &l.sp, &l.cp);
    l.steps = l.samples = 0;
    l.outcome = RayExhausted;
    l.min_r = (float)l.s.r;
}

template <typename R>
__device__ __forceinline__ void k_init(KLane<R>& l, float3 origin, float3 direction, const MarchUniforms& u) {
    k_init(l, v3_of<R>(origin), v3_of<R>(direction), u);
}

// Hamiltonian-constraint renormalisation of a Kerr state: |p_r| solved
// from 2 Sigma H = 0 (Kerr.h:39-50), Delta p_r^2 = P^2 / Delta - p_theta^2
// - g(theta), where that is positive (outside the outer horizon) and the
// new |p_r| is within kProjectLimit of the old (not near a radial turning
// point, as for Schwarzschild), keeping p_r's sign. E and L are parameters here
// and do not drift; p_theta and the Carter constant are left as integrated.
// Before projecting, the state's gauge (the larger of |Q - Q0| and |2 Sigma
// H| / max(r^2, 1)) joins the lane's running maximum, so the reported drift
// is the integrator's own per-step error. (st, ct) are sin and cos of the
// state's polar angle.
template <typename R> __device__ __forceinline__ void k_project(KLane<R>& l) {
    const KConst<R>& k = l.k;
    const R r = l.s.r;
    const R delta = fmaT(r, r - R(2), k.a2);
    R inv_sin2, inv_sc;
    k_sin_inverses(l.st, &inv_sin2, &inv_sc);
    const R p = fmaT(r * r + k.a2, k.E, -k.aL);
    const R g = fmaT(k.a2E2, k_sin2(l.st), fmaT(k.L2, inv_sin2, -k.two_aEL));
    const R rest = p * p * rcp(delta) - l.s.pt * l.s.pt - g;  // Delta p_r^2 on the null cone
    const R F = fmaT(delta, l.s.pr * l.s.pr, -rest);
    const R carter = fmaT(l.ct * l.ct, fmaT(k.L2, inv_sin2, -k.a2E2), l.s.pt * l.s.pt);
    l.gauge = gmax(l.gauge, gmax(gabs(carter - l.carter0), gabs(F) * rcp(gmax(r * r, R(1)))));
    if (delta > R(0) && rest > R(0)) {
        const R pr = sqrt(rest * rcp(delta));
        if (gabs(pr - gabs(l.s.pr)) <= R(kProjectLimit) * gabs(l.s.pr)) {
            l.s.pr = l.s.pr < R(0) ? -pr : pr;
            l.c.pr = R(0);
        }
    }
}

// One iteration of marchRayKerr's loop (march.metal:140-173). The drift of
// the state it starts from is folded in by k_increment (k_drift adds the
// final state's). Project: renormalise the state after each step
// (k_project).
template <typename R, bool Comp = true, bool Project = false>
__device__ __forceinline__ bool k_step(KLane<R>& l, const MarchUniforms& u, cudaTextureObject_t em,
                                       cudaTextureObject_t vel, bool gather) {
    const GeodesicSettings& g = u.geodesic;
    if (l.steps >= g.stepCap) return true;
    // kerrStepLength (Kerr.h:177-186)
    R above = l.s.r - (l.capture - R(KERR_CAPTURE_MARGIN));
    R pole = gmin(gmax(l.st * R(1.0 / 0.08), R(0.05)), R(1));
    R h = gmin(gmax(gmin(R(g.stepFactor) * l.s.r, R(0.2) * above) * pole, R(0.002)), R(g.stepMax));
    KState<R> inc = k_increment(l.k, l.s, h, l.st, l.ct, l.steps > 0u, l.carter0, &l.gauge);
    comp_addT<Comp>(l.s.r, l.c.r, inc.r);
    comp_addT<Comp>(l.s.th, l.c.th, inc.th);
    comp_addT<Comp>(l.s.ph, l.c.ph, inc.ph);
    comp_addT<Comp>(l.s.pr, l.c.pr, inc.pr);
    comp_addT<Comp>(l.s.pt, l.c.pt, inc.pt);
    l.steps += 1u;
    fast_sincos(l.s.th, &l.st, &l.ct);
    if constexpr (Project) k_project(l);
    // The azimuth enters only the Cartesian position (the metric is
    // axisymmetric), so in FP32 its sine and cosine are carried: rotated
    // through the step's own increment (|delta| <= 0.02: the short series of
    // sincos_shift, remainders below 3e-11), reduced afresh every 16 steps
    // and after any larger increment, so rounding does not build up.
    if constexpr (sizeof(R) == 4) {
        if ((l.steps & 15u) == 0u || !(gabs(inc.ph) <= R(0.02)) || !sincos_shift(l.sp, l.cp, inc.ph, &l.sp, &l.cp))
            fast_sincos(l.s.ph, &l.sp, &l.cp);
    } else {
        fast_sincos(l.s.ph, &l.sp, &l.cp);
    }
    const R sp = l.sp, cp = l.cp;
    V3<R> position = k_position_carried(l);
    V3<R> d = position - l.previous;
    float path = (float)asqrt(dot(d, d));
    l.travelled += path;
    l.min_r = fminf(l.min_r, (float)l.s.r);
    if (l.s.r <= l.capture) {
        l.outcome = RayCaptured;
        return true;
    }
    float3 pf = to_float3(position);
    if (gather && in_slab(pf, u.volumeHalfExtent) && l.transmittance > 0.004f) {
        R sigma = fmaT(l.k.a2, l.ct * l.ct, l.s.r * l.s.r);
        float fk = (float)(R(1) - R(2) * l.s.r * rcp(sigma));
        auto dir = [&] { return to_float3(k_direction(l, sp, cp)); };
        gather_sample_with<true>(gather_view(u, em, vel), pf, fmaxf(fk, 0.0f), dir, path, l.travelled, l.color,
                      l.transmittance, l.weighted_depth, l.depth_weight, l.samples);
    }
    l.previous = position;
    if (l.s.r >= R(g.escapeRadius)) {
        l.outcome = RayEscaped;
        return true;
    }
    return false;
}

template <typename R>
__device__ __forceinline__ PixelResult k_finish(const KLane<R>& l, const MarchUniforms& u, const float4* blackbody) {
    PixelResult r;
    r.color = l.color;
    r.drift = k_drift(l);
    r.steps = l.steps;
    r.outcome = l.outcome;
    r.depth = l.depth_weight > 0.0f ? l.weighted_depth / l.depth_weight : l.travelled;
    r.min_r = l.min_r;
    r.samples = l.samples;
    bool falls_in = l.outcome == RayCaptured || (l.outcome == RayExhausted && l.s.pr < R(0));
    if (!falls_in && u.starBrightness > 0.0f) {
        KerrState<R> ks{l.s.r, l.s.th, l.s.ph, l.s.pr, l.s.pt, l.k.E, l.k.L};
        float3 star = starfield(to_float3(kerr_direction(l.k.a, ks)), u.starSeed, blackbody);
        r.color = r.color + star * (l.transmittance * u.starBrightness);
    }
    return r;
}

// probeRays' result fields (march.metal:303-340) from a finished lane.
template <typename R>
__device__ inline RayProbeResult s_probe_result(const SLane<R>& l, const MarchUniforms& u, const SweepTables& t) {
    RayProbeResult out;
    R sn, cs;
    V3<R> pos = s_position(l, &sn, &cs);
    V3<R> dir = (l.outcome == RayEscaped && !s_falls_in(l)) ? s_sky(l, u, t) : s_direction(l, sn, cs);
    out.position = {(float)pos.x, (float)pos.y, (float)pos.z};
    out.direction = {(float)dir.x, (float)dir.y, (float)dir.z};
    out.drift = s_drift(l);
    out.outcome = l.outcome;
    out.steps = l.steps;
    double r = (double)l.s.r + (double)l.c.r;
    out.energy = (float)((1.0 - 2.0 / r) * ((double)l.s.vd + (double)l.c.vd) - ((double)l.s.rd + (double)l.c.rd));
    out.angularMomentum = (float)(r * r * ((double)l.s.pd + (double)l.c.pd));
    return out;
}

template <typename R> __device__ inline RayProbeResult k_probe_result(const KLane<R>& l) {
    RayProbeResult out;
    V3<R> pos = k_position(l);
    KerrState<R> ks{l.s.r, l.s.th, l.s.ph, l.s.pr, l.s.pt, l.k.E, l.k.L};
    V3<R> dir = kerr_direction(l.k.a, ks);
    out.position = {(float)pos.x, (float)pos.y, (float)pos.z};
    out.direction = {(float)dir.x, (float)dir.y, (float)dir.z};
    out.drift = k_drift(l);
    out.outcome = l.outcome;
    out.steps = l.steps;
    out.energy = (float)l.k.E;
    out.angularMomentum = (float)l.k.L;
    return out;
}

// One pixel through the lane path, run to completion: compensated FP32
// (renormalised with Project), or the FP64 re-integration with R = double.
template <typename R, bool Comp = true, bool Project = false>
__device__ inline PixelResult shade_pixel_lane(const MarchParams& p, uint32_t px, uint32_t py) {
    const MarchUniforms& u = p.u;
    const bool gather = p.emission != 0;
    float3 dir = camera_direction(u, px, py);
    float3 origin = to_f3(u.cameraPosition);
    if (u.spin > 0.0f) {
        KLane<R> l;
        k_init(l, origin, dir, u);
        for (uint32_t k = 0; k <= STEP_CAP_STILL; ++k)
            if (k_step<R, Comp, Project>(l, u, p.emission, p.velocity, gather)) break;
        return k_finish(l, u, p.blackbody);
    }
    SLane<R> l;
    float3 sky;
    if (s_init(l, origin, dir, u, p.tables, &sky)) return sky_only_result(sky, u, p.blackbody);
    for (uint32_t k = 0; k <= STEP_CAP_STILL; ++k)
        if (s_step<R, Comp, Project>(l, u, p.emission, p.velocity, gather)) break;
    return s_finish(l, u, p.tables, p.blackbody);
}

__device__ inline PixelResult shade_pixel_compensated(const MarchParams& p, uint32_t px, uint32_t py) {
    return shade_pixel_lane<float, true>(p, px, py);
}

// Compensated FP32 with the Hamiltonian-constraint renormalisation after
// every step.
__device__ inline PixelResult shade_pixel_renormalised(const MarchParams& p, uint32_t px, uint32_t py) {
    return shade_pixel_lane<float, true, true>(p, px, py);
}

// The plain FP32 march: the same lane code with direct adds.
__device__ inline PixelResult shade_pixel_plain(const MarchParams& p, uint32_t px, uint32_t py) {
    return shade_pixel_lane<float, false>(p, px, py);
}

}  // namespace gg
