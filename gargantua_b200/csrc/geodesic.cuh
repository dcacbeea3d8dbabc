// Null geodesics of Schwarzschild in ingoing Eddington-Finkelstein
// coordinates, reduced to each ray's orbital plane (Geodesic.h:1-236,
// Schwarzschild.swift:11-270). Templated on the real type: float for the
// march, double for the per-ray FP64 re-integration.
#pragma once

#include "common.cuh"

namespace gg {

template <typename R> struct V3 {
    R x, y, z;
};
template <typename R> __device__ __forceinline__ V3<R> v3(R x, R y, R z) { return V3<R>{x, y, z}; }
template <typename R> __device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename R> __device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename R> __device__ __forceinline__ V3<R> operator*(V3<R> a, R s) { return v3(a.x * s, a.y * s, a.z * s); }
template <typename R> __device__ __forceinline__ V3<R> operator*(R s, V3<R> a) { return v3(s * a.x, s * a.y, s * a.z); }
template <typename R> __device__ __forceinline__ R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ __forceinline__ float gsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double gsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float gabs(float x) { return fabsf(x); }
__device__ __forceinline__ double gabs(double x) { return fabs(x); }
__device__ __forceinline__ float gmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double gmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float gmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double gmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ void gsincos(float x, float* s, float* c) { sincosf(x, s, c); }
__device__ __forceinline__ void gsincos(double x, double* s, double* c) { sincos(x, s, c); }
__device__ __forceinline__ float gcos(float x) { return cosf(x); }
__device__ __forceinline__ double gcos(double x) { return cos(x); }
__device__ __forceinline__ float gsin(float x) { return sinf(x); }
__device__ __forceinline__ double gsin(double x) { return sin(x); }
__device__ __forceinline__ float gacos(float x) { return acosf(x); }
__device__ __forceinline__ double gacos(double x) { return acos(x); }
__device__ __forceinline__ float gatan2(float y, float x) { return atan2f(y, x); }
__device__ __forceinline__ double gatan2(double y, double x) { return atan2(y, x); }

template <typename R> __device__ __forceinline__ R length(V3<R> a) { return gsqrt(dot(a, a)); }
template <typename R> __device__ __forceinline__ V3<R> normalize(V3<R> a) { return a * (R(1) / length(a)); }
template <typename R> __device__ __forceinline__ V3<R> to_v3(float3 a) { return v3<R>(R(a.x), R(a.y), R(a.z)); }
template <typename R> __device__ __forceinline__ float3 to_float3(V3<R> a) { return make_float3((float)a.x, (float)a.y, (float)a.z); }

template <typename R> struct RayState {
    R v, r, phi, vDot, rDot, phiDot;
};

template <typename R> struct PlaneRay {
    RayState<R> s;
    V3<R> e1, e2;
    R energy, angularMomentum;
};

template <typename R> __device__ __forceinline__ R schwarzschild_f(R r) { return R(1) - R(R_SCHWARZSCHILD) / r; }

template <typename R> __device__ __forceinline__ RayState<R> ray_add(RayState<R> a, RayState<R> b) {
    return RayState<R>{a.v + b.v, a.r + b.r, a.phi + b.phi, a.vDot + b.vDot, a.rDot + b.rDot, a.phiDot + b.phiDot};
}
template <typename R> __device__ __forceinline__ RayState<R> ray_scale(RayState<R> a, R s) {
    return RayState<R>{a.v * s, a.r * s, a.phi * s, a.vDot * s, a.rDot * s, a.phiDot * s};
}

template <typename R> __device__ __forceinline__ R ray_energy(const RayState<R>& s) {
    return schwarzschild_f(s.r) * s.vDot - s.rDot;
}
template <typename R> __device__ __forceinline__ R ray_angular_momentum(const RayState<R>& s) {
    return s.r * s.r * s.phiDot;
}

// Euler-Lagrange equations of L = (1/2)(-f vDot^2 + 2 vDot rDot + r^2 phiDot^2)
// (Geodesic.h:42-49).
template <typename R> __device__ __forceinline__ RayState<R> ray_derivative(const RayState<R>& s) {
    R r = s.r;
    R r2 = r * r;
    R vdd = -s.vDot * s.vDot / r2 + r * s.phiDot * s.phiDot;
    R rdd = R(2) * s.rDot * s.vDot / r2 + schwarzschild_f(r) * (r * s.phiDot * s.phiDot - s.vDot * s.vDot / r2);
    R pdd = R(-2) * s.rDot * s.phiDot / r;
    return RayState<R>{s.vDot, s.rDot, s.phiDot, vdd, rdd, pdd};
}

// Classical RK4 (Geodesic.h:52-59); returns the increment (k1 + 2k2 + 2k3 +
// k4) h/6 so callers can accumulate it plainly or compensated.
template <typename R> __device__ __forceinline__ RayState<R> ray_increment(const RayState<R>& s, R h) {
    RayState<R> k1 = ray_derivative(s);
    RayState<R> k2 = ray_derivative(ray_add(s, ray_scale(k1, R(0.5) * h)));
    RayState<R> k3 = ray_derivative(ray_add(s, ray_scale(k2, R(0.5) * h)));
    RayState<R> k4 = ray_derivative(ray_add(s, ray_scale(k3, h)));
    RayState<R> sum = ray_add(ray_add(k1, ray_scale(k2, R(2))), ray_add(ray_scale(k3, R(2)), k4));
    return ray_scale(sum, h / R(6));
}

template <typename R> __device__ __forceinline__ RayState<R> ray_step(const RayState<R>& s, R h) {
    return ray_add(s, ray_increment(s, h));
}

// Launch from a point in a direction measured by a static observer there,
// local photon energy one (Geodesic.h:63-87, Schwarzschild.swift:76-97).
template <typename R> __device__ PlaneRay<R> launch_ray(V3<R> origin, V3<R> direction) {
    R r0 = length(origin);
    V3<R> e1 = origin * (R(1) / r0);
    V3<R> unit = normalize(direction);
    R dr = dot(unit, e1);
    V3<R> perpendicular = unit - dr * e1;
    R dphi = length(perpendicular);
    V3<R> e2;
    if (dphi < R(sizeof(R) == 4 ? 1e-6 : 1e-12)) {
        V3<R> helper = gabs(e1.x) < R(0.9) ? v3<R>(1, 0, 0) : v3<R>(0, 1, 0);
        e2 = normalize(helper - dot(helper, e1) * e1);
        dphi = R(0);
    } else {
        e2 = perpendicular * (R(1) / dphi);
    }
    R f0 = schwarzschild_f(r0);
    R root = gsqrt(f0);
    PlaneRay<R> ray;
    ray.s = RayState<R>{R(0), r0, R(0), (R(1) + dr) / root, root * dr, dphi / r0};
    ray.e1 = e1;
    ray.e2 = e2;
    ray.energy = ray_energy(ray.s);
    ray.angularMomentum = ray_angular_momentum(ray.s);
    return ray;
}

template <typename R> __device__ __forceinline__ V3<R> ray_position(const PlaneRay<R>& ray) {
    R s, c;
    gsincos(ray.s.phi, &s, &c);
    return ray.s.r * (c * ray.e1 + s * ray.e2);
}

// Direction a static observer at the ray's radius measures (Geodesic.h:94-100).
template <typename R> __device__ V3<R> ray_direction(const PlaneRay<R>& ray) {
    R s, c;
    gsincos(ray.s.phi, &s, &c);
    V3<R> radial = c * ray.e1 + s * ray.e2;
    V3<R> tangential = (-s) * ray.e1 + c * ray.e2;
    V3<R> local = (ray.s.rDot / gsqrt(gmax(schwarzschild_f(ray.s.r), R(1e-6)))) * radial +
                  (ray.s.r * ray.s.phiDot) * tangential;
    R len = length(local);
    return len > R(0) ? local * (R(1) / len) : radial;
}

// Table coordinate for b, remapped to texel centres (Geodesic.h:106-110).
__device__ __forceinline__ float sweep_coordinate(float low, float high, float b) {
    float x = fminf(fmaxf((b - low) / (high - low), 0.0f), 1.0f);
    float t = 1.0f - sqrtf(1.0f - x);
    return (t * ((float)SWEEP_TABLE_SIZE - 1.0f) + 0.5f) / (float)SWEEP_TABLE_SIZE;
}

__device__ __forceinline__ float sweep_lookup(const float* table, float low, float high, float b) {
    return table_lookup(table, SWEEP_TABLE_SIZE, sweep_coordinate(low, high, b));
}

template <typename R> __device__ __forceinline__ V3<R> asymptotic_direction(const PlaneRay<R>& ray, R phi) {
    R s, c;
    gsincos(phi, &s, &c);
    return c * ray.e1 + s * ray.e2;
}

struct SweepTables {
    const float* sphere;
    const float* camera;
    const float* sky;
};

template <typename R> struct PreparedRay {
    PlaneRay<R> ray;
    bool skyOnly;
    V3<R> sky;
};

// Skip the empty leg from the camera to the integration sphere
// (Geodesic.h:130-163): rays that never enter take their asymptote from the
// camera or sky table; the rest are placed on the sphere with their
// conserved E and L and the azimuth advanced by sphere - camera sweep.
template <typename R>
__device__ PreparedRay<R> prepare_ray(V3<R> origin, V3<R> direction, const MarchUniforms& u, const SweepTables& t) {
    PreparedRay<R> p;
    p.ray = launch_ray(origin, direction);
    p.skyOnly = false;
    p.sky = v3<R>(0, 0, 0);
    if (u.sphereRadius <= 0.0f || p.ray.s.r <= R(u.sphereRadius)) return p;
    float b = (float)(gabs(p.ray.angularMomentum) / p.ray.energy);
    if (p.ray.s.rDot >= R(0)) {
        float sweep = sweep_lookup(t.camera, 0.0f, u.cameraMaxB, b);
        p.skyOnly = true;
        p.sky = asymptotic_direction(p.ray, p.ray.s.phi + R(sweep));
        return p;
    }
    if (b >= u.sphereMaxB) {
        float sweep = sweep_lookup(t.sky, u.skyMinB, u.skyMaxB, b);
        p.skyOnly = true;
        p.sky = asymptotic_direction(p.ray, p.ray.s.phi + R(sweep));
        return p;
    }
    float sweep = sweep_lookup(t.sphere, 0.0f, u.sphereTableMaxB, b) - sweep_lookup(t.camera, 0.0f, u.cameraMaxB, b);
    R r = R(u.sphereRadius);
    R f = schwarzschild_f(r);
    R E = p.ray.energy;
    R L = p.ray.angularMomentum;
    R phiDot = L / (r * r);
    R rDot = -gsqrt(gmax(E * E - f * L * L / (r * r), R(0)));
    R vDot = (E + rDot) / f;
    p.ray.s = RayState<R>{R(0), r, p.ray.s.phi + R(sweep), vDot, rDot, phiDot};
    return p;
}

// Sky direction of a ray that left the sphere outward (Geodesic.h:166-172).
template <typename R>
__device__ __forceinline__ V3<R> sphere_exit_direction(const PlaneRay<R>& ray, const MarchUniforms& u, const SweepTables& t) {
    float b = (float)(gabs(ray.angularMomentum) / ray.energy);
    float sweep = sweep_lookup(t.sphere, 0.0f, u.sphereTableMaxB, b);
    return asymptotic_direction(ray, ray.s.phi + R(sweep));
}

// Step policy (Geodesic.h:177-181): coarse away from the disk slab.
template <typename R> __device__ __forceinline__ R ray_step_length(R z, R r, const GeodesicSettings& g) {
    R coarse = gmin(gmax(R(g.emptyStepFactor) * r, R(g.stepMin)), R(g.emptyStepMax));
    if (gabs(z) > R(DISK_SLAB_HALF_HEIGHT) + coarse) return coarse;
    return gmin(gmax(R(g.stepFactor) * r, R(g.stepMin)), R(g.stepMax));
}

// Relative drift of E and L from the launch values (Geodesic.h:184-188).
template <typename R> __device__ __forceinline__ R ray_drift(const PlaneRay<R>& ray) {
    R ed = gabs(ray_energy(ray.s) - ray.energy) / gabs(ray.energy);
    R ld = gabs(ray_angular_momentum(ray.s) - ray.angularMomentum) / gmax(gabs(ray.angularMomentum), R(1e-3));
    return gmax(ed, ld);
}

// Procedural starfield, a cube map of cells holding at most one star each
// (Geodesic.h:192-215).
__device__ inline float3 starfield(float3 d, uint32_t seed, const float4* blackbody) {
    float3 a = abs3(d);
    uint32_t face;
    float sx, sy, major;
    if (a.x >= a.y && a.x >= a.z) { face = d.x > 0.0f ? 0u : 1u; sx = d.y; sy = d.z; major = a.x; }
    else if (a.y >= a.z) { face = d.y > 0.0f ? 2u : 3u; sx = d.x; sy = d.z; major = a.y; }
    else { face = d.z > 0.0f ? 4u : 5u; sx = d.x; sy = d.y; major = a.z; }
    sx = sx / major * 0.5f + 0.5f;
    sy = sy / major * 0.5f + 0.5f;
    const float cells = 96.0f;
    float scx = sx * cells, scy = sy * cells;
    uint32_t cx = (uint32_t)fminf(scx, cells - 1.0f), cy = (uint32_t)fminf(scy, cells - 1.0f);
    uint4 h = pcg4d(make_uint4(cx, cy, face, seed));
    if (h.x > 0x30000000u) return make_float3(0.0f, 0.0f, 0.0f);
    float dx = scx - ((float)cx + unit_float(h.y));
    float dy = scy - ((float)cy + unit_float(h.z));
    float falloff = expf(-(dx * dx + dy * dy) * 40.0f);
    float uw = unit_float(h.w);
    float brightness = uw * uw * uw * falloff;
    float temperature = 3000.0f + (12000.0f - 3000.0f) * unit_float(h.w ^ h.y);
    float4 tint = table_lookup4(blackbody, BLACKBODY_TABLE_SIZE, blackbody_coordinate(temperature));
    return make_float3(tint.x * brightness, tint.y * brightness, tint.z * brightness);
}

// Total redshift factor g of light leaving gas moving with `gas` as a
// static observer sees it (Geodesic.h:225-236).
__device__ __forceinline__ float redshift_factor(float f, float3 direction, float3 gas) {
    float magnitude = length3(gas);
    float speed = fminf(magnitude, 8.0f);
    float beta = speed > 0.0f ? GAS_SPEED_CEILING * tanhf(speed / GAS_SPEED_CEILING) : 0.0f;
    float3 velocity = magnitude > 0.0f ? gas * (beta / magnitude) : make_float3(0.0f, 0.0f, 0.0f);
    float gamma = rsqrtf(1.0f - beta * beta);
    return sqrtf(fmaxf(f, 0.0f)) / (gamma * (1.0f + dot3(direction, velocity)));
}

struct Sample {
    float3 emission;
    float density;
    float3 velocity;
};

// Normalised texture coordinates of a position in the volume cube
// (march.metal:15-27; the sampler reads zero outside it).
__device__ __forceinline__ float3 volume_coordinates(float3 p, float half_extent) {
    float inv = 1.0f / (2.0f * half_extent);
    return make_float3((p.x + half_extent) * inv, (p.y + half_extent) * inv, (p.z + half_extent) * inv);
}


}  // namespace gg
