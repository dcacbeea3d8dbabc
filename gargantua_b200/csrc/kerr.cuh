// Null geodesics of Kerr in Boyer-Lindquist coordinates from the separable
// Hamiltonian with E and L as parameters (Kerr.h:1-188,
// KerrGeodesic.swift:9-281). The Carter constant and the null residual are
// the drift gauges. Templated on the real type like geodesic.cuh; the float
// build uses the kernel's clamps (1e-8 on sin^2, 1e-4 on sin), the double
// build the oracle's (1e-12, 1e-9).
#pragma once

#include "geodesic.cuh"

namespace gg {

template <typename R> struct KerrState {
    R r, theta, phi, pr, ptheta;
    R energy, angularMomentum;
};

template <typename R> __device__ __forceinline__ R kerr_sin2_floor() { return R(sizeof(R) == 4 ? 1e-8 : 1e-12); }
template <typename R> __device__ __forceinline__ R kerr_sin_floor() { return R(sizeof(R) == 4 ? 1e-4 : 1e-9); }

template <typename R> __device__ __forceinline__ R kerr_outer_horizon(R a) { return R(1) + gsqrt(gmax(R(1) - a * a, R(0))); }
template <typename R> __device__ __forceinline__ R kerr_delta(R a, R r) { return r * r - R(2) * r + a * a; }

// P and G of the radial and polar potentials (Kerr.h:30-37).
template <typename R> __device__ __forceinline__ void kerr_potentials(R a, const KerrState<R>& s, R sin_t, R* p, R* g) {
    *p = (s.r * s.r + a * a) * s.energy - a * s.angularMomentum;
    R sin2 = gmax(sin_t * sin_t, kerr_sin2_floor<R>());
    *g = s.angularMomentum * s.angularMomentum / sin2 - R(2) * a * s.energy * s.angularMomentum +
         a * a * s.energy * s.energy * sin2;
}

template <typename R> __device__ __forceinline__ R kerr_null_residual(R a, const KerrState<R>& s) {
    R st, ct;
    gsincos(s.theta, &st, &ct);
    R delta = kerr_delta(a, s.r);
    R p, g;
    kerr_potentials(a, s, st, &p, &g);
    return delta * s.pr * s.pr + s.ptheta * s.ptheta - p * p / delta + g;
}

template <typename R> __device__ __forceinline__ R kerr_carter(R a, const KerrState<R>& s) {
    R st, ct;
    gsincos(s.theta, &st, &ct);
    R sin2 = gmax(st * st, kerr_sin2_floor<R>());
    R term = s.angularMomentum * s.angularMomentum / sin2 - a * a * s.energy * s.energy;
    return s.ptheta * s.ptheta + ct * ct * term;
}

// The five evolving components as a compact struct.
template <typename R> struct KerrVec {
    R r, theta, phi, pr, ptheta;
};

// Hamilton's equations including the off-shell Sigma terms (Kerr.h:63-90).
template <typename R> __device__ __forceinline__ KerrVec<R> kerr_derivative(R a, const KerrState<R>& s) {
    R r = s.r;
    R e = s.energy, l = s.angularMomentum;
    R st, ct;
    gsincos(s.theta, &st, &ct);
    R delta = kerr_delta(a, r);
    R sigma = r * r + a * a * ct * ct;
    R dprime = R(2) * r - R(2);
    R sin2 = gmax(st * st, kerr_sin2_floor<R>());
    R p, g;
    kerr_potentials(a, s, st, &p, &g);
    R f = delta * s.pr * s.pr + s.ptheta * s.ptheta - p * p / delta + g;
    R ham = f / (R(2) * sigma);
    R pprime = R(2) * r * e;
    R fr = dprime * s.pr * s.pr - R(2) * p * pprime / delta + p * p * dprime / (delta * delta);
    R fth = R(-2) * l * l * ct / (sin2 * gmax(st, kerr_sin_floor<R>())) + R(2) * a * a * e * e * st * ct;
    R sigr = R(2) * r;
    R sigth = R(-2) * a * a * st * ct;
    KerrVec<R> out;
    out.r = delta * s.pr / sigma;
    out.theta = s.ptheta / sigma;
    out.phi = (a * p / delta + l / sin2 - a * e) / sigma;
    out.pr = -(fr / (R(2) * sigma) - ham * sigr / sigma);
    out.ptheta = -(fth / (R(2) * sigma) - ham * sigth / sigma);
    return out;
}

template <typename R> __device__ __forceinline__ KerrState<R> kerr_offset(const KerrState<R>& s, const KerrVec<R>& k, R f) {
    KerrState<R> o = s;
    o.r = s.r + k.r * f;
    o.theta = s.theta + k.theta * f;
    o.phi = s.phi + k.phi * f;
    o.pr = s.pr + k.pr * f;
    o.ptheta = s.ptheta + k.ptheta * f;
    return o;
}

// RK4 increment (Kerr.h:92-99).
template <typename R> __device__ __forceinline__ KerrVec<R> kerr_increment(R a, const KerrState<R>& s, R h) {
    KerrVec<R> k1 = kerr_derivative(a, s);
    KerrVec<R> k2 = kerr_derivative(a, kerr_offset(s, k1, R(0.5) * h));
    KerrVec<R> k3 = kerr_derivative(a, kerr_offset(s, k2, R(0.5) * h));
    KerrVec<R> k4 = kerr_derivative(a, kerr_offset(s, k3, h));
    R w = h / R(6);
    KerrVec<R> inc;
    inc.r = (k1.r + k2.r * R(2) + (k3.r * R(2) + k4.r)) * w;
    inc.theta = (k1.theta + k2.theta * R(2) + (k3.theta * R(2) + k4.theta)) * w;
    inc.phi = (k1.phi + k2.phi * R(2) + (k3.phi * R(2) + k4.phi)) * w;
    inc.pr = (k1.pr + k2.pr * R(2) + (k3.pr * R(2) + k4.pr)) * w;
    inc.ptheta = (k1.ptheta + k2.ptheta * R(2) + (k3.ptheta * R(2) + k4.ptheta)) * w;
    return inc;
}

template <typename R> __device__ __forceinline__ R kerr_radius_of(R a, V3<R> p) {
    R a2 = a * a;
    R rho2 = dot(p, p);
    R half = R(0.5) * (rho2 - a2);
    return gsqrt(half + gsqrt(half * half + a2 * p.z * p.z));
}

// Launch from a static-observer tetrad (Kerr.h:110-148).
template <typename R> __device__ KerrState<R> kerr_launch(R a, V3<R> origin, V3<R> direction) {
    R r = kerr_radius_of(a, origin);
    R rho = length(origin);
    R theta = gacos(gmin(gmax(origin.z / rho, R(-1)), R(1)));
    R phi = gatan2(origin.y, origin.x);
    V3<R> d = normalize(direction);
    R st, ct, sp, cp;
    gsincos(theta, &st, &ct);
    gsincos(phi, &sp, &cp);
    V3<R> rhat = v3<R>(st * cp, st * sp, ct);
    V3<R> thhat = v3<R>(ct * cp, ct * sp, -st);
    V3<R> phhat = v3<R>(-sp, cp, R(0));
    R nr = dot(d, rhat), nth = dot(d, thhat), nph = dot(d, phhat);
    R delta = kerr_delta(a, r);
    R sigma = r * r + a * a * ct * ct;
    R sin2 = gmax(st * st, kerr_sin2_floor<R>());
    R gtt = -(R(1) - R(2) * r / sigma);
    R gtph = R(-2) * a * r * sin2 / sigma;
    R gphph = (r * r + a * a + R(2) * a * a * r * sin2 / sigma) * sin2;
    R grr = sigma / delta;
    R gthth = sigma;
    R ut = R(1) / gsqrt(-gtt);
    R phinorm = gsqrt(gphph - gtph * gtph / gtt);
    R pt = ut + nph * (-gtph / gtt) / phinorm;
    R pph = nph / phinorm;
    KerrState<R> s;
    s.r = r;
    s.theta = theta;
    s.phi = phi;
    s.energy = -(gtt * pt + gtph * pph);
    s.angularMomentum = gtph * pt + gphph * pph;
    s.pr = grr * (nr / gsqrt(grr));
    s.ptheta = gthth * (nth / gsqrt(gthth));
    return s;
}

template <typename R> __device__ __forceinline__ V3<R> kerr_position(R a, const KerrState<R>& s) {
    R radial = gsqrt(s.r * s.r + a * a);
    R st, ct, sp, cp;
    gsincos(s.theta, &st, &ct);
    gsincos(s.phi, &sp, &cp);
    return v3<R>(radial * st * cp, radial * st * sp, s.r * ct);
}

// Direction of travel against the spherical frame (Kerr.h:158-173).
template <typename R> __device__ V3<R> kerr_direction(R a, const KerrState<R>& s) {
    R st, ct, sp, cp;
    gsincos(s.theta, &st, &ct);
    gsincos(s.phi, &sp, &cp);
    R delta = kerr_delta(a, s.r);
    R sigma = s.r * s.r + a * a * ct * ct;
    R sin2 = gmax(st * st, kerr_sin2_floor<R>());
    R rdot = delta * s.pr / sigma;
    R thdot = s.ptheta / sigma;
    R p, g;
    kerr_potentials(a, s, st, &p, &g);
    R phdot = (a * p / delta + s.angularMomentum / sin2 - a * s.energy) / sigma;
    V3<R> rhat = v3<R>(st * cp, st * sp, ct);
    V3<R> thhat = v3<R>(ct * cp, ct * sp, -st);
    V3<R> phhat = v3<R>(-sp, cp, R(0));
    V3<R> local = rdot * rhat + (s.r * thdot) * thhat + (s.r * st * phdot) * phhat;
    R len = length(local);
    return len > R(0) ? local * (R(1) / len) : rhat;
}

// Step length, proportional to radius, shrinking toward the horizon and the
// polar axis (Kerr.h:177-186).
template <typename R> __device__ __forceinline__ R kerr_step_length(R a, const KerrState<R>& s, const GeodesicSettings& g) {
    R above = s.r - kerr_outer_horizon(a);
    R near = R(0.2) * above;
    R pole = gmin(gmax(gsin(s.theta) / R(0.08), R(0.05)), R(1));
    return gmin(gmax(gmin(R(g.stepFactor) * s.r, near) * pole, R(0.002)), R(g.stepMax));
}

}  // namespace gg
