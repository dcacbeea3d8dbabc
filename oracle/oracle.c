/*
 * TEST INFRASTRUCTURE ONLY: the FP64 oracle, a C restatement of
 * the Swift files under Sources/Oracle. Each function names the Swift lines it follows.
 * Loaded by tests and by the bench's CPU-baseline leg; never by the product.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const double PI = 3.14159265358979323846;

/* Constants.swift values used here. */
#define C_RS 2.0
#define C_ISCO 6.0
#define C_DISK_OUTER 24.0
#define C_FEED_INNER 20.0
#define C_CAPTURE 2.02
#define C_ESCAPE 60.0
#define C_PLUNGE 12.0
#define C_DISPERSION 0.02
#define C_ASPECT 0.05
#define C_TPEAK 8000.0
#define C_FLOOR 0.01
#define C_SLAB 6.0
#define C_CEILING 0.85
#define C_BEAM_FLOOR 40.0
#define C_KERR_MARGIN 0.05
#define C_BCRIT 5.196152422706632

static double dmin(double a, double b) { return a < b ? a : b; }
static double dmax(double a, double b) { return a > b ? a : b; }
static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* ------------------------------------------------------------ Hash.swift */

/* Hash.swift:9-21 */
void o_pcg4d(const uint32_t in[4], uint32_t out[4]) {
    uint32_t v[4];
    for (int i = 0; i < 4; ++i) v[i] = in[i] * 1664525u + 1013904223u;
    v[0] += v[1] * v[3];
    v[1] += v[2] * v[0];
    v[2] += v[0] * v[1];
    v[3] += v[1] * v[2];
    for (int i = 0; i < 4; ++i) v[i] ^= v[i] >> 16;
    v[0] += v[1] * v[3];
    v[1] += v[2] * v[0];
    v[2] += v[0] * v[1];
    v[3] += v[1] * v[2];
    memcpy(out, v, sizeof v);
}

/* Hash.swift:25-29 */
void o_hash_draw(uint64_t seed, uint32_t index, uint32_t event, uint32_t lane, uint32_t out[4]) {
    uint32_t in[4] = {index, event, (uint32_t)seed ^ (lane * 0x9E3779B9u), (uint32_t)(seed >> 32)};
    o_pcg4d(in, out);
}

/* Hash.swift:32-34 */
double o_hash_unit(uint32_t x) { return (double)(x >> 8) / 16777216.0; }

/* Hash.swift:39-43 */
void o_gaussian_pair(double u1, double u2, double* g0, double* g1) {
    double radius = sqrt(-2.0 * log(1.0 - u1));
    double angle = 2.0 * PI * u2;
    *g0 = radius * cos(angle);
    *g1 = radius * sin(angle);
}

/* ------------------------------------------------------- Potential.swift */

static double pot_offset(double r) { return dmax(r - C_RS, 1e-6); } /* :30-32 */

double o_potential_energy(int potential, double r) { /* :34-39 */
    return potential ? -1.0 / pot_offset(r) : -1.0 / r;
}
double o_potential_gradient(int potential, double r) { /* :42-49 */
    if (potential) {
        double d = pot_offset(r);
        return 1.0 / (d * d);
    }
    return 1.0 / (r * r);
}
double o_circular_speed(int potential, double r) { return sqrt(r * o_potential_gradient(potential, r)); } /* :52-54 */
double o_angular_frequency(int potential, double r) { return o_circular_speed(potential, r) / r; }      /* :57-59 */
double o_circular_energy(int potential, double r) {                                                     /* :61-64 */
    double v = o_circular_speed(potential, r);
    return 0.5 * v * v + o_potential_energy(potential, r);
}
double o_circular_angular_momentum(int potential, double r) { return r * o_circular_speed(potential, r); }

/* ------------------------------------------------------- DiskModel.swift */

double o_disk_shape(double r, double floor) { /* :17-21 */
    double x = C_ISCO / r;
    double torque = dmax(1.0 - sqrt(x), floor);
    return pow(x, 0.75) * pow(torque, 0.25);
}
double o_disk_peak_radius(void) { return C_ISCO * 49.0 / 36.0; } /* :11 */
double o_disk_temperature(double r, double peak) {                /* :24-27 */
    return peak * o_disk_shape(r, C_FLOOR) / o_disk_shape(o_disk_peak_radius(), C_FLOOR);
}
double o_mass_flux_fraction(double r) { /* :31-35 */
    if (r <= C_FEED_INNER) return 1.0;
    if (r >= C_DISK_OUTER) return 0.0;
    return (C_DISK_OUTER * C_DISK_OUTER - r * r) / (C_DISK_OUTER * C_DISK_OUTER - C_FEED_INNER * C_FEED_INNER);
}
double o_steady_surface_density(double r) { /* :42-45 */
    if (r <= C_ISCO || r >= C_DISK_OUTER) return 0.0;
    return o_mass_flux_fraction(r) * (r - C_ISCO) / pow(r, 1.5);
}
double o_radial_number_density(double r) { return 2.0 * PI * r * o_steady_surface_density(r); } /* :48-50 */

/* :54-78 */
void o_radial_inverse_cdf(int count, int resolution, double* table) {
    double r0 = C_ISCO, r1 = C_DISK_OUTER;
    double dr = (r1 - r0) / (double)resolution;
    double* cumulative = (double*)calloc((size_t)resolution + 1, sizeof(double));
    double previous = o_radial_number_density(r0);
    for (int i = 1; i <= resolution; ++i) {
        double r = r0 + (double)i * dr;
        double density = o_radial_number_density(r);
        cumulative[i] = cumulative[i - 1] + 0.5 * (previous + density) * dr;
        previous = density;
    }
    double total = cumulative[resolution];
    int i = 0;
    for (int k = 0; k < count; ++k) {
        double target = total * (double)k / (double)(count - 1);
        while (i < resolution && cumulative[i + 1] < target) ++i;
        if (i >= resolution) {
            table[k] = r1;
            continue;
        }
        double span = cumulative[i + 1] - cumulative[i];
        double t = span > 0 ? (target - cumulative[i]) / span : 0.0;
        table[k] = r0 + ((double)i + t) * dr;
    }
    table[count - 1] = r1;
    free(cumulative);
}

/* :83-107 */
void o_disk_spawn(uint32_t index, uint32_t event, uint64_t seed, const double* cdf, int cdf_count, int potential,
                  double st[6]) {
    uint32_t h0[4], h1[4];
    o_hash_draw(seed, index, event, 0, h0);
    o_hash_draw(seed, index, event, 1, h1);
    double u0 = o_hash_unit(h0[0]), u1 = o_hash_unit(h0[1]), u2 = o_hash_unit(h0[2]), u3 = o_hash_unit(h0[3]);
    double u4 = o_hash_unit(h1[0]), u5 = o_hash_unit(h1[1]);
    double r;
    if (event == 0) {
        double position = u0 * (double)(cdf_count - 1);
        int k = (int)position;
        if (k > cdf_count - 2) k = cdf_count - 2;
        r = cdf[k] + (position - (double)k) * (cdf[k + 1] - cdf[k]);
    } else {
        double inner = C_FEED_INNER * C_FEED_INNER;
        double outer2 = C_DISK_OUTER * C_DISK_OUTER;
        r = sqrt(inner + (outer2 - inner) * u0);
    }
    double phi = 2.0 * PI * u1;
    double g0, g1, g2, g3;
    o_gaussian_pair(u2, u3, &g0, &g1);
    o_gaussian_pair(u4, u5, &g2, &g3);
    double vc = o_circular_speed(potential, r);
    st[0] = r * cos(phi);
    st[1] = r * sin(phi);
    st[2] = C_ASPECT * r * g0;
    st[3] = -vc * sin(phi) + C_DISPERSION * vc * g1;
    st[4] = vc * cos(phi) + C_DISPERSION * vc * g2;
    st[5] = 0.0 + C_DISPERSION * vc * g3;
}

/* :110-115 */
void o_circular_orbit(double r, double phi, int potential, double st[6]) {
    double v = o_circular_speed(potential, r);
    st[0] = r * cos(phi);
    st[1] = r * sin(phi);
    st[2] = 0.0;
    st[3] = -v * sin(phi);
    st[4] = v * cos(phi);
    st[5] = 0.0;
}

/* ----------------------------------------------- ParticleDynamics.swift */

/* :31-38: gravity kick, drag, drift */
void o_dynamics_step(int potential, double dt, double alpha, double st[6]) {
    double r = sqrt(dot3(st, st));
    double k = -o_potential_gradient(potential, r) / r;
    double omega = o_angular_frequency(potential, r);
    for (int i = 0; i < 3; ++i) st[3 + i] += st[i] * k * dt;
    double drag = alpha * omega * dt;
    for (int i = 0; i < 3; ++i) st[3 + i] -= st[3 + i] * drag;
    for (int i = 0; i < 3; ++i) st[i] += st[3 + i] * dt;
}

/* :43-52 */
int o_dynamics_removed(const double before[3], const double st[6]) {
    double travel[3] = {st[0] - before[0], st[1] - before[1], st[2] - before[2]};
    double len2 = dmax(dot3(travel, travel), 1e-12);
    double along = dmin(dmax(-dot3(before, travel) / len2, 0.0), 1.0);
    double closest[3] = {before[0] + along * travel[0], before[1] + along * travel[1], before[2] + along * travel[2]};
    double c = sqrt(dot3(closest, closest));
    double radius = sqrt(dot3(st, st));
    double speed = sqrt(dot3(st + 3, st + 3));
    return c < C_CAPTURE || radius > C_ESCAPE || speed > C_PLUNGE;
}

double o_specific_energy(int potential, const double st[6]) { /* :59-61 */
    double v2 = dot3(st + 3, st + 3);
    return 0.5 * v2 + o_potential_energy(potential, sqrt(dot3(st, st)));
}
double o_angular_momentum_z(const double st[6]) { return st[0] * st[4] - st[1] * st[3]; } /* :64-66 */

/* GoldenTests.swift:39-64 */
void o_disk_settle(uint32_t count, uint64_t seed, uint32_t substeps, int potential, double dt, double alpha,
                   double* radii, uint32_t* total_respawns) {
    double cdf[1024];
    o_radial_inverse_cdf(1024, 8192, cdf);
    uint64_t total = 0;
#pragma omp parallel for reduction(+ : total) schedule(static)
    for (int64_t i = 0; i < (int64_t)count; ++i) {
        double st[6];
        uint32_t respawns = 0;
        o_disk_spawn((uint32_t)i, 0, seed, cdf, 1024, potential, st);
        for (uint32_t s = 0; s < substeps; ++s) {
            double before[3] = {st[0], st[1], st[2]};
            o_dynamics_step(potential, dt, alpha, st);
            if (o_dynamics_removed(before, st)) {
                respawns += 1;
                o_disk_spawn((uint32_t)i, respawns, seed, cdf, 1024, potential, st);
            }
        }
        radii[i] = sqrt(st[0] * st[0] + st[1] * st[1]);
        total += respawns;
    }
    *total_respawns = (uint32_t)total;
}

/* --------------------------------------------------------- DiskEdge.swift */

/* :14-43 */
double o_disk_inner_edge(const double* radii, int n, double bin_width, double fit_inner, double fit_outer) {
    int count = (int)llround((fit_outer - fit_inner) / bin_width);
    double* counts = (double*)calloc((size_t)count, sizeof(double));
    for (int i = 0; i < n; ++i) {
        double r = radii[i];
        if (r >= fit_inner && r < fit_outer) {
            int b = (int)((r - fit_inner) / bin_width);
            if (b > count - 1) b = count - 1;
            counts[b] += 1.0;
        }
    }
    double sx = 0, sy = 0, sxx = 0, sxy = 0;
    for (int k = 0; k < count; ++k) {
        double center = fit_inner + ((double)k + 0.5) * bin_width;
        double sigma = counts[k] / (2.0 * PI * center * bin_width);
        double y = sigma * pow(center, 1.5);
        sx += center;
        sy += y;
        sxx += center * center;
        sxy += center * y;
    }
    double nn = (double)count;
    double slope = (nn * sxy - sx * sy) / (nn * sxx - sx * sx);
    double intercept = (sy - slope * sx) / nn;
    free(counts);
    return -intercept / slope;
}

/* --------------------------------------------------- Schwarzschild.swift */

double o_f(double r) { return 1.0 - C_RS / r; } /* :14-16 */

/* :167-172 */
void o_settings_interactive(o_settings* s) {
    s->step_factor = 0.02; s->step_min = 0.02; s->step_max = 0.5;
    s->capture_radius = C_CAPTURE; s->escape_radius = C_ESCAPE;
    s->step_cap = 256; s->empty_step_factor = 0.1; s->empty_step_max = 3.0;
}
void o_settings_still(o_settings* s) {
    o_settings_interactive(s);
    s->step_cap = 4096; s->empty_step_factor = 0.06; s->empty_step_max = 1.5;
}

double o_energy(const double s[6]) { return o_f(s[1]) * s[3] - s[4]; }     /* :106-108 */
double o_angular_momentum(const double s[6]) { return s[1] * s[1] * s[5]; } /* :110-112 */
double o_null_residual(const double s[6]) {                                  /* :115-117 */
    return -o_f(s[1]) * s[3] * s[3] + 2.0 * s[3] * s[4] + s[1] * s[1] * s[5] * s[5];
}

/* :121-127 */
void o_derivative(const double s[6], double out[6]) {
    double r = s[1];
    double vdd = -s[3] * s[3] / (r * r) + r * s[5] * s[5];
    double rdd = 2.0 * s[4] * s[3] / (r * r) + o_f(r) * (r * s[5] * s[5] - s[3] * s[3] / (r * r));
    double pdd = -2.0 * s[4] * s[5] / r;
    out[0] = s[3]; out[1] = s[4]; out[2] = s[5];
    out[3] = vdd; out[4] = rdd; out[5] = pdd;
}

/* :130-136 */
void o_step(const double s[6], double h, double out[6]) {
    double k1[6], k2[6], k3[6], k4[6], t[6];
    o_derivative(s, k1);
    for (int i = 0; i < 6; ++i) t[i] = s[i] + k1[i] * (0.5 * h);
    o_derivative(t, k2);
    for (int i = 0; i < 6; ++i) t[i] = s[i] + k2[i] * (0.5 * h);
    o_derivative(t, k3);
    for (int i = 0; i < 6; ++i) t[i] = s[i] + k3[i] * h;
    o_derivative(t, k4);
    for (int i = 0; i < 6; ++i) out[i] = s[i] + (k1[i] + k2[i] * 2.0 + k3[i] * 2.0 + k4[i]) * (h / 6.0);
}

/* :174-184 */
double o_step_length(const o_settings* st, double r, double z) {
    double coarse = dmin(dmax(st->empty_step_factor * r, st->step_min), st->empty_step_max);
    if (fabs(z) > C_SLAB + coarse) return coarse;
    return dmin(dmax(st->step_factor * r, st->step_min), st->step_max);
}

/* :55-57 */
void o_ray_position(const o_ray* ray, double out[3]) {
    double c = cos(ray->s[2]), sn = sin(ray->s[2]), r = ray->s[1];
    out[0] = r * (c * ray->e1.x + sn * ray->e2.x);
    out[1] = r * (c * ray->e1.y + sn * ray->e2.y);
    out[2] = r * (c * ray->e1.z + sn * ray->e2.z);
}

/* :61-67 */
void o_ray_direction(const o_ray* ray, double out[3]) {
    double c = cos(ray->s[2]), sn = sin(ray->s[2]);
    double radial[3] = {c * ray->e1.x + sn * ray->e2.x, c * ray->e1.y + sn * ray->e2.y, c * ray->e1.z + sn * ray->e2.z};
    double tang[3] = {-sn * ray->e1.x + c * ray->e2.x, -sn * ray->e1.y + c * ray->e2.y, -sn * ray->e1.z + c * ray->e2.z};
    double a = ray->s[4] / sqrt(dmax(o_f(ray->s[1]), 1e-6));
    double b = ray->s[1] * ray->s[5];
    double local[3] = {a * radial[0] + b * tang[0], a * radial[1] + b * tang[1], a * radial[2] + b * tang[2]};
    double len = sqrt(dot3(local, local));
    for (int i = 0; i < 3; ++i) out[i] = len > 0 ? local[i] / len : radial[i];
}

/* :76-97 */
void o_launch(const double origin[3], const double d[3], o_ray* ray) {
    double r0 = sqrt(dot3(origin, origin));
    double e1[3] = {origin[0] / r0, origin[1] / r0, origin[2] / r0};
    double dl = sqrt(dot3(d, d));
    double unit[3] = {d[0] / dl, d[1] / dl, d[2] / dl};
    double dr = dot3(unit, e1);
    double perp[3] = {unit[0] - dr * e1[0], unit[1] - dr * e1[1], unit[2] - dr * e1[2]};
    double dphi = sqrt(dot3(perp, perp));
    if (dphi < 1e-12) {
        double helper[3] = {0, 0, 0};
        if (fabs(e1[0]) < 0.9) helper[0] = 1.0; else helper[1] = 1.0;
        double hd = dot3(helper, e1);
        for (int i = 0; i < 3; ++i) perp[i] = helper[i] - hd * e1[i];
        double pl = sqrt(dot3(perp, perp));
        for (int i = 0; i < 3; ++i) perp[i] /= pl;
        dphi = 0.0;
    } else {
        for (int i = 0; i < 3; ++i) perp[i] /= dphi;
    }
    double f0 = o_f(r0);
    ray->s[0] = 0.0;
    ray->s[1] = r0;
    ray->s[2] = 0.0;
    ray->s[3] = (1.0 + dr) / sqrt(f0);
    ray->s[4] = sqrt(f0) * dr;
    ray->s[5] = dphi / r0;
    ray->e1.x = e1[0]; ray->e1.y = e1[1]; ray->e1.z = e1[2];
    ray->e2.x = perp[0]; ray->e2.y = perp[1]; ray->e2.z = perp[2];
    ray->energy = o_energy(ray->s);
    ray->angular_momentum = o_angular_momentum(ray->s);
}

/* :100-104 */
void o_launch_b(double radius, double b, o_ray* ray) {
    double dphi = b * sqrt(o_f(radius)) / radius;
    double dr = -sqrt(dmax(0.0, 1.0 - dphi * dphi));
    double origin[3] = {radius, 0.0, 0.0};
    double dir[3] = {dr, dphi, 0.0};
    o_launch(origin, dir, ray);
}

/* :200-220 */
int o_integrate(o_ray* ray, const o_settings* st, int64_t* steps_out, double* drift_out) {
    int64_t steps = 0;
    double drift = 0.0;
    double e0 = ray->energy, l0 = ray->angular_momentum;
    double lscale = dmax(fabs(l0), 1e-3);
    int outcome = O_EXHAUSTED;
    while (steps < st->step_cap) {
        double pos[3];
        o_ray_position(ray, pos);
        double h = o_step_length(st, ray->s[1], pos[2]);
        double next[6];
        o_step(ray->s, h, next);
        memcpy(ray->s, next, sizeof next);
        steps += 1;
        double ed = fabs(o_energy(ray->s) - e0) / fabs(e0);
        double ld = fabs(o_angular_momentum(ray->s) - l0) / lscale;
        drift = dmax(drift, dmax(ed, ld));
        if (ray->s[1] <= st->capture_radius) { outcome = O_CAPTURED; break; }
        if (ray->s[1] >= st->escape_radius) { outcome = O_ESCAPED; break; }
    }
    *steps_out = steps;
    *drift_out = drift;
    return outcome;
}

/* :230-240 */
double o_redshift_factor(double r, const double direction[3], const double gas[3]) {
    double magnitude = sqrt(dot3(gas, gas));
    double speed = dmin(magnitude, 8.0);
    double beta = speed > 0 ? C_CEILING * tanh(speed / C_CEILING) : 0.0;
    double vel[3] = {0, 0, 0};
    if (magnitude > 0) for (int i = 0; i < 3; ++i) vel[i] = gas[i] * (beta / magnitude);
    double gamma = 1.0 / sqrt(1.0 - beta * beta);
    return sqrt(dmax(o_f(r), 0.0)) / (gamma * (1.0 + dot3(direction, vel)));
}

/* :244-252 */
double o_deflection(const o_ray* launch, const o_ray* result) {
    double d0[3], d1[3];
    o_ray_direction(launch, d0);
    o_ray_direction(result, d1);
    double e1a[3] = {launch->e1.x, launch->e1.y, launch->e1.z}, e2a[3] = {launch->e2.x, launch->e2.y, launch->e2.z};
    double e1b[3] = {result->e1.x, result->e1.y, result->e1.z}, e2b[3] = {result->e2.x, result->e2.y, result->e2.z};
    double ax = dot3(d0, e1a), ay = dot3(d0, e2a);
    double bx = dot3(d1, e1b), by = dot3(d1, e2b);
    return atan2(ax * by - ay * bx, ax * bx + ay * by);
}

/* :256-269 */
double o_critical_impact_parameter(double launch_radius, const o_settings* st, int iterations) {
    double low = 3.0, high = 8.0;
    for (int i = 0; i < iterations; ++i) {
        double mid = 0.5 * (low + high);
        o_ray ray;
        o_launch_b(launch_radius, mid, &ray);
        int64_t steps;
        double drift;
        int outcome = o_integrate(&ray, st, &steps, &drift);
        if (outcome == O_CAPTURED) low = mid;
        else if (outcome == O_ESCAPED) high = mid;
        else return mid;
    }
    return 0.5 * (low + high);
}

void o_integrate_batch(const double* probes, int n, const o_settings* st, double* results, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; ++i) {
        o_ray ray;
        o_launch(probes + 6 * i, probes + 6 * i + 3, &ray);
        int64_t steps;
        double drift;
        int outcome = o_integrate(&ray, st, &steps, &drift);
        double* out = results + 11 * i;
        o_ray_position(&ray, out);
        o_ray_direction(&ray, out + 3);
        out[6] = drift;
        out[7] = outcome;
        out[8] = (double)steps;
        out[9] = ray.energy;
        out[10] = ray.angular_momentum;
    }
}

/* ------------------------------------------------------------ bake.metal */

/* bakeRays (bake.metal:46-91) in FP64 for rays launched at the camera (no
 * sphere jump): integrate with the oracle's step and step policy; after each
 * step, a point inside the disk slab (|z| < 6, |x|, |y| < half_extent) at
 * least `spacing` of path since the last stored one is stored (position and
 * that path), up to `capacity` points (a ray with more is `overflowed`).
 * Per ray: samples[capacity][4], count, overflowed, falls_in (captured, or
 * exhausted inbound inside the critical impact parameter), final direction
 * and depth (path to the first stored point, else the whole path, over
 * 2 R_ESCAPE, at most 1). */
void o_bake_batch(const double* probes, int n, const o_settings* st, double spacing, double half_extent, int capacity,
                  double* samples, int* counts, int* overflowed, int* falls_in, double* direction_depth, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; ++i) {
        o_ray ray;
        o_launch(probes + 6 * i, probes + 6 * i + 3, &ray);
        double* slot = samples + (int64_t)i * capacity * 4;
        double previous[3];
        o_ray_position(&ray, previous);
        double since = 0.0, travelled = 0.0, first_depth = -1.0;
        int count = 0, over = 0, outcome = O_EXHAUSTED;
        for (int64_t k = 0; k < st->step_cap; ++k) {
            double h = o_step_length(st, ray.s[1], previous[2]);
            double next[6];
            o_step(ray.s, h, next);
            memcpy(ray.s, next, sizeof next);
            double pos[3];
            o_ray_position(&ray, pos);
            double d[3] = {pos[0] - previous[0], pos[1] - previous[1], pos[2] - previous[2]};
            double path = sqrt(dot3(d, d));
            since += path;
            travelled += path;
            memcpy(previous, pos, sizeof pos);
            if (ray.s[1] <= st->capture_radius) { outcome = O_CAPTURED; break; }
            if (fabs(pos[2]) < C_SLAB && fabs(pos[0]) < half_extent && fabs(pos[1]) < half_extent && since >= spacing) {
                if (count < capacity) {
                    slot[4 * count + 0] = pos[0];
                    slot[4 * count + 1] = pos[1];
                    slot[4 * count + 2] = pos[2];
                    slot[4 * count + 3] = since;
                    count += 1;
                    if (first_depth < 0.0) first_depth = travelled;
                } else {
                    over = 1;
                }
                since = 0.0;
            }
            if (ray.s[1] >= st->escape_radius) { outcome = O_ESCAPED; break; }
        }
        counts[i] = count;
        overflowed[i] = over;
        falls_in[i] = outcome == O_CAPTURED ||
                      (outcome == O_EXHAUSTED && ray.s[4] < 0.0 && fabs(ray.angular_momentum) < C_BCRIT * ray.energy);
        o_ray_direction(&ray, direction_depth + 4 * i);
        double depth = first_depth >= 0.0 ? first_depth : travelled;
        direction_depth[4 * i + 3] = dmin(depth / (2.0 * C_ESCAPE), 1.0);
    }
}

/* ---------------------------------------------------- KerrGeodesic.swift */

double o_kerr_outer_horizon(double a) { return 1.0 + sqrt(1.0 - a * a); } /* :17 */
static double kdelta(double a, double r) { return r * r - 2.0 * r + a * a; }
static double ksigma(double a, double r, double th) {
    double c = cos(th);
    return r * r + a * a * c * c;
}

/* :52-59 */
static void kpotentials(double a, const double s[7], double* p, double* g) {
    double e = s[5], l = s[6];
    *p = (s[0] * s[0] + a * a) * e - a * l;
    double sn = sin(s[1]);
    double sin2 = dmax(sn * sn, 1e-12);
    *g = l * l / sin2 - 2.0 * a * e * l + a * a * e * e * sin2;
}

double o_kerr_null_residual(double a, const double s[7]) { /* :62-66 */
    double delta = kdelta(a, s[0]);
    double p, g;
    kpotentials(a, s, &p, &g);
    return delta * s[3] * s[3] + s[4] * s[4] - p * p / delta + g;
}

double o_kerr_carter(double a, const double s[7]) { /* :69-74 */
    double c = cos(s[1]);
    double sn = sin(s[1]);
    double sin2 = dmax(sn * sn, 1e-12);
    double term = s[6] * s[6] / sin2 - a * a * s[5] * s[5];
    return s[4] * s[4] + c * c * term;
}

/* :77-105 */
void o_kerr_derivative(double a, const double s[7], double out[7]) {
    double e = s[5], l = s[6];
    double r = s[0], th = s[1];
    double delta = kdelta(a, r);
    double sigma = ksigma(a, r, th);
    double dprime = 2.0 * r - 2.0;
    double st = sin(th), ct = cos(th);
    double sin2 = dmax(st * st, 1e-12);
    double p, g;
    kpotentials(a, s, &p, &g);
    double f = delta * s[3] * s[3] + s[4] * s[4] - p * p / delta + g;
    double ham = f / (2.0 * sigma);
    double pprime = 2.0 * r * e;
    double fr = dprime * s[3] * s[3] - 2.0 * p * pprime / delta + p * p * dprime / (delta * delta);
    double fth = -2.0 * l * l * ct / (sin2 * dmax(st, 1e-9)) + 2.0 * a * a * e * e * st * ct;
    double sigr = 2.0 * r;
    double sigth = -2.0 * a * a * st * ct;
    out[0] = delta * s[3] / sigma;
    out[1] = s[4] / sigma;
    out[2] = (a * p / delta + l / sin2 - a * e) / sigma;
    out[3] = -(fr / (2.0 * sigma) - ham * sigr / sigma);
    out[4] = -(fth / (2.0 * sigma) - ham * sigth / sigma);
    out[5] = e;
    out[6] = l;
}

/* :107-113 (E and L ride along unchanged) */
void o_kerr_step(double a, const double s[7], double h, double out[7]) {
    double k1[7], k2[7], k3[7], k4[7], t[7];
    o_kerr_derivative(a, s, k1);
    memcpy(t, s, sizeof t);
    for (int i = 0; i < 5; ++i) t[i] = s[i] + k1[i] * (0.5 * h);
    o_kerr_derivative(a, t, k2);
    for (int i = 0; i < 5; ++i) t[i] = s[i] + k2[i] * (0.5 * h);
    o_kerr_derivative(a, t, k3);
    for (int i = 0; i < 5; ++i) t[i] = s[i] + k3[i] * h;
    o_kerr_derivative(a, t, k4);
    memcpy(out, s, 7 * sizeof(double));
    for (int i = 0; i < 5; ++i) out[i] = s[i] + (k1[i] + k2[i] * 2.0 + k3[i] * 2.0 + k4[i]) * (h / 6.0);
}

double o_kerr_radius(double a, const double p[3]) { /* :116-121 */
    double a2 = a * a;
    double rho2 = dot3(p, p);
    double half = 0.5 * (rho2 - a2);
    return sqrt(half + sqrt(half * half + a2 * p[2] * p[2]));
}

/* :128-168 */
void o_kerr_launch(double a, const double origin[3], const double direction[3], double s[7]) {
    double r = o_kerr_radius(a, origin);
    double rho = sqrt(dot3(origin, origin));
    double th = acos(dmin(dmax(origin[2] / rho, -1.0), 1.0));
    double ph = atan2(origin[1], origin[0]);
    double dl = sqrt(dot3(direction, direction));
    double d[3] = {direction[0] / dl, direction[1] / dl, direction[2] / dl};
    double st = sin(th), ct = cos(th);
    double rhat[3] = {st * cos(ph), st * sin(ph), ct};
    double thhat[3] = {ct * cos(ph), ct * sin(ph), -st};
    double phhat[3] = {-sin(ph), cos(ph), 0.0};
    double nr = dot3(d, rhat), nth = dot3(d, thhat), nph = dot3(d, phhat);
    double delta = kdelta(a, r);
    double sigma = ksigma(a, r, th);
    double sin2 = dmax(st * st, 1e-12);
    double gtt = -(1.0 - 2.0 * r / sigma);
    double gtph = -2.0 * a * r * sin2 / sigma;
    double gphph = (r * r + a * a + 2.0 * a * a * r * sin2 / sigma) * sin2;
    double grr = sigma / delta;
    double gthth = sigma;
    double ut = 1.0 / sqrt(-gtt);
    double phinorm = sqrt(gphph - gtph * gtph / gtt);
    double pt = ut + nph * (-gtph / gtt) / phinorm;
    double pph = nph / phinorm;
    double prup = nr / sqrt(grr);
    double pthup = nth / sqrt(gthth);
    s[0] = r;
    s[1] = th;
    s[2] = ph;
    s[5] = -(gtt * pt + gtph * pph);
    s[6] = gtph * pt + gphph * pph;
    s[3] = grr * prup;
    s[4] = gthth * pthup;
}

void o_kerr_position(double a, const double s[7], double out[3]) { /* :170-174 */
    double radial = sqrt(s[0] * s[0] + a * a);
    double st = sin(s[1]);
    out[0] = radial * st * cos(s[2]);
    out[1] = radial * st * sin(s[2]);
    out[2] = s[0] * cos(s[1]);
}

/* The kernel's direction convention (Kerr.h:158-173) in FP64; the Swift
 * oracle has no direction function, the probe results report this one. */
void o_kerr_direction(double a, const double s[7], double out[3]) {
    double delta = kdelta(a, s[0]);
    double sigma = ksigma(a, s[0], s[1]);
    double sn = sin(s[1]);
    double sin2 = dmax(sn * sn, 1e-12);
    double rdot = delta * s[3] / sigma;
    double thdot = s[4] / sigma;
    double p, g;
    kpotentials(a, s, &p, &g);
    double phdot = (a * p / delta + s[6] / sin2 - a * s[5]) / sigma;
    double st = sin(s[1]), ct = cos(s[1]);
    double rhat[3] = {st * cos(s[2]), st * sin(s[2]), ct};
    double thhat[3] = {ct * cos(s[2]), ct * sin(s[2]), -st};
    double phhat[3] = {-sin(s[2]), cos(s[2]), 0.0};
    double local[3];
    for (int i = 0; i < 3; ++i) local[i] = rdot * rhat[i] + s[0] * thdot * thhat[i] + s[0] * st * phdot * phhat[i];
    double len = sqrt(dot3(local, local));
    for (int i = 0; i < 3; ++i) out[i] = len > 0 ? local[i] / len : rhat[i];
}

/* :184-197 */
void o_kerr_settings_default(o_kerr_settings* s, int64_t step_cap) {
    s->step_factor = 0.02;
    s->step_min = 0.005;
    s->step_max = 0.5;
    s->capture_margin = C_KERR_MARGIN;
    s->escape_radius = C_ESCAPE;
    s->step_cap = step_cap;
}

/* :214-221 */
double o_kerr_step_length(double a, const double s[7], const o_kerr_settings* st) {
    double above = s[0] - o_kerr_outer_horizon(a);
    double near = 0.2 * above;
    double pole = dmin(dmax(sin(s[1]) / 0.08, 0.05), 1.0);
    return dmin(dmax(dmin(st->step_factor * s[0], near) * pole, 0.4 * st->step_min), st->step_max);
}

/* :223-244 */
int o_kerr_integrate(double a, double s[7], const o_kerr_settings* st, int64_t* steps_out, double* drift_out) {
    double carter0 = o_kerr_carter(a, s);
    double scale = dmax(fabs(carter0), s[5] * s[5]);
    double drift = 0.0;
    int64_t steps = 0;
    double capture = o_kerr_outer_horizon(a) + st->capture_margin;
    int outcome = O_EXHAUSTED;
    while (steps < st->step_cap) {
        double next[7];
        o_kerr_step(a, s, o_kerr_step_length(a, s, st), next);
        memcpy(s, next, sizeof next);
        steps += 1;
        double cd = fabs(o_kerr_carter(a, s) - carter0) / scale;
        double nd = fabs(o_kerr_null_residual(a, s)) / (scale * dmax(s[0] * s[0], 1.0));
        drift = dmax(drift, dmax(cd, nd));
        if (s[0] <= capture) { outcome = O_CAPTURED; break; }
        if (s[0] >= st->escape_radius) { outcome = O_ESCAPED; break; }
    }
    *steps_out = steps;
    *drift_out = drift;
    return outcome;
}

/* :249-262 */
double o_kerr_bisect_critical_xi(double a, double radius, double side, const o_kerr_settings* st, int iterations) {
    double low = 0.0, high = 12.0 / radius;
    double origin[3] = {radius, 0.0, 0.0};
    for (int i = 0; i < iterations; ++i) {
        double aim = 0.5 * (low + high);
        double dir[3] = {-1.0, side * aim, 0.0};
        double s[7];
        o_kerr_launch(a, origin, dir, s);
        int64_t steps;
        double drift;
        if (o_kerr_integrate(a, s, st, &steps, &drift) == O_CAPTURED) low = aim; else high = aim;
    }
    double dir[3] = {-1.0, side * 0.5 * (low + high), 0.0};
    double s[7];
    o_kerr_launch(a, origin, dir, s);
    return s[6] / s[5];
}

double o_kerr_critical_xi(double a, double rc) { /* :267-269 */
    return (rc * rc * (3.0 - rc) - a * a * (rc + 1.0)) / (a * (rc - 1.0));
}
double o_kerr_critical_eta(double a, double rc) { /* :271-273 */
    return rc * rc * rc * (4.0 * a * a - rc * (rc - 3.0) * (rc - 3.0)) / (a * a * (rc - 1.0) * (rc - 1.0));
}
void o_kerr_photon_orbits(double a, double* pro, double* retro) { /* :277-281 */
    *pro = 2.0 * (1.0 + cos(2.0 / 3.0 * acos(-a)));
    *retro = 2.0 * (1.0 + cos(2.0 / 3.0 * acos(a)));
}

void o_kerr_integrate_batch(double a, const double* probes, int n, const o_kerr_settings* st, double* results,
                            int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; ++i) {
        double s[7];
        o_kerr_launch(a, probes + 6 * i, probes + 6 * i + 3, s);
        int64_t steps;
        double drift;
        int outcome = o_kerr_integrate(a, s, st, &steps, &drift);
        double* out = results + 11 * i;
        o_kerr_position(a, s, out);
        o_kerr_direction(a, s, out + 3);
        out[6] = drift;
        out[7] = outcome;
        out[8] = (double)steps;
        out[9] = s[5];
        out[10] = s[6];
    }
}

/* ------------------------------------------------------ Deflection.swift */

double o_max_impact_parameter(double r) { return r / sqrt(1.0 - C_RS / r); } /* :20-22 */

/* :29-45: midpoint rule after u = uMax sin^2(theta) */
double o_sweep(double r, double b, int intervals) {
    if (!(b > 0.0)) return 0.0;
    double bound = dmin(b, o_max_impact_parameter(r));
    double umax = 1.0 / r;
    double h = (PI / 2.0) / (double)intervals;
    double sum = 0.0;
    for (int k = 0; k < intervals; ++k) {
        double th = ((double)k + 0.5) * h;
        double sn = sin(th), c = cos(th);
        double u = umax * sn * sn;
        double inner = 1.0 - bound * bound * u * u * (1.0 - 2.0 * u);
        if (inner > 0.0) sum += bound * 2.0 * umax * sn * c / sqrt(inner);
    }
    return sum * h;
}

double o_table_impact_parameter(double low, double high, double t) { /* :51-54 */
    double back = 1.0 - t;
    return low + (high - low) * (1.0 - back * back);
}
double o_table_coordinate(double low, double high, double b) { /* :57-60 */
    double x = dmin(dmax((b - low) / (high - low), 0.0), 1.0);
    return 1.0 - sqrt(1.0 - x);
}

/* :65-75 */
double o_periapsis(double b) {
    double u = 1.0 / b;
    for (int i = 0; i < 60; ++i) {
        double value = 1.0 - b * b * u * u * (1.0 - 2.0 * u);
        double slope = -b * b * (2.0 * u - 6.0 * u * u);
        double next = u - value / slope;
        if (fabs(next - u) < 1e-15) { u = next; break; }
        u = next;
    }
    return 1.0 / u;
}

double o_turning_sweep(double r, double b, int intervals) { /* :83-86 */
    double peri = o_periapsis(b);
    return 2.0 * (o_sweep(peri, b, intervals) - o_sweep(r, b, intervals));
}
double o_escape_sweep(double r, double b, int intervals) { /* :90-92 */
    return o_turning_sweep(r, b, intervals) + o_sweep(r, b, intervals);
}

void o_sweep_table(double r, int count, int intervals, double* out) { /* :95-98 */
    double bmax = o_max_impact_parameter(r);
    for (int k = 0; k < count; ++k)
        out[k] = o_sweep(r, o_table_impact_parameter(0.0, bmax, (double)k / (double)(count - 1)), intervals);
}

void o_sky_table(double camera_radius, double sphere_radius, int count, int intervals, double* out) { /* :102-106 */
    double low = o_max_impact_parameter(sphere_radius);
    double high = o_max_impact_parameter(camera_radius);
    for (int k = 0; k < count; ++k)
        out[k] = o_escape_sweep(camera_radius, o_table_impact_parameter(low, high, (double)k / (double)(count - 1)),
                                intervals);
}

/* ------------------------------------------------------- Blackbody.swift */

static const double BB_C2 = 1.438776877e-2; /* :16 */

static double planck(double nm, double t) { /* :19-23 */
    double lambda = nm * 1e-9;
    double exponent = BB_C2 / (lambda * t);
    return 1.0 / (pow(lambda, 5.0) * (exp(exponent) - 1.0));
}
static double lobe(double x, double mu, double s1, double s2) { /* :26-30 */
    double sigma = x < mu ? s1 : s2;
    double t = (x - mu) / sigma;
    return exp(-0.5 * t * t);
}
static void matching(double x, double out[3]) { /* :36-41 */
    out[0] = 1.056 * lobe(x, 599.8, 37.9, 31.0) + 0.362 * lobe(x, 442.0, 16.0, 26.7) - 0.065 * lobe(x, 501.1, 20.4, 26.2);
    out[1] = 0.821 * lobe(x, 568.8, 46.9, 40.5) + 0.286 * lobe(x, 530.9, 16.3, 31.1);
    out[2] = 1.217 * lobe(x, 437.0, 11.8, 36.0) + 0.681 * lobe(x, 459.0, 26.0, 13.4);
}
static void bb_xyz(double t, double out[3]) { /* :44-52 */
    out[0] = out[1] = out[2] = 0.0;
    double w = 380.0;
    while (w <= 780.0) {
        double m[3];
        matching(w, m);
        double p = planck(w, t);
        for (int i = 0; i < 3; ++i) out[i] += m[i] * p;
        w += 1.0;
    }
}
void o_blackbody_chromaticity(double t, double* x, double* y) { /* :54-58 */
    double c[3];
    bb_xyz(t, c);
    double total = c[0] + c[1] + c[2];
    *x = c[0] / total;
    *y = c[1] / total;
}
void o_blackbody_color(double t, double rgb[3]) { /* :63-77 */
    double c[3];
    bb_xyz(t, c);
    double r = 3.2406 * c[0] - 1.5372 * c[1] - 0.4986 * c[2];
    double g = -0.9689 * c[0] + 1.8758 * c[1] + 0.0415 * c[2];
    double b = 0.0557 * c[0] - 0.2040 * c[1] + 1.0570 * c[2];
    r = dmax(r, 0.0); g = dmax(g, 0.0); b = dmax(b, 0.0);
    double peak = dmax(r, dmax(g, b));
    if (peak > 0.0) { rgb[0] = r / peak; rgb[1] = g / peak; rgb[2] = b / peak; }
    else { rgb[0] = rgb[1] = rgb[2] = 1.0; }
}
void o_blackbody_table(int count, double tmin, double tmax, double* rgb) { /* :80-86 */
    for (int k = 0; k < count; ++k) {
        double t = (double)k / (double)(count - 1);
        double temperature = exp(log(tmin) + t * (log(tmax) - log(tmin)));
        o_blackbody_color(temperature, rgb + 3 * k);
    }
}
double o_blackbody_coordinate(double t, double tmin, double tmax) { /* :88-90 */
    double c = dmin(dmax(t, tmin), tmax);
    return (log(c) - log(tmin)) / (log(tmax) - log(tmin));
}

/* ----------------------------------------------------- VolumeField.swift */

/* :40-63 */
void o_volume_sample(int size, double half, const double* em, const double* vel, const double p[3], double e4[4],
                     double v3[3]) {
    double t[3], base[3], frac[3];
    for (int i = 0; i < 3; ++i) {
        double unit = (p[i] + half) / (2.0 * half);
        t[i] = unit * (double)size - 0.5;
        base[i] = floor(t[i]);
        frac[i] = t[i] - base[i];
    }
    int x0 = (int)base[0], y0 = (int)base[1], z0 = (int)base[2];
    for (int i = 0; i < 4; ++i) e4[i] = 0.0;
    for (int i = 0; i < 3; ++i) v3[i] = 0.0;
    for (int dz = 0; dz <= 1; ++dz) {
        double wz = dz == 0 ? 1.0 - frac[2] : frac[2];
        for (int dy = 0; dy <= 1; ++dy) {
            double wy = dy == 0 ? 1.0 - frac[1] : frac[1];
            for (int dx = 0; dx <= 1; ++dx) {
                double wx = dx == 0 ? 1.0 - frac[0] : frac[0];
                double w = wx * wy * wz;
                if (w == 0.0) continue;
                int x = x0 + dx, y = y0 + dy, z = z0 + dz;
                if (x < 0 || y < 0 || z < 0 || x >= size || y >= size || z >= size) continue;
                int64_t idx = ((int64_t)z * size + y) * size + x;
                for (int i = 0; i < 4; ++i) e4[i] += em[4 * idx + i] * w;
                for (int i = 0; i < 3; ++i) v3[i] += vel[3 * idx + i] * w;
            }
        }
    }
}

/* ---------------------------------------------------- LensedRender.swift */

/* :46-79 */
static void lensed_trace(const double origin[3], const double dir[3], int size, double half, const double* em,
                         const double* vel, const o_settings* st, double opacity, double slab, int redshift,
                         double out[3]) {
    o_ray ray;
    o_launch(origin, dir, &ray);
    double color[3] = {0, 0, 0};
    double transmittance = 1.0;
    double previous[3];
    o_ray_position(&ray, previous);
    for (int64_t k = 0; k < st->step_cap; ++k) {
        double next[6];
        o_step(ray.s, o_step_length(st, ray.s[1], previous[2]), next);
        memcpy(ray.s, next, sizeof next);
        double pos[3];
        o_ray_position(&ray, pos);
        if (ray.s[1] <= st->capture_radius) break;
        if (fabs(pos[2]) < slab && fabs(pos[0]) < half && fabs(pos[1]) < half && transmittance > 0.004) {
            double e4[4], v3[3];
            o_volume_sample(size, half, em, vel, pos, e4, v3);
            if (e4[3] > 0.0) {
                double dpos[3] = {pos[0] - previous[0], pos[1] - previous[1], pos[2] - previous[2]};
                double path = sqrt(dot3(dpos, dpos));
                double g3 = 1.0;
                if (redshift) {
                    double d[3];
                    o_ray_direction(&ray, d);
                    double g = o_redshift_factor(ray.s[1], d, v3);
                    double gravity = sqrt(dmax(o_f(ray.s[1]), 0.0));
                    double bulk = dmin(e4[3] / C_BEAM_FLOOR, 1.0);
                    g3 = gravity * gravity * gravity * (1.0 - bulk) + g * g * g * bulk;
                }
                double alpha = 1.0 - exp(-opacity * e4[3] * path);
                for (int i = 0; i < 3; ++i) color[i] += transmittance * e4[i] * g3 * path;
                transmittance *= 1.0 - alpha;
            }
        }
        memcpy(previous, pos, sizeof pos);
        if (ray.s[1] >= st->escape_radius) break;
    }
    memcpy(out, color, sizeof color);
}

/* :84-93 and Camera.direction :23-28 */
void o_lensed_image(int width, int height, const double* cam, int size, double half, const double* em,
                    const double* vel, const o_settings* st, double opacity, double slab, int redshift,
                    double* out_rgb, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            double sx = (2.0 * ((double)x + 0.5) / (double)width - 1.0) * cam[12];
            double sy = (1.0 - 2.0 * ((double)y + 0.5) / (double)height) * cam[13];
            double d[3];
            for (int i = 0; i < 3; ++i) d[i] = cam[9 + i] + sx * cam[3 + i] + sy * cam[6 + i];
            double l = sqrt(dot3(d, d));
            for (int i = 0; i < 3; ++i) d[i] /= l;
            lensed_trace(cam, d, size, half, em, vel, st, opacity, slab, redshift, out_rgb + 3 * ((int64_t)y * width + x));
        }
    }
}

double o_luminance(const double rgb[3]) { return 0.2126 * rgb[0] + 0.7152 * rgb[1] + 0.0722 * rgb[2]; } /* :97-99 */

double o_side_ratio(const double* lum, int width, int height) { /* :103-112 */
    double left = 0.0, right = 0.0;
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            if (x < width / 2) left += lum[y * width + x]; else right += lum[y * width + x];
        }
    double hi = dmax(left, right), lo = dmin(left, right);
    return lo > 0.0 ? hi / lo : INFINITY;
}

/* ------------------------------------------------------ present.metal */

/* present.metal:22-35, in FP64 */
void o_pbr_neutral(const double in[3], double out[3]) {
    const double start = 0.8 - 0.04;
    const double desat = 0.15;
    double c[3] = {in[0], in[1], in[2]};
    double x = dmin(c[0], dmin(c[1], c[2]));
    double offset = x < 0.08 ? x - 6.25 * x * x : 0.04;
    for (int i = 0; i < 3; ++i) c[i] -= offset;
    double peak = dmax(c[0], dmax(c[1], c[2]));
    if (peak < start) { memcpy(out, c, sizeof c); return; }
    double d = 1.0 - start;
    double np = 1.0 - d * d / (peak + d - start);
    for (int i = 0; i < 3; ++i) c[i] *= np / peak;
    double g = 1.0 - 1.0 / (desat * (peak - np) + 1.0);
    for (int i = 0; i < 3; ++i) out[i] = c[i] + (np - c[i]) * g;
}
