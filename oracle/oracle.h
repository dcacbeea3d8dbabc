/*
 * TEST INFRASTRUCTURE ONLY. This is the oracle: a CPU restatement of
 * gargantua's FP64 oracle (the Swift files under Sources/Oracle) plus FP32 replicas of the
 * particle and deposit kernels. Only tests, the smoke check and the bench's
 * CPU-baseline leg may load it, and only as the checker or the timed CPU
 * baseline; the product never links or calls it.
 *
 * Parity anchors (the reference ships no bit-level vectors for this path):
 * the oracle is pinned by the reference's own known-answer tests, restated
 * in tests/test_oracle.py (b_c = 3 sqrt 3, 4/b deflection, Bardeen's shadow
 * edges, Carter drift, sweep tables vs RK4, the ISCO edge of a settled disk)
 * and by the 11 goldens (the JSON files under goldens, copied to tests/golden/goldens).
 *
 * Built with -ffp-contract=off so float replicas give the same bits as the
 * kernels built with --fmad=false.
 */
#ifndef GG_ORACLE_H
#define GG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double x, y, z; } o_vec3;

/* Hash.swift:9-43 */
void o_pcg4d(const uint32_t in[4], uint32_t out[4]);
void o_hash_draw(uint64_t seed, uint32_t index, uint32_t event, uint32_t lane, uint32_t out[4]);
double o_hash_unit(uint32_t x);
void o_gaussian_pair(double u1, double u2, double* g0, double* g1);

/* Potential.swift:16-60; potential 0 Newtonian, 1 Paczynski-Wiita */
double o_potential_energy(int potential, double r);
double o_potential_gradient(int potential, double r);
double o_circular_speed(int potential, double r);
double o_angular_frequency(int potential, double r);
double o_circular_energy(int potential, double r);
double o_circular_angular_momentum(int potential, double r);

/* DiskModel.swift:17-107 */
double o_disk_shape(double r, double floor);
double o_disk_temperature(double r, double peak);
double o_disk_peak_radius(void);
double o_mass_flux_fraction(double r);
double o_steady_surface_density(double r);
double o_radial_number_density(double r);
void o_radial_inverse_cdf(int count, int resolution, double* table);
/* state: x y z vx vy vz */
void o_disk_spawn(uint32_t index, uint32_t event, uint64_t seed, const double* inverse_cdf, int cdf_count,
                  int potential, double state[6]);
void o_circular_orbit(double r, double phi, int potential, double state[6]);

/* ParticleDynamics.swift:31-67 */
void o_dynamics_step(int potential, double dt, double alpha, double state[6]);
int o_dynamics_removed(const double before[3], const double state[6]);
double o_specific_energy(int potential, const double state[6]);
double o_angular_momentum_z(const double state[6]);
/* The oracle disk of GoldenTests.swift:39-64: spawn `count` particles, step
 * `substeps` substeps with respawn; returns cylindrical radii. */
void o_disk_settle(uint32_t count, uint64_t seed, uint32_t substeps, int potential, double dt, double alpha,
                   double* cylindrical_radii, uint32_t* total_respawns);

/* DiskEdge.swift:14-43 */
double o_disk_inner_edge(const double* radii, int n, double bin_width, double fit_inner, double fit_outer);

/* Schwarzschild.swift:11-270. state: v r phi vDot rDot phiDot */
typedef struct {
    double s[6];
    o_vec3 e1, e2;
    double energy, angular_momentum;
} o_ray;

typedef struct {
    double step_factor, step_min, step_max, capture_radius, escape_radius;
    int64_t step_cap;
    double empty_step_factor, empty_step_max;
} o_settings;

enum { O_CAPTURED = 0, O_ESCAPED = 1, O_EXHAUSTED = 2 };

void o_settings_interactive(o_settings* s);
void o_settings_still(o_settings* s);
double o_f(double r);
void o_launch(const double origin[3], const double direction[3], o_ray* ray);
void o_launch_b(double radius, double b, o_ray* ray);
double o_energy(const double s[6]);
double o_angular_momentum(const double s[6]);
double o_null_residual(const double s[6]);
void o_derivative(const double s[6], double out[6]);
void o_step(const double s[6], double h, double out[6]);
double o_step_length(const o_settings* st, double r, double z);
void o_ray_position(const o_ray* ray, double out[3]);
void o_ray_direction(const o_ray* ray, double out[3]);
/* Integrate; returns outcome, fills steps and max-over-steps drift. */
int o_integrate(o_ray* ray, const o_settings* st, int64_t* steps, double* drift);
double o_redshift_factor(double r, const double direction[3], const double gas[3]);
double o_deflection(const o_ray* launch, const o_ray* result);
double o_critical_impact_parameter(double launch_radius, const o_settings* st, int iterations);

/* Batch form for tests: probes[i] = origin xyz, direction xyz; results[i] =
 * position xyz, direction xyz, drift, outcome, steps, energy, L. */
void o_integrate_batch(const double* probes, int n, const o_settings* st, double* results, int threads);

/* bakeRays (bake.metal:46-91) in FP64 for rays launched at the camera (no
 * sphere jump). samples: n x capacity x (x, y, z, path since the previous
 * stored point); direction_depth: n x (final direction xyz, depth). */
void o_bake_batch(const double* probes, int n, const o_settings* st, double spacing, double half_extent, int capacity,
                  double* samples, int* counts, int* overflowed, int* falls_in, double* direction_depth, int threads);

/* KerrGeodesic.swift:9-281. state: r theta phi pr ptheta energy L */
typedef struct { double step_factor, step_min, step_max, capture_margin, escape_radius; int64_t step_cap; } o_kerr_settings;
void o_kerr_settings_default(o_kerr_settings* s, int64_t step_cap);
double o_kerr_outer_horizon(double a);
double o_kerr_null_residual(double a, const double s[7]);
double o_kerr_carter(double a, const double s[7]);
void o_kerr_derivative(double a, const double s[7], double out[7]);
void o_kerr_step(double a, const double s[7], double h, double out[7]);
double o_kerr_radius(double a, const double p[3]);
void o_kerr_launch(double a, const double origin[3], const double direction[3], double s[7]);
void o_kerr_position(double a, const double s[7], double out[3]);
void o_kerr_direction(double a, const double s[7], double out[3]);
double o_kerr_step_length(double a, const double s[7], const o_kerr_settings* st);
int o_kerr_integrate(double a, double s[7], const o_kerr_settings* st, int64_t* steps, double* drift);
double o_kerr_bisect_critical_xi(double a, double radius, double side, const o_kerr_settings* st, int iterations);
double o_kerr_critical_xi(double a, double rc);
double o_kerr_critical_eta(double a, double rc);
void o_kerr_photon_orbits(double a, double* prograde, double* retrograde);
void o_kerr_integrate_batch(double a, const double* probes, int n, const o_kerr_settings* st, double* results,
                            int threads);

/* Deflection.swift:14-100 */
double o_max_impact_parameter(double r);
double o_sweep(double r, double b, int intervals);
double o_table_impact_parameter(double low, double high, double t);
double o_table_coordinate(double low, double high, double b);
double o_periapsis(double b);
double o_turning_sweep(double r, double b, int intervals);
double o_escape_sweep(double r, double b, int intervals);
void o_sweep_table(double r, int count, int intervals, double* out);
void o_sky_table(double camera_radius, double sphere_radius, int count, int intervals, double* out);

/* Blackbody.swift:11-90 */
void o_blackbody_color(double temperature, double rgb[3]);
void o_blackbody_chromaticity(double temperature, double* x, double* y);
void o_blackbody_table(int count, double tmin, double tmax, double* rgb);
double o_blackbody_coordinate(double t, double tmin, double tmax);

/* VolumeField.swift:40-63: emission size^3 x 4, velocity size^3 x 3. */
void o_volume_sample(int size, double half_extent, const double* emission, const double* velocity,
                     const double p[3], double e4[4], double v3[3]);

/* LensedRender.swift:46-109. camera: position, right, up, forward (3 each)
 * and tanHalfFov (2). out: width*height rgb. */
void o_lensed_image(int width, int height, const double* camera, int size, double half_extent,
                    const double* emission, const double* velocity, const o_settings* st, double opacity,
                    double slab, int redshift, double* out_rgb, int threads);
double o_luminance(const double rgb[3]);
double o_side_ratio(const double* luminance, int width, int height);

/* FP32 replicas of the particle kernels (sim.metal:6-79 with the sqrt-form
 * powers), bit-exact with the device. SimUniforms fields are passed
 * explicitly. particles: n x 8 words in the Particle layout; slot i is the
 * particle of global index first_index + i (0 for an unsharded system). */
void o32_seed(float* particles, uint32_t n, uint32_t seed_lo, uint32_t seed_hi, uint32_t potential,
              const float* inverse_cdf, uint32_t cdf_count, float temperature_scale, uint32_t first_index);
/* o32_seed with a second seeding table: a seed whose third word of the
 * second hash draw is below profile_fraction reads its radius from
 * `profile` (the device's gg_particles_seed_profile). */
void o32_seed_profile(float* particles, uint32_t n, uint32_t seed_lo, uint32_t seed_hi, uint32_t potential,
                      const float* inverse_cdf, uint32_t cdf_count, float temperature_scale, uint32_t first_index,
                      const float* profile, float profile_fraction);
void o32_step(float* particles, uint32_t n, uint32_t seed_lo, uint32_t seed_hi, uint32_t potential,
              const float* inverse_cdf, uint32_t cdf_count, float dt, float alpha, float temperature_scale,
              uint32_t dispatches, int threads, uint32_t first_index);
uint64_t o_fnv1a(const void* bytes, uint64_t count);

/* FP32 replica of the deposit (splat.metal:25-88) into the reference
 * layouts: emission u32[2 n^3], momentum i32[3 n^3], mass u32[n^3]. */
void o32_deposit(const float* particles, uint32_t count, uint32_t size, float half_extent, float peak_temperature,
                 float emission_scale, uint32_t frame, uint32_t exact, uint32_t seed_lo, uint32_t seed_hi,
                 uint32_t* emission, int32_t* momentum, uint32_t* mass, uint32_t first_index, int threads);

/* Resolve (splat.metal:93-120) in FP32 with a float blackbody table
 * (count x 3, linearly interpolated); outputs float rgba per voxel. */
void o32_resolve(const uint32_t* emission, const int32_t* momentum, const uint32_t* mass, uint32_t size,
                 float half_extent, float peak_temperature, const float* blackbody_rgb, int bb_count,
                 float* emission_out, float* velocity_out, int threads);

/* The tone-map kernel's arithmetic in FP32, each operation rounded on its
 * own: per pixel, PBR Neutral (present.metal:22-35) of max(rgb * exposure,
 * 0) from `rgba` (float copies of the half4 colour target), or, when
 * debug_view, the drift heat map (present.metal:40-46) of the half4 debug
 * target with `drift_budget`. Writes rgb before the half rounding. */
void o32_present(const float* rgba, uint32_t count, float exposure, uint32_t debug_view, float drift_budget,
                 float* rgb);

/* Linear [0, 1] (clamped) to 8-bit sRGB, IEC 61966-2-1, rounded to
 * nearest, in FP32. */
void o32_srgb8(const float* v, uint64_t count, uint8_t* out);

/* PBR Neutral (present.metal:22-35) on one colour. */
void o_pbr_neutral(const double in[3], double out[3]);

#ifdef __cplusplus
}
#endif
#endif
