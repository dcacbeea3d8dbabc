/*
 * TEST INFRASTRUCTURE ONLY: FP32 replicas of the particle, deposit and
 * resolve kernels, for bit-exact comparison with the device. They restate
 * sim.metal:6-79 and splat.metal:25-120 in single precision with one fixed
 * operation order (left to right as written in the shaders, no fused
 * multiply-add: built with -ffp-contract=off). The few transcendentals come
 * from gargantua_detmath.h, the series implementations both sides share, so
 * that sin, cos and log give the same bits on the CPU and the GPU.
 *
 * Two deliberate, documented choices, shared with the kernels:
 *  - pow(x, 0.75) and pow(t, 0.25) in the disk profile are evaluated as
 *    sqrt(x) sqrt(sqrt(x)) and sqrt(sqrt(t)) (exact identities, each factor
 *    correctly rounded);
 *  - the cloud-in-cell weight mix(1 - f, f, bit) is evaluated as the
 *    selection it stands for, bit ? f : 1 - f.
 */
#include "oracle.h"
#include "../include/gargantua_types.h"
#include "../include/gargantua_constants.h"
#include "../include/gargantua_detmath.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_F 3.14159265358979323846f

static void pcg(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t out[4]) {
    uint32_t in[4] = {a, b, c, d};
    o_pcg4d(in, out);
}

static float unitf(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

static float gradf(float r, uint32_t potential) {
    if (potential == PotentialPaczynskiWiita) {
        float d = fmaxf(r - R_SCHWARZSCHILD, 1e-6f);
        return 1.0f / (d * d);
    }
    return 1.0f / (r * r);
}

static float circular_speedf(float r, uint32_t potential) { return sqrtf(r * gradf(r, potential)); }

static float disk_shapef(float r) {
    float x = R_ISCO / r;
    float h = sqrtf(x);
    float torque = fmaxf(1.0f - h, ZERO_TORQUE_FLOOR);
    return gg_disk_powers(x, h, torque);
}

static float length3f(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

typedef struct {
    uint32_t seed_lo, seed_hi, potential, cdf_count;
    const float* cdf;
    float dt, alpha, temperature_scale;
    const float* profile; /* second seeding table or NULL */
    float profile_fraction;
} sim32;

/* sim.metal:6-34 */
static void spawn32(uint32_t index, uint32_t event, const sim32* u, int from_disk, float* p) {
    uint32_t h0[4], h1[4];
    pcg(index, event, u->seed_lo, u->seed_hi, h0);
    pcg(index, event, u->seed_lo ^ 0x9E3779B9u, u->seed_hi, h1);
    float u0 = unitf(h0[0]), u1 = unitf(h0[1]), u2 = unitf(h0[2]), u3 = unitf(h0[3]);
    float u4 = unitf(h1[0]), u5 = unitf(h1[1]);
    float r;
    if (from_disk) {
        const float* table = (u->profile && unitf(h1[2]) < u->profile_fraction) ? u->profile : u->cdf;
        float position = u0 * (float)(u->cdf_count - 1u);
        uint32_t k = (uint32_t)position;
        if (k > u->cdf_count - 2u) k = u->cdf_count - 2u;
        float a = table[k], b = table[k + 1u];
        r = a + (b - a) * (position - (float)k);
    } else {
        float inner = R_FEED_INNER * R_FEED_INNER;
        float outer = R_DISK_OUTER * R_DISK_OUTER;
        r = sqrtf(inner + (outer - inner) * u0);
    }
    float phi = 2.0f * PI_F * u1;
    float radius01 = sqrtf(-2.0f * gg_logf(1.0f - u2));
    float angle01 = 2.0f * PI_F * u3;
    float s01, c01;
    gg_sincosf(angle01, &s01, &c01);
    float g0 = radius01 * c01, g1 = radius01 * s01;
    float radius23 = sqrtf(-2.0f * gg_logf(1.0f - u4));
    float angle23 = 2.0f * PI_F * u5;
    float s23, c23;
    gg_sincosf(angle23, &s23, &c23);
    float g2 = radius23 * c23, g3 = radius23 * s23;
    float vc = circular_speedf(r, u->potential);
    float sphi, cphi;
    gg_sincosf(phi, &sphi, &cphi);
    float spread = FEED_VELOCITY_DISPERSION * vc;
    p[0] = r * cphi;
    p[1] = r * sphi;
    p[2] = DISK_ASPECT * r * g0;
    p[3] = vc * (-sphi) + spread * g1;
    p[4] = vc * cphi + spread * g2;
    p[5] = vc * 0.0f + spread * g3;
    p[6] = u->temperature_scale * disk_shapef(r);
    memcpy(&p[7], &event, 4);
}

/* g(r) = 1 / kick_denominator(r) (Common.h:32-46). */
static float kick_denominator(float r, uint32_t potential) {
    if (potential == PotentialPaczynskiWiita) {
        float d = fmaxf(r - R_SCHWARZSCHILD, 1e-6f);
        return d * d;
    }
    return r * r;
}

/* sim.metal:44-79, with the kick factor as one divide, k = -1 / (d^2 r)
 * (the reference divides 1 / d^2 by r), and the angular frequency as
 * sqrt(-k) = sqrt(g / r) (the reference divides circular_speed(r) =
 * sqrt(r g) by r), as the kernel computes them. */
static void step32(uint32_t i, const sim32* u, float* p) {
    float px = p[0], py = p[1], pz = p[2];
    float vx = p[3], vy = p[4], vz = p[5];
    for (uint32_t s = 0; s < SIM_SUBSTEPS; ++s) {
        float r = length3f(px, py, pz);
        float k = -1.0f / (kick_denominator(r, u->potential) * r);
        float omega = sqrtf(-k);
        vx = vx + px * k * u->dt;
        vy = vy + py * k * u->dt;
        vz = vz + pz * k * u->dt;
        float drag = u->alpha * omega * u->dt;
        vx = vx - vx * drag;
        vy = vy - vy * drag;
        vz = vz - vz * drag;
        float bx = px, by = py, bz = pz;
        px = px + vx * u->dt;
        py = py + vy * u->dt;
        pz = pz + vz * u->dt;
        r = length3f(px, py, pz);
        float tx = px - bx, ty = py - by, tz = pz - bz;
        float bt = bx * tx + by * ty + bz * tz;
        float tt = tx * tx + ty * ty + tz * tz;
        float along = fminf(fmaxf(-bt / fmaxf(tt, 1e-12f), 0.0f), 1.0f);
        float closest = length3f(bx + along * tx, by + along * ty, bz + along * tz);
        if (closest < R_CAPTURE || r > R_ESCAPE || length3f(vx, vy, vz) > PLUNGE_SPEED_LIMIT) {
            uint32_t respawns;
            memcpy(&respawns, &p[7], 4);
            spawn32(i, respawns + 1u, u, 0, p);
            px = p[0]; py = p[1]; pz = p[2];
            vx = p[3]; vy = p[4]; vz = p[5];
        }
    }
    p[0] = px; p[1] = py; p[2] = pz;
    p[3] = vx; p[4] = vy; p[5] = vz;
    p[6] = u->temperature_scale * disk_shapef(length3f(px, py, pz));
}

void o32_seed(float* particles, uint32_t n, uint32_t seed_lo, uint32_t seed_hi, uint32_t potential,
              const float* cdf, uint32_t cdf_count, float temperature_scale, uint32_t first_index) {
    o32_seed_profile(particles, n, seed_lo, seed_hi, potential, cdf, cdf_count, temperature_scale, first_index, NULL,
                     0.0f);
}

void o32_seed_profile(float* particles, uint32_t n, uint32_t seed_lo, uint32_t seed_hi, uint32_t potential,
                      const float* cdf, uint32_t cdf_count, float temperature_scale, uint32_t first_index,
                      const float* profile, float profile_fraction) {
    sim32 u = {seed_lo, seed_hi, potential, cdf_count, cdf, 0.0f, 0.0f, temperature_scale, profile, profile_fraction};
    for (uint32_t i = 0; i < n; ++i) spawn32(first_index + i, 0u, &u, 1, particles + 8 * (uint64_t)i);
}

void o32_step(float* particles, uint32_t n, uint32_t seed_lo, uint32_t seed_hi, uint32_t potential,
              const float* cdf, uint32_t cdf_count, float dt, float alpha, float temperature_scale,
              uint32_t dispatches, int threads, uint32_t first_index) {
    sim32 u = {seed_lo, seed_hi, potential, cdf_count, cdf, dt, alpha, temperature_scale, NULL, 0.0f};
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i)
        for (uint32_t d = 0; d < dispatches; ++d) step32(first_index + (uint32_t)i, &u, particles + 8 * i);
}

/* Validate.swift:378-387 */
uint64_t o_fnv1a(const void* bytes, uint64_t count) {
    const uint8_t* b = (const uint8_t*)bytes;
    uint64_t hash = 0xcbf29ce484222325ULL;
    for (uint64_t i = 0; i < count; ++i) {
        hash ^= (uint64_t)b[i];
        hash *= 0x100000001b3ULL;
    }
    return hash;
}

/* Add v to *word; shared between threads when `atomic` (the sums are
 * integers, so the order of the adds does not change the result). */
static inline void add_u32(uint32_t* word, uint32_t v, int atomic) {
    if (atomic) {
#pragma omp atomic
        *word += v;
    } else {
        *word += v;
    }
}

/* splat.metal:25-37: one corner's six fixed-point sums */
static void deposit32(uint32_t* em, int32_t* mo, uint32_t* ma, uint32_t index, float weight, float energy,
                      float relative, float vx, float vy, float vz, int atomic) {
    uint32_t fe = (uint32_t)(energy * weight * 16777216.0f + 0.5f);
    uint32_t fet = (uint32_t)(energy * relative * weight * 1048576.0f + 0.5f);
    float ms = weight * 4096.0f;
    int32_t mx = (int32_t)rintf(vx * ms), my = (int32_t)rintf(vy * ms), mz = (int32_t)rintf(vz * ms);
    uint32_t fm = (uint32_t)(weight * 256.0f + 0.5f);
    /* momentum words add in two's complement with wraparound, as the
     * device's integer atomics do */
    uint32_t* mu = (uint32_t*)mo;
    add_u32(&em[2u * index + 0u], fe, atomic);
    add_u32(&em[2u * index + 1u], fet, atomic);
    add_u32(&mu[3u * index + 0u], (uint32_t)mx, atomic);
    add_u32(&mu[3u * index + 1u], (uint32_t)my, atomic);
    add_u32(&mu[3u * index + 2u], (uint32_t)mz, atomic);
    add_u32(&ma[index], fm, atomic);
}

/* splat.metal:44-88. threads == 1 deposits serially; otherwise the particles
 * are split over OpenMP threads (threads <= 0: the runtime's default count)
 * that add into the shared sums atomically. */
void o32_deposit(const float* particles, uint32_t count, uint32_t n, float half_extent, float peak_temperature,
                 float emission_scale, uint32_t frame, uint32_t exact, uint32_t seed_lo, uint32_t seed_hi,
                 uint32_t* em, int32_t* mo, uint32_t* ma, uint32_t first_index, int threads) {
    const int atomic = threads != 1;
#ifdef _OPENMP
    if (threads > 1) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(static) if (atomic)
    for (int64_t ii = 0; ii < (int64_t)count; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const float* p = particles + 8 * (uint64_t)i;
        float pos[3] = {p[0], p[1], p[2]};
        float unit[3];
        int outside = 0;
        for (int a = 0; a < 3; ++a) {
            unit[a] = (pos[a] + half_extent) / (2.0f * half_extent);
            if (unit[a] < 0.0f || unit[a] >= 1.0f) outside = 1;
        }
        if (outside) continue;
        float relative = p[6] / peak_temperature;
        float energy = relative * relative * relative * relative * emission_scale;
        int low[3], high[3];
        float frac[3];
        for (int a = 0; a < 3; ++a) {
            float grid = unit[a] * (float)n - 0.5f;
            float base = floorf(grid);
            frac[a] = grid - base;
            int b = (int)base;
            high[a] = b + 1 < (int)n - 1 ? b + 1 : (int)n - 1;
            low[a] = b > 0 ? b : 0;
        }
        if (exact) {
            for (uint32_t c = 0; c < CIC_CORNERS; ++c) {
                int corner[3];
                float w3[3];
                for (int a = 0; a < 3; ++a) {
                    int bit = (c >> a) & 1u;
                    corner[a] = bit ? high[a] : low[a];
                    w3[a] = bit ? frac[a] : 1.0f - frac[a];
                }
                float w = w3[0] * w3[1] * w3[2];
                if (w <= 0.0f) continue;
                uint32_t index = ((uint32_t)corner[2] * n + (uint32_t)corner[1]) * n + (uint32_t)corner[0];
                deposit32(em, mo, ma, index, w, energy, relative, p[3], p[4], p[5], atomic);
            }
        } else {
            uint32_t h[4];
            pcg(first_index + i, frame, seed_lo, seed_hi, h);
            int corner[3];
            for (int a = 0; a < 3; ++a) corner[a] = unitf(h[a]) < frac[a] ? high[a] : low[a];
            uint32_t index = ((uint32_t)corner[2] * n + (uint32_t)corner[1]) * n + (uint32_t)corner[0];
            deposit32(em, mo, ma, index, 1.0f, energy, relative, p[3], p[4], p[5], atomic);
        }
    }
}

/* Blackbody table coordinate (Common.h:56-59), evaluated in double with the
 * shared series log and rounded once. */
static float bb_coordinate(float temperature) {
    float t = fminf(fmaxf(temperature, BLACKBODY_T_MIN), BLACKBODY_T_MAX);
    double lo = gg_log_d((double)BLACKBODY_T_MIN);
    double hi = gg_log_d((double)BLACKBODY_T_MAX);
    return (float)((gg_log_d((double)t) - lo) / (hi - lo));
}

/* splat.metal:93-120 with the linear clamp-to-edge lookup done in FP32.
 * Voxels are split over `threads` OpenMP threads (1: serial; <= 0: the
 * runtime's default count); each voxel is independent. */
void o32_resolve(const uint32_t* em, const int32_t* mo, const uint32_t* ma, uint32_t n, float half_extent,
                 float peak_temperature, const float* bb, int bb_count, float* eo, float* vo, int threads) {
    float voxel = 2.0f * half_extent / (float)n;
    float inverse_volume = 1.0f / (voxel * voxel * voxel);
    int64_t total = (int64_t)n * n * n;
#ifdef _OPENMP
    if (threads > 1) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(static) if (threads != 1)
    for (int64_t index = 0; index < total; ++index) {
        float count = (float)ma[index] / 256.0f;
        float energy = (float)em[2 * index + 0] / 16777216.0f;
        float energy_t = (float)em[2 * index + 1] / 1048576.0f;
        float tint[3] = {0.0f, 0.0f, 0.0f};
        if (energy > 0.0f) {
            float mean_t = energy_t / energy * peak_temperature;
            float x = bb_coordinate(mean_t) * (float)bb_count - 0.5f;
            float fl = floorf(x);
            float f = x - fl;
            int i0 = (int)fl, i1 = i0 + 1;
            if (i0 < 0) i0 = 0;
            if (i0 > bb_count - 1) i0 = bb_count - 1;
            if (i1 < 0) i1 = 0;
            if (i1 > bb_count - 1) i1 = bb_count - 1;
            for (int c = 0; c < 3; ++c) {
                float a = bb[3 * i0 + c], b = bb[3 * i1 + c];
                tint[c] = a + (b - a) * f;
            }
        }
        float m[3] = {(float)mo[3 * index + 0] / 4096.0f, (float)mo[3 * index + 1] / 4096.0f,
                      (float)mo[3 * index + 2] / 4096.0f};
        float density = count * inverse_volume;
        for (int c = 0; c < 3; ++c) {
            eo[4 * index + c] = tint[c] * energy * inverse_volume;
            vo[4 * index + c] = count > 0.0f ? m[c] / count : 0.0f;
        }
        eo[4 * index + 3] = density;
        vo[4 * index + 3] = 1.0f;
    }
}

/* present.metal:22-35 (pbrNeutral), FP32 */
static void pbr_neutral32(float c[3]) {
    const float start = 0.8f - 0.04f;
    const float desat = 0.15f;
    float x = fminf(c[0], fminf(c[1], c[2]));
    float offset = x < 0.08f ? x - 6.25f * x * x : 0.04f;
    for (int i = 0; i < 3; ++i) c[i] = c[i] - offset;
    float peak = fmaxf(c[0], fmaxf(c[1], c[2]));
    if (peak < start) return;
    const float d = 1.0f - start;
    float np = 1.0f - d * d / (peak + d - start);
    float sc = np / peak;
    for (int i = 0; i < 3; ++i) c[i] = c[i] * sc;
    float g = 1.0f - 1.0f / (desat * (peak - np) + 1.0f);
    for (int i = 0; i < 3; ++i) c[i] = c[i] + (np - c[i]) * g;
}

/* present.metal:40-46 (driftHeat), FP32 */
static void drift_heat32(const float d[4], float budget, float out[3]) {
    float t = fminf(fmaxf(d[0] / budget, 0.0f), 2.0f) * 0.5f;
    float heat[3] = {t, 1.0f - fabsf(t - 0.5f) * 2.0f, 1.0f - t};
    float shade = 0.2f + 0.8f * fminf(fmaxf(d[1] / (float)STEP_CAP_INTERACTIVE, 0.0f), 1.0f);
    if (d[2] < 0.5f) shade = shade * 0.35f;
    for (int i = 0; i < 3; ++i) out[i] = heat[i] * shade;
}

void o32_present(const float* rgba, uint32_t count, float exposure, uint32_t debug_view, float drift_budget,
                 float* rgb) {
    for (uint32_t i = 0; i < count; ++i) {
        const float* h = rgba + 4 * (uint64_t)i;
        float* o = rgb + 3 * (uint64_t)i;
        if (debug_view) {
            drift_heat32(h, drift_budget, o);
        } else {
            float c[3] = {fmaxf(h[0] * exposure, 0.0f), fmaxf(h[1] * exposure, 0.0f), fmaxf(h[2] * exposure, 0.0f)};
            pbr_neutral32(c);
            o[0] = c[0];
            o[1] = c[1];
            o[2] = c[2];
        }
    }
}

void o32_srgb8(const float* v, uint64_t count, uint8_t* out) {
    for (uint64_t i = 0; i < count; ++i) {
        float x = fminf(fmaxf(v[i], 0.0f), 1.0f);
        float e = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
        out[i] = (uint8_t)lrintf(e * 255.0f);
    }
}
