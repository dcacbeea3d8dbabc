// Particle pass: seed and step (sim.metal:6-79), one thread per particle,
// each reading and writing only its own slot, so a seed reproduces the
// state bit for bit.
//
// HBM layout: structure of arrays, two float4 streams, pos = (x, y, z,
// temperature) and vel = (vx, vy, vz, respawns as bits). A warp moves 512
// contiguous bytes per stream with one 16-byte load or store per lane; 32
// bytes per particle are read and written once per dispatch of SIM_SUBSTEPS
// substeps, which makes the step a pure HBM stream.
//
// This translation unit is compiled with --fmad=false: every multiply and
// add is rounded separately, in the order written, so the results equal the
// CPU replica's (oracle/replica.c) bit for bit. The spawn's sin, cos and log
// come from gargantua_detmath.h for the same reason.
#include <cstring>
#include <vector>

#include "../../include/gargantua_detmath.h"
#include "common.cuh"
#include "runtime.h"

namespace gg {

struct SimArgs {
    float4* __restrict__ pos;
    float4* __restrict__ vel;
    const float* __restrict__ inverse_cdf;
    SimUniforms u;
    uint32_t first_index;  // global index of slot 0: the hash is keyed on global indices
    const float* __restrict__ profile_cdf;  // second seeding table, or null
    float profile_fraction;                 // share of seeds drawn from it
};

// Unnormalized thin-disk profile (Common.h:49-53) with the powers as square
// roots: x^(3/4) t^(1/4) = sqrt(x) sqrt(sqrt(x t)), sqrt(x) shared with the
// zero-torque factor.
__device__ __forceinline__ float disk_shape_f(float r) {
    float x = R_ISCO / r;
    float h = sqrtf(x);
    float torque = fmaxf(1.0f - h, ZERO_TORQUE_FLOOR);
    return gg_disk_powers(x, h, torque);
}

__device__ __forceinline__ float square3(float x, float y, float z) { return x * x + y * y + z * z; }
__device__ __forceinline__ float len3(float x, float y, float z) { return sqrtf(square3(x, y, z)); }

// The step's two tests of a length against a limit, made on the squared
// length: sqrt rounds correctly and monotonically, so sqrt(s) > 12 exactly
// when s > 144 (no float lies between 144 and (12 + half an ulp)^2), and
// sqrt(s) < 2.02f exactly when s < 4.0803995f (bits 0x408292a2, the least
// float whose square root rounds to 2.02f or above). Both bounds were found
// by testing every float near the squares; a CPU test repeats that search.
// g(r) = 1 / kick_denominator(r): d^2 with d = max(r - 2, 1e-6) for
// Paczynski-Wiita, r^2 for Newton (Common.h:32-46).
__device__ __forceinline__ float kick_denominator(float r, uint32_t potential) {
    if (potential == PotentialPaczynskiWiita) {
        float d = fmaxf(r - R_SCHWARZSCHILD, 1e-6f);
        return d * d;
    }
    return r * r;
}

constexpr float kPlungeSpeedSquared = 144.0f;
constexpr uint32_t kCaptureClosestSquaredBits = 0x408292a2u;
static_assert(PLUNGE_SPEED_LIMIT == 12.0f && R_CAPTURE == 2.02f, "the squared bounds belong to these limits");

// spawn (sim.metal:6-34): event 0 seeds from the steady profile, later
// events respawn into the feeding annulus. With a second seeding table
// (gg_particles_seed_profile), a seed whose spare hash word h1.z falls below
// the profile's share reads its radius from that table instead.
__device__ void spawn(uint32_t index, uint32_t event, const SimArgs& a, bool from_disk, float4& p, float4& v) {
    const SimUniforms& u = a.u;
    uint4 h0 = pcg4d(make_uint4(index, event, u.seed.x, u.seed.y));
    uint4 h1 = pcg4d(make_uint4(index, event, u.seed.x ^ 0x9E3779B9u, u.seed.y));
    float u0 = unit_float(h0.x), u1 = unit_float(h0.y), u2 = unit_float(h0.z), u3 = unit_float(h0.w);
    float u4 = unit_float(h1.x), u5 = unit_float(h1.y);
    float r;
    if (from_disk) {
        const float* table =
            (a.profile_cdf && unit_float(h1.z) < a.profile_fraction) ? a.profile_cdf : a.inverse_cdf;
        float position = u0 * (float)(u.inverseCdfCount - 1u);
        uint32_t k = (uint32_t)position;
        if (k > u.inverseCdfCount - 2u) k = u.inverseCdfCount - 2u;
        float lo = __ldg(table + k), hi = __ldg(table + k + 1u);
        r = lo + (hi - lo) * (position - (float)k);
    } else {
        float inner = R_FEED_INNER * R_FEED_INNER;
        float outer = R_DISK_OUTER * R_DISK_OUTER;
        r = sqrtf(inner + (outer - inner) * u0);
    }
    float phi = 2.0f * GG_PI_F * u1;
    float radius01 = sqrtf(-2.0f * gg_logf(1.0f - u2));
    float angle01 = 2.0f * GG_PI_F * u3;
    float s01, c01;
    gg_sincosf(angle01, &s01, &c01);
    float g0 = radius01 * c01, g1 = radius01 * s01;
    float radius23 = sqrtf(-2.0f * gg_logf(1.0f - u4));
    float angle23 = 2.0f * GG_PI_F * u5;
    float s23, c23;
    gg_sincosf(angle23, &s23, &c23);
    float g2 = radius23 * c23, g3 = radius23 * s23;
    float vc = circular_speed(r, u.potential);
    float sphi, cphi;
    gg_sincosf(phi, &sphi, &cphi);
    float spread = FEED_VELOCITY_DISPERSION * vc;
    p.x = r * cphi;
    p.y = r * sphi;
    p.z = DISK_ASPECT * r * g0;
    p.w = u.temperatureScale * disk_shape_f(r);
    v.x = vc * (-sphi) + spread * g1;
    v.y = vc * cphi + spread * g2;
    v.z = vc * 0.0f + spread * g3;
    v.w = __uint_as_float(event);
}

__global__ void __launch_bounds__(256) seed_kernel(SimArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.u.particleCount) return;
    float4 p, v;
    spawn(a.first_index + i, 0u, a, true, p, v);
    a.pos[i] = p;
    a.vel[i] = v;
}

// stepParticles (sim.metal:44-79): per substep a gravity kick, drag
// proportional to the local circular angular frequency, a drift, and a
// respawn when the swept chord passes inside R_CAPTURE, the particle leaves
// R_ESCAPE or outruns PLUNGE_SPEED_LIMIT; the temperature follows the final
// radius.
//
// Three changes against the reference's arithmetic, shared with the CPU
// replica: the kick factor k = -g(r) / r is one divide, -1 / (d^2 r) with d
// = max(r - 2, 1e-6) (the reference divides 1 / d^2 by r); the angular
// frequency is sqrt(-k) = sqrt(g / r), where the reference divides
// circular_speed(r) = sqrt(r g) by r (the same quantity, one divide fewer);
// and the chord's closest approach is only computed when
// it can matter. A substep that starts at |x| > 4 and moves less than 1
// keeps every point of its chord more than 3 from the centre, so the
// computed squared distance (exact up to a few ulps) is far above the
// capture bound 4.08 and the test cannot fire: skipping it gives the same
// outcome bit for bit, and saves its divide for nearly every particle.
__global__ void __launch_bounds__(256) step_kernel(SimArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.u.particleCount) return;
    const SimUniforms& u = a.u;
    float4 p = a.pos[i];
    float4 v = a.vel[i];
    float px = p.x, py = p.y, pz = p.z;
    float vx = v.x, vy = v.y, vz = v.z;
    const float capture_squared = __uint_as_float(kCaptureClosestSquaredBits);
    float r = len3(px, py, pz);  // |x| at the start of each substep
#pragma unroll
    for (uint32_t s = 0; s < SIM_SUBSTEPS; ++s) {
        float k = -1.0f / (kick_denominator(r, u.potential) * r);
        float omega = sqrtf(-k);
        const float r_before = r;
        vx = vx + px * k * u.dt;
        vy = vy + py * k * u.dt;
        vz = vz + pz * k * u.dt;
        float drag = u.alpha * omega * u.dt;
        vx = vx - vx * drag;
        vy = vy - vy * drag;
        vz = vz - vz * drag;
        float bx = px, by = py, bz = pz;
        px = px + vx * u.dt;
        py = py + vy * u.dt;
        pz = pz + vz * u.dt;
        r = len3(px, py, pz);
        float tx = px - bx, ty = py - by, tz = pz - bz;
        float tt = tx * tx + ty * ty + tz * tz;
        // closest < R_CAPTURE and |v| > PLUNGE_SPEED_LIMIT, on the squares
        bool captured = false;
        if (!(r_before > 4.0f && tt < 1.0f)) {
            float bt = bx * tx + by * ty + bz * tz;
            float along = fminf(fmaxf(-bt / fmaxf(tt, 1e-12f), 0.0f), 1.0f);
            float closest_squared = square3(bx + along * tx, by + along * ty, bz + along * tz);
            captured = closest_squared < capture_squared;
        }
        if (captured || r > R_ESCAPE || square3(vx, vy, vz) > kPlungeSpeedSquared) {
            float4 np, nv;
            spawn(a.first_index + i, __float_as_uint(v.w) + 1u, a, false, np, nv);
            px = np.x; py = np.y; pz = np.z;
            vx = nv.x; vy = nv.y; vz = nv.z;
            v.w = nv.w;
            r = len3(px, py, pz);
        }
    }
    float t = u.temperatureScale * disk_shape_f(r);
    a.pos[i] = make_float4(px, py, pz, t);
    a.vel[i] = make_float4(vx, vy, vz, v.w);
}

}  // namespace gg

using namespace gg;

static int check_particles(const gg_particles* ps, const char* what) {
    if (!ps) return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s needs a particle system.", what);
    return GG_OK;
}

static SimArgs sim_args(gg_particles* ps) {
    SimArgs a;
    a.pos = ps->pos;
    a.vel = ps->vel;
    a.inverse_cdf = ps->inverse_cdf;
    a.u = ps->uniforms;
    a.first_index = ps->first_index;
    a.profile_cdf = ps->profile_cdf;
    a.profile_fraction = ps->profile_fraction;
    return a;
}

extern "C" {

GG_API int gg_particles_create(gg_context* ctx, uint32_t count, uint64_t seed, uint32_t potential,
                               gg_particles** out) {
    return gg_particles_create_shard(ctx, count, 0u, seed, potential, out);
}

GG_API int gg_particles_create_shard(gg_context* ctx, uint32_t count, uint32_t first_index, uint64_t seed,
                                     uint32_t potential, gg_particles** out) {
    if (!ctx || !out) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_particles_create needs a context and an output.");
    if ((uint64_t)first_index + count > 0xffffffffull)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Shard [%u, %u + %u) exceeds 32-bit particle indices.", first_index,
                        first_index, count);
    *out = nullptr;
    if (count == 0) return gg::fail(GG_ERR_INVALID_ARGUMENT, "A particle system needs at least one particle.");
    if (potential != PotentialNewtonian && potential != PotentialPaczynskiWiita)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Unknown potential %u.", potential);
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    uint64_t bytes = (uint64_t)count * 32u + INVERSE_CDF_COUNT * sizeof(float);
    if (ctx->used + bytes > ctx->budget)
        return gg::fail(GG_ERR_OVER_BUDGET, "%u particles need %llu bytes but the budget has %llu bytes left.", count,
                        (unsigned long long)bytes, (unsigned long long)(ctx->budget - ctx->used));
    gg_particles* ps = new gg_particles();
    ps->ctx = ctx;
    ps->count = count;
    ps->first_index = first_index;
    ps->seed = seed;
    ps->potential = potential;
    int s = gg::device_alloc(ctx, (uint64_t)count * 16u, (void**)&ps->pos, "particle positions");
    if (s == GG_OK) s = gg::device_alloc(ctx, (uint64_t)count * 16u, (void**)&ps->vel, "particle velocities");
    if (s == GG_OK)
        s = gg::device_alloc(ctx, INVERSE_CDF_COUNT * sizeof(float), (void**)&ps->inverse_cdf, "seeding table");
    if (s != GG_OK) {
        gg_particles_destroy(ps);
        return s;
    }
    // ParticleSystem.swift:23-26: FP64 table rounded to float.
    std::vector<double> table(INVERSE_CDF_COUNT);
    gg::radial_inverse_cdf(INVERSE_CDF_COUNT, 8192, table.data());
    std::vector<float> tf(table.begin(), table.end());
    s = gg::cuda_status(cudaMemcpyAsync(ps->inverse_cdf, tf.data(), tf.size() * sizeof(float),
                                        cudaMemcpyHostToDevice, ctx->stream),
                        "seeding table upload");
    if (s == GG_OK) s = gg::cuda_status(cudaStreamSynchronize(ctx->stream), "seeding table upload");
    if (s != GG_OK) {
        gg_particles_destroy(ps);
        return s;
    }
    // ParticleSystem.swift:59-70.
    double peak_r = R_ISCO * 49.0 / 36.0;
    double peak_shape = gg::disk_shape(peak_r, ZERO_TORQUE_FLOOR);
    SimUniforms& u = ps->uniforms;
    u.seed.x = (uint32_t)seed;
    u.seed.y = (uint32_t)(seed >> 32);
    u.particleCount = count;
    u.potential = potential;
    u.inverseCdfCount = INVERSE_CDF_COUNT;
    u.dt = SIM_DT;
    u.alpha = DRAG_ALPHA;
    u.temperatureScale = (float)((double)T_PEAK_DEFAULT / peak_shape);
    *out = ps;
    return GG_OK;
}

GG_API void gg_particles_destroy(gg_particles* ps) {
    if (!ps) return;
    gg_context* ctx = ps->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    gg::device_free(ctx, ps->pos, (uint64_t)ps->count * 16u);
    gg::device_free(ctx, ps->vel, (uint64_t)ps->count * 16u);
    gg::device_free(ctx, ps->inverse_cdf, INVERSE_CDF_COUNT * sizeof(float));
    gg::device_free(ctx, ps->profile_cdf, INVERSE_CDF_COUNT * sizeof(float));
    delete ps;
}

GG_API int gg_particles_uniforms(gg_particles* ps, SimUniforms* out) {
    GG_CHECK(check_particles(ps, "gg_particles_uniforms"));
    if (!out) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_particles_uniforms needs an output.");
    *out = ps->uniforms;
    return GG_OK;
}

GG_API int gg_particles_seed(gg_particles* ps) {
    GG_CHECK(check_particles(ps, "gg_particles_seed"));
    gg_context* ctx = ps->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    uint32_t blocks = (ps->count + 255u) / 256u;
    seed_kernel<<<blocks, 256, 0, ctx->stream>>>(sim_args(ps));
    return gg::launch_status("seed particles");
}

GG_API int gg_particles_step(gg_particles* ps, uint32_t dispatches) {
    gg::Range range("gg_particles_step");
    GG_CHECK(check_particles(ps, "gg_particles_step"));
    gg_context* ctx = ps->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    uint32_t blocks = (ps->count + 255u) / 256u;
    SimArgs a = sim_args(ps);
    for (uint32_t d = 0; d < dispatches; ++d) step_kernel<<<blocks, 256, 0, ctx->stream>>>(a);
    return gg::launch_status("step particles");
}

GG_API int gg_particles_read(gg_particles* ps, Particle* out, uint32_t count) {
    GG_CHECK(check_particles(ps, "gg_particles_read"));
    if (!out || count != ps->count)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_particles_read needs an array of exactly %u particles.", ps->count);
    gg_context* ctx = ps->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    std::vector<float4> p(count), v(count);
    GG_CUDA(cudaMemcpyAsync(p.data(), ps->pos, (size_t)count * 16u, cudaMemcpyDeviceToHost, ctx->stream), "particle readback");
    GG_CUDA(cudaMemcpyAsync(v.data(), ps->vel, (size_t)count * 16u, cudaMemcpyDeviceToHost, ctx->stream), "particle readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "particle readback");
    for (uint32_t i = 0; i < count; ++i) {
        Particle& q = out[i];
        q.position = {p[i].x, p[i].y, p[i].z};
        q.velocity = {v[i].x, v[i].y, v[i].z};
        q.temperature = p[i].w;
        std::memcpy(&q.respawns, &v[i].w, 4);
    }
    return GG_OK;
}

GG_API int gg_particles_write(gg_particles* ps, const Particle* in, uint32_t count) {
    GG_CHECK(check_particles(ps, "gg_particles_write"));
    if (!in || count != ps->count)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_particles_write needs an array of exactly %u particles.", ps->count);
    gg_context* ctx = ps->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    std::vector<float4> p(count), v(count);
    for (uint32_t i = 0; i < count; ++i) {
        const Particle& q = in[i];
        p[i] = make_float4(q.position.x, q.position.y, q.position.z, q.temperature);
        float bits;
        std::memcpy(&bits, &q.respawns, 4);
        v[i] = make_float4(q.velocity.x, q.velocity.y, q.velocity.z, bits);
    }
    GG_CUDA(cudaMemcpyAsync(ps->pos, p.data(), (size_t)count * 16u, cudaMemcpyHostToDevice, ctx->stream), "particle upload");
    GG_CUDA(cudaMemcpyAsync(ps->vel, v.data(), (size_t)count * 16u, cudaMemcpyHostToDevice, ctx->stream), "particle upload");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "particle upload");
    return GG_OK;
}

// FNV-1a 64 over the AoS bytes (Validate.swift:378-387), on the host after a
// readback: the hash is a serial chain over every byte.
GG_API int gg_particles_checksum(gg_particles* ps, uint64_t* out) {
    GG_CHECK(check_particles(ps, "gg_particles_checksum"));
    if (!out) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_particles_checksum needs an output.");
    std::vector<Particle> aos(ps->count);
    GG_CHECK(gg_particles_read(ps, aos.data(), ps->count));
    const uint8_t* b = reinterpret_cast<const uint8_t*>(aos.data());
    uint64_t hash = 0xcbf29ce484222325ULL;
    const uint64_t n = (uint64_t)aos.size() * sizeof(Particle);
    for (uint64_t i = 0; i < n; ++i) {
        hash ^= b[i];
        hash *= 0x100000001b3ULL;
    }
    *out = hash;
    return GG_OK;
}

GG_API int gg_particles_seed_profile(gg_particles* ps, float fraction, float exponent) {
    GG_CHECK(check_particles(ps, "gg_particles_seed_profile"));
    if (!(fraction >= 0.0f && fraction <= 1.0f) || !(exponent >= 0.0f && exponent <= 8.0f))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Seed profile needs a share in [0, 1] and an exponent in [0, 8].");
    gg_context* ctx = ps->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (!ps->profile_cdf)
        GG_CHECK(gg::device_alloc(ctx, INVERSE_CDF_COUNT * sizeof(float), (void**)&ps->profile_cdf, "profile table"));
    std::vector<double> table(INVERSE_CDF_COUNT);
    gg::power_law_inverse_cdf(INVERSE_CDF_COUNT, (double)exponent, table.data());
    std::vector<float> tf(table.begin(), table.end());
    GG_CUDA(cudaMemcpyAsync(ps->profile_cdf, tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice,
                            ctx->stream),
            "profile table upload");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "profile table upload");
    ps->profile_fraction = fraction;
    return GG_OK;
}

GG_API int gg_particles_profile_table(gg_particles* ps, float* out, uint32_t count) {
    GG_CHECK(check_particles(ps, "gg_particles_profile_table"));
    if (!out || count != INVERSE_CDF_COUNT)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_particles_profile_table needs %u floats.", INVERSE_CDF_COUNT);
    if (!ps->profile_cdf) return gg::fail(GG_ERR_INVALID_ARGUMENT, "No seed profile was set.");
    gg_context* ctx = ps->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    GG_CUDA(cudaMemcpyAsync(out, ps->profile_cdf, count * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream),
            "table readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "table readback");
    return GG_OK;
}

GG_API int gg_particles_inverse_cdf(gg_particles* ps, float* out, uint32_t count) {
    GG_CHECK(check_particles(ps, "gg_particles_inverse_cdf"));
    if (!out || count != INVERSE_CDF_COUNT)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_particles_inverse_cdf needs %u floats.", INVERSE_CDF_COUNT);
    gg_context* ctx = ps->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    GG_CUDA(cudaMemcpyAsync(out, ps->inverse_cdf, count * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream), "table readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "table readback");
    return GG_OK;
}

}  // extern "C"
