// Internal runtime of the library: the context, status reporting, budgeted
// device allocation and the handle structs every translation unit shares.
// Not part of the public interface (include/gargantua.h is).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/gargantua.h"
#include "../../include/gargantua_constants.h"

namespace gg {

// A named NVTX range for the scope (the pass entry points and the server's
// scheduling steps), so a profiler's timeline shows which call launched
// what. NVTX is header-only and costs a branch when no tool is attached.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

// Record `status` with a sentence for gg_last_error() and return it.
int fail(int status, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

// Map a CUDA error to GG_ERR_DEVICE (or GG_ERR_OUT_OF_MEMORY), recording
// where it happened; returns GG_OK for cudaSuccess.
int cuda_status(cudaError_t e, const char* what);

#define GG_CUDA(call, what)                               \
    do {                                                  \
        int gg_s_ = ::gg::cuda_status((call), (what));    \
        if (gg_s_ != GG_OK) return gg_s_;                 \
    } while (0)

#define GG_CHECK(expr)                 \
    do {                               \
        int gg_s_ = (expr);            \
        if (gg_s_ != GG_OK) return gg_s_; \
    } while (0)

// Check the last kernel launch.
int launch_status(const char* what);

}  // namespace gg

// The sweep tables of one camera radius (DeflectionTables.swift:29-76):
// device pointers to SWEEP_TABLE_SIZE floats each plus the bounds the march
// reads them with.
struct gg_sweep {
    float* camera = nullptr;
    float* sky = nullptr;
    double camera_radius = 0.0;
    float camera_max_b = 0.0f;
    float sky_max_b = 0.0f;
};

struct gg_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t budget = 0;
    uint64_t used = 0;
    int sm_count = 0;
    std::recursive_mutex mu;

    // Fixed sphere table (SWEEP_TABLE_SIZE floats) and its bounds.
    float* sphere_table = nullptr;
    float sphere_max_b = 0.0f;        // tangential b at the entry radius (29)
    float sphere_table_max_b = 0.0f;  // tangential b at the sphere (30)
    // Camera-dependent tables for the plain per-call path.
    gg_sweep sweep;

    // Blackbody colours: BLACKBODY_TABLE_SIZE float4 (rgb from half, 1).
    float4* blackbody = nullptr;

    // Small per-call device scratch: counters and the probe buffers.
    MarchCounters* counters = nullptr;
    unsigned long long* stats = nullptr;  // last march: ray steps, samples, FP64 rays, spare
    int fp64_policy = 0;  // gg_fp64_policy of gg_march and gg_probe
    uint32_t march_block_w = MARCH_THREADGROUP_WIDTH;   // image kernel block (gg_context_set_march_block)
    uint32_t march_block_h = MARCH_THREADGROUP_HEIGHT;
    void* probe_buffer = nullptr;
    uint64_t probe_capacity = 0;  // bytes
    uint32_t* flagged = nullptr;  // FP64 re-integration list
    uint64_t flagged_capacity = 0;  // entries
};

namespace gg {

// Budgeted device allocation: refuses with GG_ERR_OVER_BUDGET before
// calling cudaMalloc when the context would exceed its budget
// (Budget.swift:17-21).
int device_alloc(gg_context* ctx, uint64_t bytes, void** out, const char* what);
void device_free(gg_context* ctx, void* ptr, uint64_t bytes);
int ensure_capacity(gg_context* ctx, void** ptr, uint64_t* capacity, uint64_t bytes, const char* what);

// Host-side table construction (FP64, then rounded), the work
// ParticleSystem.init does on the host (ParticleSystem.swift:23-47).
void radial_inverse_cdf(int count, int resolution, double* table);
void power_law_inverse_cdf(int count, double exponent, double* table);
void blackbody_table(int count, double tmin, double tmax, double* rgb);
double disk_shape(double r, double floor);

// Sweep tables (tables.cu).
int sweep_init(gg_context* ctx);
int sweep_build(gg_context* ctx, cudaStream_t stream, double camera_radius, gg_sweep* out);
// The camera and sky tables of `count` camera radii, one launch per 128.
int sweep_build_batch(gg_context* ctx, cudaStream_t stream, const double* camera_radius, gg_sweep* const* out,
                      int count);
void sweep_apply(const gg_context* ctx, const gg_sweep* sweep, MarchUniforms* u);

// Blackbody table on the device (present.cu).
int blackbody_init(gg_context* ctx);

}  // namespace gg

struct gg_particles {
    gg_context* ctx = nullptr;
    uint32_t count = 0;
    uint32_t first_index = 0;  // global index of slot 0 (shards of a larger system)
    float* profile_cdf = nullptr;   // optional second seeding table (gg_particles_seed_profile)
    float profile_fraction = 0.0f;  // share of seeded particles drawn from it
    uint64_t seed = 0;
    uint32_t potential = PotentialPaczynskiWiita;
    float4* pos = nullptr;  // x, y, z, temperature
    float4* vel = nullptr;  // vx, vy, vz, respawns (bits)
    float* inverse_cdf = nullptr;
    SimUniforms uniforms{};
};

struct gg_volume {
    gg_context* ctx = nullptr;
    uint32_t size = 0;
    uint32_t* sums = nullptr;  // 6 words per voxel: energy, energyT, px, py, pz, mass
    cudaArray_t emission = nullptr;
    cudaArray_t velocity = nullptr;
    cudaTextureObject_t emission_tex = 0;
    cudaTextureObject_t velocity_tex = 0;
    cudaSurfaceObject_t emission_surf = 0;
    cudaSurfaceObject_t velocity_surf = 0;
    uint64_t bytes = 0;
    // Splat shape per deposit mode ([0] stochastic, [1] exact): brick edge B
    // (0: direct global atomics) and particles per deposit work item.
    uint32_t brick_edge[2] = {0u, 8u};    // [stochastic, exact]; set per size by gg_volume_create
    uint32_t brick_chunk[2] = {0u, 1024u};
    void* brick_scratch = nullptr;  // counts, cursor, offsets, items, sorted slots, keys
    uint64_t brick_scratch_capacity = 0;
    bool brick_counts_zero = false;  // the counts region holds zeros (the count pass re-zeroes it)
    // Other ranks' sums opened from their IPC handles (gg_volume_attach_peers):
    // every deposit word is added into each of them as well.
    uint32_t* peer_sums[GG_MAX_PEERS] = {};
    uint32_t peers = 0;
};

struct gg_targets {
    gg_context* ctx = nullptr;
    uint32_t width = 0, height = 0;
    ushort4* color = nullptr;
    ushort4* debug = nullptr;
    float* depth = nullptr;
    ushort2* motion = nullptr;
    uint64_t bytes = 0;
    uchar4* srgb = nullptr;  // gg_tonemap's device output, allocated by its first call and kept
};

struct gg_bake {
    gg_context* ctx = nullptr;
    uint32_t width = 0, height = 0;
    ushort4* samples = nullptr;
    BakedRay* headers = nullptr;
    uint32_t* overflow = nullptr;
    uint64_t bytes = 0;
};
