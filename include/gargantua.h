/*
 * gargantua-b200: the per-frame compute of gargantua (particle sim,
 * cloud-in-cell splat and resolve, null-geodesic march, probes, bake and
 * walk, tone curve) as sm_100a kernels behind a plain C interface.
 *
 * The interface replaces the Metal passes a gargantua host encodes
 * (the Swift files of Sources/Gargantua/Passes) one for one. Structs are the
 * ShaderTypes.h layouts (gargantua_types.h). Every handle is opaque and owned
 * by the library; device state (particles, volumes, tables, targets) stays
 * resident between calls. Host pointers passed in are caller-owned and are
 * only read or written during the call.
 *
 * Errors: every entry point returns a gg_status. Nothing inside the library
 * exits or traps; gg_last_error() gives one sentence about the most recent
 * failure on the calling thread. A host maps GG_ERR_INVALID_ARGUMENT to its
 * usage exit (64) and every other failure to its operational exit (2), as
 * Sources/Gargantua/Exit.swift:5-18 does.
 *
 * Threading: calls on one context are serialised by a mutex inside the
 * library; all device work of a context is ordered on the context's stream.
 */
#ifndef GARGANTUA_H
#define GARGANTUA_H

#include <stdint.h>
#include "gargantua_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define GG_API __attribute__((visibility("default")))

typedef enum {
    GG_OK = 0,
    GG_ERR_INVALID_ARGUMENT = 1,
    GG_ERR_OUT_OF_MEMORY = 2,
    GG_ERR_OVER_BUDGET = 3,
    GG_ERR_DEVICE = 4,
    GG_ERR_TIMEOUT = 5,
    GG_ERR_NOT_READY = 6,
    GG_ERR_NO_DEVICE = 7,
    GG_ERR_UNSUPPORTED = 8,
    GG_ERR_CANCELLED = 9     /* a served request withdrawn by gg_server_cancel */
} gg_status;

typedef struct gg_context gg_context;
typedef struct gg_particles gg_particles;
typedef struct gg_volume gg_volume;
typedef struct gg_targets gg_targets;
typedef struct gg_bake gg_bake;
typedef struct gg_server gg_server;

/* ---------------------------------------------------------------- context */

/* Library version string. Replaces Program.version (Program.swift:5). */
GG_API const char* gg_version(void);

/* The most recent failure on this thread as one sentence, "" if none. */
GG_API const char* gg_last_error(void);

/* Name of a status code. */
GG_API const char* gg_status_name(int status);

/* Open CUDA device `device` with a memory budget. budget_bytes == 0 applies
 * the reference's rule, min(MEMORY_BUDGET_FRACTION of device memory,
 * MEMORY_BUDGET_CAP_BYTES) (Budget.swift:6-22); any allocation that would
 * exceed the budget is refused with GG_ERR_OVER_BUDGET before it is made.
 * Replaces GpuContext.init (Gpu/GpuContext.swift:7-26) and MemoryBudget. */
GG_API int gg_context_create(int device, uint64_t budget_bytes, gg_context** out);
GG_API void gg_context_destroy(gg_context* ctx);

/* Block until every call made on the context has finished on the device. A
 * device fault reported here is GG_ERR_DEVICE (GpuContext.swift:75-87). */
GG_API int gg_context_synchronize(gg_context* ctx);

/* Budget accounting: bytes the context may allocate and bytes it holds. */
GG_API int gg_context_memory(gg_context* ctx, uint64_t* budget, uint64_t* used);

/* The context's CUDA stream (a cudaStream_t), for hosts that order their own
 * device work with the library's. */
GG_API void* gg_context_stream(gg_context* ctx);

/* Page-locked host memory (cudaHostAlloc, usable with any device) for the
 * host buffers the library copies into or out of, such as served requests'
 * outputs: those copies run at the link's rate, where pageable memory goes
 * through the driver's staging (a 1920x1080 result: 0.3 against 1.7 to 4.5
 * ms on a B200). Not counted in the context's budget. gg_host_free releases
 * a block gg_host_alloc returned (NULL is ignored). No reference counterpart:
 * the Metal host's buffers are shared with the GPU. */
GG_API int gg_host_alloc(gg_context* ctx, uint64_t bytes, void** out);
GG_API void gg_host_free(void* p);

/* Copy the blackbody colour table the kernels sample (BLACKBODY_TABLE_SIZE
 * float4: rgb rounded through half as the reference's rgba16f table, 1) to
 * the host. The table is Blackbody.table (Blackbody.swift:80-86). */
GG_API int gg_context_blackbody(gg_context* ctx, float* rgba, uint32_t count);

/* -------------------------------------------------------------- particles */

/* A particle system of `count` particles in device memory, seeded from
 * `seed`, with its inverse-CDF seeding table (1024 entries, built in FP64 on
 * the host and rounded to float, DiskModel.swift:54-78) and blackbody colour
 * table (256 entries, Blackbody.swift:74-82). Replaces ParticleSystem.init
 * (Sim/ParticleSystem.swift:17-48). potential is PotentialNewtonian or
 * PotentialPaczynskiWiita. */
GG_API int gg_particles_create(gg_context* ctx, uint32_t count, uint64_t seed, uint32_t potential,
                               gg_particles** out);
GG_API void gg_particles_destroy(gg_particles* ps);

/* A shard of a larger particle system: `count` particles whose global
 * indices start at first_index. The counter-based hash is keyed on the
 * global index (sim.metal:7-8, splat.metal:75), so shards on several GPUs
 * reproduce the unsharded system slot for slot and their splat grids sum to
 * the unsharded grid exactly. No reference counterpart (one GPU there). */
GG_API int gg_particles_create_shard(gg_context* ctx, uint32_t count, uint32_t first_index, uint64_t seed,
                                     uint32_t potential, gg_particles** out);

/* Seed a share of the particles from a second radial profile, a surface
 * density Sigma ~ r^-exponent on [R_ISCO, R_DISK_OUTER] (rising toward the
 * ISCO for exponent > 0): at event 0, a particle whose spare hash word (the
 * third word of the second pcg4d draw) is below `fraction` reads its radius
 * from this profile's inverse-CDF table instead of the steady disk's. The
 * max preset's contention workload (70 % from a power law near r = 6) has no
 * reference counterpart; fraction 0 restores the reference's seeding. Call
 * before gg_particles_seed. */
GG_API int gg_particles_seed_profile(gg_particles* ps, float fraction, float exponent);

/* Copy the profile's INVERSE_CDF_COUNT-entry table (FP64 rounded to float). */
GG_API int gg_particles_profile_table(gg_particles* ps, float* out, uint32_t count);

/* The uniforms the particle kernels run with (ParticleSystem.swift:59-70). */
GG_API int gg_particles_uniforms(gg_particles* ps, SimUniforms* out);

/* Seed every particle from the steady disk profile, event 0. Replaces
 * SimPass.encodeSeed -> seedParticles (SimPass.swift:24-26, sim.metal:36-42). */
GG_API int gg_particles_seed(gg_particles* ps);

/* Advance `dispatches` dispatches of SIM_SUBSTEPS substeps each. Replaces
 * SimPass.encodeStep -> stepParticles (SimPass.swift:28-31, sim.metal:44-79). */
GG_API int gg_particles_step(gg_particles* ps, uint32_t dispatches);

/* Copy the state out as ShaderTypes Particle records (32 bytes each) into a
 * host array of `count` entries (count must equal the system's count).
 * Replaces Validate.readback (Validate.swift:88-100). */
GG_API int gg_particles_read(gg_particles* ps, Particle* out, uint32_t count);

/* Replace the device state with `count` host Particle records. */
GG_API int gg_particles_write(gg_particles* ps, const Particle* in, uint32_t count);

/* 64-bit FNV-1a over the AoS bytes of the state (Validate.swift:378-387). */
GG_API int gg_particles_checksum(gg_particles* ps, uint64_t* out);

/* The float inverse-CDF table the seeding reads (1024 floats). */
GG_API int gg_particles_inverse_cdf(gg_particles* ps, float* out, uint32_t count);

/* ----------------------------------------------------------------- volume */

/* A size^3 volume: six 32-bit fixed-point sums per voxel and two rgba16f 3-D
 * textures (emission, velocity). Replaces Volume.init (Gpu/Volume.swift:14-30).
 * The sums start zeroed. */
GG_API int gg_volume_create(gg_context* ctx, uint32_t size, gg_volume** out);
GG_API void gg_volume_destroy(gg_volume* vol);

/* Bin the particles with cloud-in-cell fixed-point atomics, resolve the sums
 * into the two half-precision textures, and zero the sums, in one call.
 * u->volumeSize and u->particleCount must match the handles. Replaces
 * SplatPass.encode (SplatPass.swift:71-76: encodeBin, encodeResolve,
 * Volume.encodeClear). */
GG_API int gg_splat(gg_particles* ps, gg_volume* vol, const SplatUniforms* u);

/* The binning alone, leaving the sums in place (SplatPass.encodeBin,
 * SplatPass.swift:34-49). */
GG_API int gg_splat_bin(gg_particles* ps, gg_volume* vol, const SplatUniforms* u);

/* The resolve of the current sums into the textures, then zeroing the sums
 * (SplatPass.encodeResolve + Volume.encodeClear, SplatPass.swift:52-69,
 * Volume.swift:34-43). */
GG_API int gg_splat_resolve(gg_volume* vol, const SplatUniforms* u, const gg_particles* ps);

/* Zero the sums (Volume.encodeClear). */
GG_API int gg_volume_clear(gg_volume* vol);

/* Copy the sums to host arrays in the reference's buffer layouts:
 * emission u32[2 n^3] (energy, energy*T pairs), momentum i32[3 n^3], mass
 * u32[n^3], voxel index (z n + y) n + x (splat.metal:21-23). */
GG_API int gg_volume_read_sums(gg_volume* vol, uint32_t* emission, int32_t* momentum, uint32_t* mass);

/* Replace the sums with host arrays in the same layouts, e.g. after summing
 * the grids of several GPUs' particle shards. */
GG_API int gg_volume_write_sums(gg_volume* vol, const uint32_t* emission, const int32_t* momentum, const uint32_t* mass);

/* How gg_splat_bin deposits, per mode (exact != 0: the exact eight-corner
 * deposit, else the stochastic one). brick_edge 0: one thread per particle
 * adding into the sums with global atomics. brick_edge 4, 8 or 16: the grid
 * is cut into bricks of that edge, particles are sorted by brick, and each
 * work item of `chunk` particles of one brick deposits into a shared-memory
 * copy of its (edge+1)^3 voxels before adding the non-zero words to the
 * sums. Every shape gives the same sums bit for bit. Defaults: exact, edge
 * 16 with chunks of 4096 (96^3), 8192 (up to 128^3) and 16384 particles
 * (larger), edge 8 with chunks of 1024 below 96^3; stochastic, edge 0. */
GG_API int gg_volume_splat_shape(gg_volume* vol, int exact, uint32_t brick_edge, uint32_t chunk);

/* Time gg_splat_bin under each shape on these particles (u->exactDeposit
 * selects the mode) and keep the fastest for that mode. Outputs (each may be
 * NULL): the chosen edge and chunk and its time in ms. The sums are left
 * zeroed. */
GG_API int gg_splat_autotune(gg_particles* ps, gg_volume* vol, const SplatUniforms* u, uint32_t* brick_edge,
                             uint32_t* chunk, float* best_ms);

/* Device address and length (in 32-bit words) of the volume's sums: one
 * record of six words per voxel (energy, energy*T, momentum x/y/z, mass),
 * voxel index (z n + y) n + x. Every word is a two's-complement sum, so the
 * grids of several GPUs' particle shards combine with one element-wise
 * integer all-reduce (sum) over this buffer, done on the context's stream
 * (gg_context_stream) between gg_splat_bin and gg_splat_resolve. Valid until
 * the volume is destroyed. */
GG_API int gg_volume_sums(gg_volume* vol, void** device_words, uint64_t* words);

/* The all-reduce done by the deposit itself, over peer memory. Each rank
 * (one process per GPU) exports its volume's sums as a CUDA IPC handle
 * (GG_IPC_HANDLE_BYTES bytes) and attaches the other ranks' handles, volumes
 * of the same size; from then on gg_splat_bin adds every deposit word into
 * its own sums and into each attached rank's, with peer atomics over
 * NVLink, so once every rank's bin has finished each grid holds the sum of
 * all shards, bit for bit as the integer all-reduce gives it, with no
 * separate collective. The ranks order themselves on the host: every
 * rank's previous resolve (which clears its sums) finishes before any rank
 * bins, every bin finishes before any rank resolves, and every rank has
 * detached (count 0, or destroyed its volume) before any rank destroys the
 * volume the others have attached. At most
 * GG_MAX_PEERS peers; count 0 detaches. No reference counterpart: the
 * reference renders on one GPU. */
#define GG_IPC_HANDLE_BYTES 64
#define GG_MAX_PEERS 7
GG_API int gg_volume_ipc_handle(gg_volume* vol, void* handle);
GG_API int gg_volume_attach_peers(gg_volume* vol, const void* handles, uint32_t count);

/* Copy the resolved textures to host arrays of n^3 half4 (IEEE binary16 bit
 * patterns, x fastest). Replaces Validate.readVolume (Validate.swift:204-230). */
GG_API int gg_volume_read(gg_volume* vol, uint16_t* emission_half4, uint16_t* velocity_half4);

/* Upload host half4 textures (n^3 each), e.g. an analytic field for tests. */
GG_API int gg_volume_write(gg_volume* vol, const uint16_t* emission_half4, const uint16_t* velocity_half4);

/* ------------------------------------------------------ deflection tables */

/* Enable the sphere jump in `inout` for a camera at `camera_radius`: builds
 * the camera and sky sweep tables for that radius in FP64 on the device (the
 * sphere table is built once per context), and fills sphereRadius,
 * cameraRadius, sphereMaxB, sphereTableMaxB, cameraMaxB, skyMinB, skyMaxB.
 * Replaces DeflectionTables.update + apply (DeflectionTables.swift:57-76). */
GG_API int gg_tables_update(gg_context* ctx, float camera_radius, MarchUniforms* inout);

/* Copy the three float tables (SWEEP_TABLE_SIZE entries each) to the host;
 * any pointer may be NULL. */
GG_API int gg_tables_read(gg_context* ctx, float* sphere, float* camera, float* sky);

/* ------------------------------------------------------------------ march */

/* Render targets of width x height: colour rgba16f, debug rgba16f (drift,
 * steps, outcome, 1), depth r32f, motion rg16f. Replaces
 * MarchPass.makeTargets (MarchPass.swift:42-50). */
GG_API int gg_targets_create(gg_context* ctx, uint32_t width, uint32_t height, gg_targets** out);
GG_API void gg_targets_destroy(gg_targets* t);

/* Copy targets to host arrays (any pointer may be NULL): colour and debug
 * as width*height half4, depth as floats, motion as half2. */
GG_API int gg_targets_read(gg_targets* t, uint16_t* color_half4, uint16_t* debug_half4, float* depth,
                           uint16_t* motion_half2);

/* Load colour and/or debug pixels (width x height half4, NULL to skip) into
 * the targets, e.g. a served request's output before gg_tonemap. */
GG_API int gg_targets_write(gg_targets* t, const uint16_t* color_half4, const uint16_t* debug_half4);

/* Precision policy of the march. Every policy takes the reference's steps
 * (march.metal:51-184: the same RK4, step policy and termination), so ray
 * step counts agree; they differ in how each step's arithmetic runs. */
typedef enum {
    /* FP32, direct state update, with this library's step arithmetic (one
     * reciprocal per derivative, the RK4 stages as a loop, series sin/cos). */
    GG_PRECISION_PLAIN = 0,
    /* The same FP32 step arithmetic with compensated (TwoSum) accumulation
     * of the state update, and rays whose drift exceeds the budget inside
     * r < 4 re-integrated in FP64. */
    GG_PRECISION_COMPENSATED = 1,
    /* FP32 with the reference kernel's arithmetic as written: four
     * derivative calls per step with their divides, library sin/cos
     * (Geodesic.h:42-59, Kerr.h:63-99). The per-request baseline. */
    GG_PRECISION_PLAIN_AS_WRITTEN = 2,
    /* GG_PRECISION_COMPENSATED with the Hamiltonian-constraint
     * renormalisation after every step: a Schwarzschild state is put back on
     * the null cone with its starting E and L (phiDot from L, rDot and vDot
     * from E and the constraint, in double); a Kerr state gets |p_r| from
     * 2 Sigma H = 0 (Kerr.h:39-50). The drift reported is the largest drift
     * of a state before its projection, the integrator's per-step error
     * (after it the gauges read roundoff by construction). gg_march and
     * gg_probe; no reference counterpart. */
    GG_PRECISION_RENORMALISED = 3
} gg_precision;

/* Which flagged rays the compensated march re-integrates in FP64. A ray is
 * flagged when its drift exceeds the budget after it passed inside r < 4.
 * A captured ray's drift is dominated by the integrator's truncation error
 * next to the horizon, which FP64 does not change: on a 480x270 Kerr
 * (a = 0.9) still, 1,326 of 1,409 flagged rays were captured and 1,394 of
 * the 1,409 were still over the budget after FP64, with the same median
 * drift (2e-2). */
typedef enum {
    /* Flagged rays that escape or reach the step cap (the default). */
    GG_FP64_ESCAPING = 0,
    /* Every flagged ray, captured ones included. */
    GG_FP64_ALL_FLAGGED = 1
} gg_fp64_policy;

/* Thread block of the image kernels (gg_march, gg_march_compensated_noalloc
 * and the serial serving modes) on this context: width x height pixels,
 * 32..256 threads in whole warps. Default 8x8, the reference's threadgroup
 * (MarchPass.swift:101). */
GG_API int gg_context_set_march_block(gg_context* ctx, uint32_t width, uint32_t height);

/* The policy gg_march and gg_probe use on this context. */
GG_API int gg_context_set_fp64_policy(gg_context* ctx, int policy);

/* March one image (or a tile of it: u->tileOrigin selects the tile, the
 * targets' size is the tile size) through the volume. vol may be NULL for a
 * march with no gas. counters may be NULL; when given it is overwritten with
 * this call's counters. Replaces MarchPass.encodeImage -> marchImage
 * (MarchPass.swift:103-124, march.metal:194-288). `blackbody` colours come
 * from the particle system's table; ps may be NULL (stars use the same table,
 * built on first use). */
GG_API int gg_march(gg_context* ctx, const gg_volume* vol, const MarchUniforms* u, gg_targets* targets,
                    int precision, MarchCounters* counters);

/* Totals of the most recent gg_march on this context: RK4 ray steps (the
 * `steps` each ray reports, march.metal:70, summed), in-slab gather samples,
 * and rays re-integrated in FP64. Any pointer may be NULL. */
GG_API int gg_march_stats(gg_context* ctx, uint64_t* ray_steps, uint64_t* samples, uint64_t* fp64_rays);

/* Integrate `count` probe rays with no gather. Host arrays in and out.
 * Replaces MarchPass.encodeProbes -> probeRays (MarchPass.swift:148-168,
 * march.metal:290-341) and Probes.run (Probes.swift:26-43). */
GG_API int gg_probe(gg_context* ctx, const MarchUniforms* u, const RayProbe* probes, RayProbeResult* results,
                    uint32_t count, int precision);

/* The capture boundary (the shadow's edge) along a one-parameter family of
 * rays, bisected in FP64 on the device: rays leave `origin` along base + t
 * axis for t in [lo, hi]; each round marches rays_per_round FP64 rays at the
 * centres of equal cells of the bracket and keeps the cell pair after the
 * last ray whose outcome (captured or not) matches the first ray's, so each
 * round narrows the bracket by rays_per_round / 2 or more; isolated rays of
 * the other outcome before it (a captured ray that one step carries across
 * the horizon can end as an escape, as in the reference's integrator) do
 * not count. A ray just past that last ray which reaches the step cap orbits
 * on the boundary and ends the search there (the rule of
 * Validate.swift:125-150). u supplies spin, step policy and escape radius.
 * *t_out: the boundary's t. */
GG_API int gg_capture_boundary(gg_context* ctx, const MarchUniforms* u, const double origin[3], const double base[3],
                               const double axis[3], double lo, double hi, uint32_t rays_per_round, uint32_t rounds,
                               double* t_out);

/* Largest target, in pixels, gg_march_compensated_noalloc serves. */
#define NOALLOC_MAX_PIXELS 2097152u

/* The compensated march of gg_march (GG_PRECISION_COMPENSATED) for callers
 * that must not allocate device memory once they run: hosts whose device
 * memory is handed to their own pool up front, frame loops that cannot
 * absorb cudaMalloc/cudaFree (cudaFree synchronises the device) or an
 * allocation failure mid-frame, plugins inside a program that owns the
 * memory budget. It allocates nothing: the FP64 re-integration list lives in
 * a fixed device array of NOALLOC_MAX_PIXELS + 64 words (about 8 MiB) that
 * every GPU loading the library holds until exit, and targets larger than
 * NOALLOC_MAX_PIXELS are refused with GG_ERR_INVALID_ARGUMENT. The caller
 * passes inputs and outputs as for gg_march (sweep tables, when enabled,
 * come from an earlier gg_tables_update). Each call looks up the array's
 * device address (the first lookup on a device loads the array: make that
 * first call before any stream capture; a call during a capture of the
 * context's stream reuses the last address looked up on the device).
 * All calls on a device share the array: calls whose work overlaps on the
 * GPU race, so serialise them. This entry point has no counterpart in the
 * reference, whose host allocates every buffer up front. */
GG_API int gg_march_compensated_noalloc(gg_context* ctx, const gg_volume* vol, const MarchUniforms* u,
                                        gg_targets* targets, MarchCounters* counters);

/* ------------------------------------------------------------ bake / walk */

/* Bake storage for width x height rays: BAKE_SAMPLES half4 samples per ray
 * plus a BakedRay header per ray (BakePass.swift:31-38). */
GG_API int gg_bake_create(gg_context* ctx, uint32_t width, uint32_t height, gg_bake** out);
GG_API void gg_bake_destroy(gg_bake* b);

/* Bake rows [row_begin, row_end) (u->bakeSpacing, u->bakeCapacity and the
 * still policy in u->geodesic). Rays over the sample capacity add to the
 * overflow count. Replaces BakePass.encodeBakeChunk -> bakeRays
 * (BakePass.swift:55-76, bake.metal:17-92). */
GG_API int gg_bake_rows(gg_bake* b, const MarchUniforms* u, uint32_t row_begin, uint32_t row_end);

/* Rays of the current bake that overflowed the sample budget; reset with
 * reset != 0 (BakePass.swift:47-48, 57-60). */
GG_API int gg_bake_overflow(gg_bake* b, uint32_t* count, int reset);

/* Walk the stored samples through the volume into targets (same size as
 * the bake). Replaces BakePass.encodeWalk -> walkRays (BakePass.swift:86-102,
 * bake.metal:94-144). */
GG_API int gg_walk(gg_bake* b, const gg_volume* vol, const MarchUniforms* u, gg_targets* targets);

/* Copy the baked samples (width*height*BAKE_SAMPLES half4) and headers to
 * the host; either pointer may be NULL. */
GG_API int gg_bake_read(gg_bake* b, uint16_t* samples_half4, BakedRay* headers);

/* ------------------------------------------------------------------ present */

/* Tone map the colour target (exposure x HDR -> PBR Neutral -> sRGB
 * encoding) into width*height*4 bytes of 8-bit sRGB RGBA on the host, or, with
 * u->debugView != 0, the drift heat map of the debug target. Replaces the
 * present pass's tonemapFragment (present.metal:22-58) with a headless
 * buffer in place of the drawable. The first call on a targets handle
 * allocates its 4 bytes per pixel of device output, kept until
 * gg_targets_destroy. */
GG_API int gg_tonemap(gg_targets* t, const PresentUniforms* u, uint8_t* rgba8);

/* Write an 8-bit RGBA image as a PNG file (zlib-compressed, no filter).
 * Replaces Capture.writePNG (App/Capture.swift:80-94). */
GG_API int gg_write_png(const char* path, const uint8_t* rgba8, uint32_t width, uint32_t height);

/* ---------------------------------------------------------------- serving */

/* One still request: an orbit camera (Camera.swift:15-33: azimuth,
 * elevation, distance, vertical field of view in radians), an image size, a
 * step budget (256 selects the interactive policy, anything above the still
 * policy, Schwarzschild.swift:167-172), a spin (0 renders Schwarzschild with
 * the sphere jump, > 0 Kerr) and a star seed. The server writes width*height
 * rgba16f pixels into `output` (host memory the caller keeps alive until the
 * request completes; page-locked memory, cudaHostAlloc, copies at the link's
 * rate: a 1920x1080 result's 16.6 MB took 0.3 ms into page-locked memory and
 * 1.7 to 4.5 ms into pageable memory on a B200) and, when debug_output is not
 * NULL, the debug target
 * (drift, steps, outcome, 1). Kerr cameras beyond R_ESCAPE escape at
 * camera distance + 10 instead of R_ESCAPE, so rays start inside the scene.
 * Replaces a `--still` render (Still.swift:9-99) as a served unit of work. */
typedef struct {
    float azimuth, elevation, distance, fov_y;
    uint32_t width, height;
    uint32_t step_cap;
    float spin;
    uint32_t star_seed;
    uint32_t flags; /* GG_REQUEST_* */
    uint16_t* output;
    uint16_t* debug_output;
    /* The volume this request marches through; NULL: the server's. It must
     * stay unchanged (no splat into it) until the request is waited for:
     * a sequence advances its own particles and volume between frames. */
    const gg_volume* volume;
} gg_request;

#define GG_REQUEST_NO_STARS 1u   /* starBrightness 0 */
#define GG_REQUEST_NO_REDSHIFT 2u
/* The bake strategy (bake.metal:17-144, BakePass.swift): the request's rays
 * are integrated once at its step policy with their in-slab points stored
 * (BAKE_SAMPLES half4 and a 16-byte header per pixel, about 400 MB at
 * 960x540, counted in the request's admission footprint), then walked
 * through its volume into the output; the debug output stays zero.
 * Schwarzschild only (GG_ERR_UNSUPPORTED for spin > 0). */
#define GG_REQUEST_BAKE 4u

/* Per-request outcome, times in seconds on the server's monotonic clock. */
typedef struct {
    double submitted, admitted, finished;
    uint64_t ray_steps, samples, fp64_rays;
    MarchCounters counters;
    int status;
} gg_request_result;

typedef enum {
    /* Continuous batching: requests are admitted as device memory frees up,
     * their rays packed across requests into persistent, work-stealing
     * launches replayed from CUDA graphs, compensated FP32 with FP64
     * re-integration of flagged rays. */
    GG_SERVE_BATCHED = 0,
    /* One request at a time through the plain FP32 image kernel
     * (gg_march with GG_PRECISION_PLAIN): what batching adds over
     * per-request launches of the same step arithmetic. */
    GG_SERVE_SERIAL_PLAIN = 1,
    /* One request at a time through the image kernel with the reference's
     * arithmetic (GG_PRECISION_PLAIN_AS_WRITTEN): the reference's
     * per-request march. */
    GG_SERVE_SERIAL_PLAIN_AS_WRITTEN = 2
} gg_serve_mode;

/* How the persistent serve kernels hand rays to lanes. Both steal chunks of
 * rays with one atomic per warp and give the same pixels. */
typedef enum {
    /* A warp takes a chunk, runs each lane's ray to its end, then takes the
     * next: no warp-level work inside the step loop (the default, faster
     * on B200 on the served mix). */
    GG_SCHEDULE_CHUNKS = 0,
    /* Lanes that finish are refilled with new rays between rounds of
     * steps_per_round steps once refill_idle lanes are idle. */
    GG_SCHEDULE_LANE_REFILL = 1
} gg_schedule;

typedef struct {
    int mode;                  /* gg_serve_mode */
    uint64_t memory_bytes;     /* device memory for admitted requests' targets; 0: a quarter of the budget left */
    uint32_t wave_rays;        /* rays packed into one persistent launch; 0: 4 Mi */
    uint32_t chunk_rays;       /* rays per work-stealing chunk; 0: 32, one per lane of a warp */
    uint32_t max_waves_in_flight; /* 0: 6; at most 8 */
    uint32_t fp64_policy;      /* gg_fp64_policy */
    uint32_t steps_per_round;  /* lane refill: RK4 steps a warp takes between refills of idle lanes; 0: 8 */
    uint32_t refill_idle;      /* lane refill: idle lanes of a warp that trigger a refill; 0: 8 */
    uint32_t schedule;         /* gg_schedule */
} gg_server_config;

/* A server over a resident volume (vol may be NULL: no gas). */
GG_API int gg_server_create(gg_context* ctx, const gg_volume* vol, const gg_server_config* config, gg_server** out);

/* Stop accepting work, finish what was submitted, release everything. */
GG_API void gg_server_destroy(gg_server* s);

/* Queue a request; *ticket identifies it. Returns GG_ERR_OVER_BUDGET when
 * the request alone can never fit the server's memory. */
GG_API int gg_server_submit(gg_server* s, const gg_request* req, uint64_t* ticket);

/* *done = 1 once the request's pixels are in its host buffers. */
/* Failure-path test hook: the scheduler treats its next device call as
 * failed with `status` (non-zero), exactly as it treats a real device error:
 * it stops, every waiter and every later call gets the status, and
 * gg_server_destroy still releases everything. Nothing fails on the device;
 * the context stays usable. */
GG_API int gg_server_inject_fault(gg_server* s, int status);

GG_API int gg_server_poll(gg_server* s, uint64_t ticket, int* done);

/* Withdraw a request that is still waiting for admission: it never runs,
 * and gg_server_wait on it returns GG_ERR_CANCELLED (and forgets the
 * ticket). A request already admitted has its rays on the device and
 * completes: GG_ERR_NOT_READY, nothing changes. No reference counterpart. */
GG_API int gg_server_cancel(gg_server* s, uint64_t ticket);

/* Block until the request completes or timeout_s passes (GG_ERR_TIMEOUT);
 * on success fills *result (may be NULL) and forgets the ticket. */
GG_API int gg_server_wait(gg_server* s, uint64_t ticket, double timeout_s, gg_request_result* result);

/* Totals since creation or the last reset: requests completed, ray steps,
 * kernel launches (each wave's two persistent kernels and its FP64 pass,
 * one sweep-table build per admission round of Schwarzschild requests, two
 * kernels per bake request, or one image kernel
 * per request in the plain modes), device-busy
 * seconds (union of the launches' CUDA-event intervals) and device span
 * seconds (first launch start to last launch end, on the device clock).
 * reset != 0 zeroes them after reading. Any output pointer may be NULL. */
GG_API int gg_server_totals(gg_server* s, int reset, uint64_t* requests, uint64_t* ray_steps, uint64_t* launches,
                            double* busy_seconds, double* span_seconds);

/* ------------------------------------------------------------ measurement */

/* FP32 throughput of this device measured with a dependent-FMA kernel over
 * every SM (each FMA counted as two flops): the peak the march's roofline is
 * quoted against. */
GG_API int gg_measure_fp32_peak(gg_context* ctx, double* tflops);

/* The device's rate, in G adds/s, of relaxed 32-bit global atomic adds into
 * a grid of `records` six-word records (the splat's sums layout) at
 * uniformly scattered records: the denominator of the splat's roofline. */
GG_API int gg_measure_atomic_peak(gg_context* ctx, uint32_t records, double* gatomics);

/* The same rate, in G adds/s, for 32-bit atomic adds into a shared-memory
 * tile of 9^3 six-word records padded to seven words, the brick deposit's
 * layout (the brick splat's tile at edge 8). */
GG_API int gg_measure_shared_atomic_peak(gg_context* ctx, double* gatomics);

#ifdef __cplusplus
}
#endif

#endif
