// Splat pass (splat.metal:16-120): cloud-in-cell deposit of every particle
// into six 32-bit fixed-point sums per voxel, then a resolve of the sums into
// two rgba16f 3-D textures that also zeroes the sums for the next frame.
//
// Sums layout: one 24-byte record per voxel, interleaved (energy u32,
// energy*T u32, momentum x/y/z i32, mass u32), voxel index (z n + y) n + x.
// A corner's six atomics land in one or two 32-byte sectors, and the resolve
// reads and clears a warp's 32 records as 768 contiguous bytes.
//
// Integer sums are order-independent, so the grids are bit-exact whatever
// order the atomics arrive in, as long as each corner's fixed-point values
// are: this translation unit is built with --fmad=false and evaluates every
// float expression in the order the CPU replica (oracle/replica.c) does.
#include <vector>

#include "../../include/gargantua_detmath.h"
#include "common.cuh"
#include "runtime.h"

namespace gg {

constexpr float ENERGY_FIXED = 16777216.0f;  // 2^24
constexpr float ENERGY_T_FIXED = 1048576.0f; // 2^20
constexpr float MOMENTUM_FIXED = 4096.0f;    // 2^12
constexpr float MASS_FIXED = 256.0f;         // 2^8

struct SplatArgs {
    const float4* __restrict__ pos;
    const float4* __restrict__ vel;
    uint32_t* __restrict__ sums;
    SplatUniforms u;
    uint32_t first_index;  // global index of slot 0, for the stochastic pick
};

// One corner's six fixed-point atomics (splat.metal:25-37).
__device__ __forceinline__ void deposit(uint32_t* sums, uint32_t index, float weight, float energy, float relative,
                                        float vx, float vy, float vz) {
    uint32_t fe = (uint32_t)(energy * weight * ENERGY_FIXED + 0.5f);
    uint32_t fet = (uint32_t)(energy * relative * weight * ENERGY_T_FIXED + 0.5f);
    float ms = weight * MOMENTUM_FIXED;
    int32_t mx = (int32_t)rintf(vx * ms), my = (int32_t)rintf(vy * ms), mz = (int32_t)rintf(vz * ms);
    uint32_t fm = (uint32_t)(weight * MASS_FIXED + 0.5f);
    uint32_t* rec = sums + 6u * index;
    atomicAdd(rec + 0, fe);
    atomicAdd(rec + 1, fet);
    atomicAdd(rec + 2, (uint32_t)mx);
    atomicAdd(rec + 3, (uint32_t)my);
    atomicAdd(rec + 4, (uint32_t)mz);
    atomicAdd(rec + 5, fm);
}

// splatParticles (splat.metal:44-88): positions mapped to voxel-centre
// space of a cube of half extent u.halfExtent; exact mode deposits all eight
// corners with trilinear weights, stochastic mode one corner drawn with
// those weights as probabilities from pcg4d(i, frame, seed).
__global__ void __launch_bounds__(256) bin_kernel(SplatArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const SplatUniforms& u = a.u;
    if (i >= u.particleCount) return;
    float4 p = a.pos[i];
    const uint32_t gi = a.first_index + i;
    float ux = (p.x + u.halfExtent) / (2.0f * u.halfExtent);
    float uy = (p.y + u.halfExtent) / (2.0f * u.halfExtent);
    float uz = (p.z + u.halfExtent) / (2.0f * u.halfExtent);
    if (ux < 0.0f || uy < 0.0f || uz < 0.0f || ux >= 1.0f || uy >= 1.0f || uz >= 1.0f) return;
    float4 v = a.vel[i];
    float relative = p.w / u.peakTemperature;
    float energy = relative * relative * relative * relative * u.emissionScale;
    const int n = (int)u.volumeSize;
    float gx = ux * (float)n - 0.5f, gy = uy * (float)n - 0.5f, gz = uz * (float)n - 0.5f;
    float bx = floorf(gx), by = floorf(gy), bz = floorf(gz);
    float fx = gx - bx, fy = gy - by, fz = gz - bz;
    int lx = (int)bx, ly = (int)by, lz = (int)bz;
    int hx = min(lx + 1, n - 1), hy = min(ly + 1, n - 1), hz = min(lz + 1, n - 1);
    lx = max(lx, 0);
    ly = max(ly, 0);
    lz = max(lz, 0);
    if (u.exactDeposit != 0u) {
#pragma unroll
        for (uint32_t c = 0; c < CIC_CORNERS; ++c) {
            bool bxs = (c & 1u) != 0u, bys = (c & 2u) != 0u, bzs = (c & 4u) != 0u;
            float wx = bxs ? fx : 1.0f - fx;
            float wy = bys ? fy : 1.0f - fy;
            float wz = bzs ? fz : 1.0f - fz;
            float w = wx * wy * wz;
            if (w <= 0.0f) continue;
            uint32_t index = ((uint32_t)(bzs ? hz : lz) * (uint32_t)n + (uint32_t)(bys ? hy : ly)) * (uint32_t)n +
                             (uint32_t)(bxs ? hx : lx);
            deposit(a.sums, index, w, energy, relative, v.x, v.y, v.z);
        }
    } else {
        uint4 h = pcg4d(make_uint4(gi, u.frame, u.seed.x, u.seed.y));
        int cx = unit_float(h.x) < fx ? hx : lx;
        int cy = unit_float(h.y) < fy ? hy : ly;
        int cz = unit_float(h.z) < fz ? hz : lz;
        uint32_t index = ((uint32_t)cz * (uint32_t)n + (uint32_t)cy) * (uint32_t)n + (uint32_t)cx;
        deposit(a.sums, index, 1.0f, energy, relative, v.x, v.y, v.z);
    }
}

struct ResolveArgs {
    uint32_t* __restrict__ sums;
    cudaSurfaceObject_t emission;
    cudaSurfaceObject_t velocity;
    const float4* __restrict__ blackbody;
    SplatUniforms u;
};

// Blackbody coordinate (Common.h:56-59) in double with the shared series
// log, rounded once, so the resolve's bits match the CPU replica's.
__device__ __forceinline__ float bb_coordinate_det(float temperature) {
    float t = fminf(fmaxf(temperature, BLACKBODY_T_MIN), BLACKBODY_T_MAX);
    double lo = gg_log_d((double)BLACKBODY_T_MIN);
    double hi = gg_log_d((double)BLACKBODY_T_MAX);
    return (float)((gg_log_d((double)t) - lo) / (hi - lo));
}

// resolveVolume (splat.metal:93-120) fused with the clear of the sums
// (Volume.swift:34-43): each voxel's record is read once and written back
// as zeros.
__global__ void __launch_bounds__(256) resolve_kernel(ResolveArgs a) {
    const uint32_t n = a.u.volumeSize;
    const uint64_t total = (uint64_t)n * n * n;
    uint64_t index = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= total) return;
    uint2* rec = reinterpret_cast<uint2*>(a.sums + 6u * index);
    uint2 r0 = rec[0], r1 = rec[1], r2 = rec[2];
    rec[0] = make_uint2(0u, 0u);
    rec[1] = make_uint2(0u, 0u);
    rec[2] = make_uint2(0u, 0u);
    uint32_t x = (uint32_t)(index % n);
    uint32_t y = (uint32_t)((index / n) % n);
    uint32_t z = (uint32_t)(index / ((uint64_t)n * n));
    float voxel = 2.0f * a.u.halfExtent / (float)n;
    float inverse_volume = 1.0f / (voxel * voxel * voxel);
    float count = (float)r2.y / MASS_FIXED;
    float energy = (float)r0.x / ENERGY_FIXED;
    float energy_t = (float)r0.y / ENERGY_T_FIXED;
    float tr = 0.0f, tg = 0.0f, tb = 0.0f;
    if (energy > 0.0f) {
        float mean_t = energy_t / energy * a.u.peakTemperature;
        float c = bb_coordinate_det(mean_t) * (float)BLACKBODY_TABLE_SIZE - 0.5f;
        float fl = floorf(c);
        float f = c - fl;
        int i0 = (int)fl, i1 = i0 + 1;
        i0 = min(max(i0, 0), (int)BLACKBODY_TABLE_SIZE - 1);
        i1 = min(max(i1, 0), (int)BLACKBODY_TABLE_SIZE - 1);
        float4 ta = __ldg(a.blackbody + i0), tb4 = __ldg(a.blackbody + i1);
        tr = ta.x + (tb4.x - ta.x) * f;
        tg = ta.y + (tb4.y - ta.y) * f;
        tb = ta.z + (tb4.z - ta.z) * f;
    }
    float mx = (float)(int32_t)r1.x / MOMENTUM_FIXED;
    float my = (float)(int32_t)r1.y / MOMENTUM_FIXED;
    float mz = (float)(int32_t)r2.x / MOMENTUM_FIXED;
    float density = count * inverse_volume;
    float vx = count > 0.0f ? mx / count : 0.0f;
    float vy = count > 0.0f ? my / count : 0.0f;
    float vz = count > 0.0f ? mz / count : 0.0f;
    surf3Dwrite(pack_half4(tr * energy * inverse_volume, tg * energy * inverse_volume, tb * energy * inverse_volume,
                           density),
                a.emission, x * 8, y, z);
    surf3Dwrite(pack_half4(vx, vy, vz, 1.0f), a.velocity, x * 8, y, z);
}

__global__ void clear_kernel(uint4* sums, uint64_t count16) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count16) sums[i] = make_uint4(0u, 0u, 0u, 0u);
}

}  // namespace gg

using namespace gg;

static int check_splat(const gg_particles* ps, const gg_volume* vol, const SplatUniforms* u, const char* what) {
    if (!vol || !u) return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s needs a volume and uniforms.", what);
    if (u->volumeSize != vol->size)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s: uniforms give a %u^3 volume but the volume is %u^3.", what,
                        u->volumeSize, vol->size);
    if (ps && u->particleCount != ps->count)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s: uniforms give %u particles but the system has %u.", what,
                        u->particleCount, ps->count);
    if (ps && ps->ctx != vol->ctx) return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s: handles from different contexts.", what);
    if (!(u->halfExtent > 0.0f) || !(u->peakTemperature > 0.0f))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s: halfExtent and peakTemperature must be positive.", what);
    return GG_OK;
}

extern "C" {

GG_API int gg_volume_create(gg_context* ctx, uint32_t size, gg_volume** out) {
    if (!ctx || !out) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_create needs a context and an output.");
    *out = nullptr;
    if (size < 2 || size > 1024) return gg::fail(GG_ERR_INVALID_ARGUMENT, "Volume size %u is outside 2..1024.", size);
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t voxels = (uint64_t)size * size * size;
    const uint64_t sums_bytes = voxels * 24u;
    const uint64_t tex_bytes = voxels * 8u * 2u;
    if (ctx->used + sums_bytes + tex_bytes > ctx->budget)
        return gg::fail(GG_ERR_OVER_BUDGET, "A %u^3 volume needs %llu bytes but the budget has %llu bytes left.", size,
                        (unsigned long long)(sums_bytes + tex_bytes), (unsigned long long)(ctx->budget - ctx->used));
    gg_volume* vol = new gg_volume();
    vol->ctx = ctx;
    vol->size = size;
    int s = gg::device_alloc(ctx, sums_bytes, (void**)&vol->sums, "volume sums");
    if (s == GG_OK) s = gg::cuda_status(cudaMemsetAsync(vol->sums, 0, sums_bytes, ctx->stream), "volume clear");
    cudaChannelFormatDesc desc = cudaCreateChannelDescHalf4();
    cudaExtent extent = make_cudaExtent(size, size, size);
    if (s == GG_OK) s = gg::cuda_status(cudaMalloc3DArray(&vol->emission, &desc, extent, cudaArraySurfaceLoadStore), "emission volume");
    if (s == GG_OK) s = gg::cuda_status(cudaMalloc3DArray(&vol->velocity, &desc, extent, cudaArraySurfaceLoadStore), "velocity volume");
    if (s == GG_OK) ctx->used += tex_bytes;
    vol->bytes = sums_bytes + tex_bytes;
    for (int k = 0; k < 2 && s == GG_OK; ++k) {
        cudaArray_t arr = k == 0 ? vol->emission : vol->velocity;
        cudaResourceDesc res{};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = arr;
        // Trilinear, normalized coordinates, zero outside (march.metal:18).
        cudaTextureDesc td{};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 1;
        cudaTextureObject_t tex = 0;
        cudaSurfaceObject_t surf = 0;
        s = gg::cuda_status(cudaCreateTextureObject(&tex, &res, &td, nullptr), "volume texture");
        if (s == GG_OK) s = gg::cuda_status(cudaCreateSurfaceObject(&surf, &res), "volume surface");
        if (k == 0) { vol->emission_tex = tex; vol->emission_surf = surf; }
        else { vol->velocity_tex = tex; vol->velocity_surf = surf; }
    }
    if (s == GG_OK) {
        // Start with empty textures: a resolve of the zeroed sums.
        SplatUniforms u{};
        u.volumeSize = size;
        u.halfExtent = VOLUME_HALF_EXTENT;
        u.peakTemperature = T_PEAK_DEFAULT;
        s = gg_splat_resolve(vol, &u, nullptr);
    }
    if (s == GG_OK) s = gg::cuda_status(cudaStreamSynchronize(ctx->stream), "volume set-up");
    if (s != GG_OK) {
        gg_volume_destroy(vol);
        return s;
    }
    *out = vol;
    return GG_OK;
}

GG_API void gg_volume_destroy(gg_volume* vol) {
    if (!vol) return;
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (vol->emission_tex) cudaDestroyTextureObject(vol->emission_tex);
    if (vol->velocity_tex) cudaDestroyTextureObject(vol->velocity_tex);
    if (vol->emission_surf) cudaDestroySurfaceObject(vol->emission_surf);
    if (vol->velocity_surf) cudaDestroySurfaceObject(vol->velocity_surf);
    if (vol->emission) cudaFreeArray(vol->emission);
    if (vol->velocity) cudaFreeArray(vol->velocity);
    const uint64_t voxels = (uint64_t)vol->size * vol->size * vol->size;
    gg::device_free(ctx, vol->sums, voxels * 24u);
    uint64_t tex = voxels * 16u;
    ctx->used -= tex < ctx->used ? tex : ctx->used;
    delete vol;
}

GG_API int gg_splat_bin(gg_particles* ps, gg_volume* vol, const SplatUniforms* u) {
    if (!ps) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_splat_bin needs a particle system.");
    GG_CHECK(check_splat(ps, vol, u, "gg_splat_bin"));
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    SplatArgs a{ps->pos, ps->vel, vol->sums, *u, ps->first_index};
    bin_kernel<<<(ps->count + 255u) / 256u, 256, 0, ctx->stream>>>(a);
    return gg::launch_status("splat bin");
}

GG_API int gg_splat_resolve(gg_volume* vol, const SplatUniforms* u, const gg_particles* ps) {
    GG_CHECK(check_splat(ps, vol, u, "gg_splat_resolve"));
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    ResolveArgs a{vol->sums, vol->emission_surf, vol->velocity_surf, ctx->blackbody, *u};
    const uint64_t total = (uint64_t)vol->size * vol->size * vol->size;
    resolve_kernel<<<(unsigned)((total + 255u) / 256u), 256, 0, ctx->stream>>>(a);
    return gg::launch_status("splat resolve");
}

GG_API int gg_splat(gg_particles* ps, gg_volume* vol, const SplatUniforms* u) {
    GG_CHECK(gg_splat_bin(ps, vol, u));
    return gg_splat_resolve(vol, u, ps);
}

GG_API int gg_volume_clear(gg_volume* vol) {
    if (!vol) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_clear needs a volume.");
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t bytes = (uint64_t)vol->size * vol->size * vol->size * 24u;
    const uint64_t n16 = bytes / 16u;  // 24 n^3 is a multiple of 16 for even n; the tail is cleared below
    if (n16) clear_kernel<<<(unsigned)((n16 + 255u) / 256u), 256, 0, ctx->stream>>>(reinterpret_cast<uint4*>(vol->sums), n16);
    GG_CHECK(gg::launch_status("volume clear"));
    if (bytes % 16u) GG_CUDA(cudaMemsetAsync(reinterpret_cast<char*>(vol->sums) + n16 * 16u, 0, bytes % 16u, ctx->stream), "volume clear");
    return GG_OK;
}

GG_API int gg_volume_read_sums(gg_volume* vol, uint32_t* emission, int32_t* momentum, uint32_t* mass) {
    if (!vol || !emission || !momentum || !mass)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_read_sums needs a volume and three output arrays.");
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t voxels = (uint64_t)vol->size * vol->size * vol->size;
    std::vector<uint32_t> rec(voxels * 6u);
    GG_CUDA(cudaMemcpyAsync(rec.data(), vol->sums, voxels * 24u, cudaMemcpyDeviceToHost, ctx->stream), "sums readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "sums readback");
    for (uint64_t i = 0; i < voxels; ++i) {
        emission[2 * i + 0] = rec[6 * i + 0];
        emission[2 * i + 1] = rec[6 * i + 1];
        momentum[3 * i + 0] = (int32_t)rec[6 * i + 2];
        momentum[3 * i + 1] = (int32_t)rec[6 * i + 3];
        momentum[3 * i + 2] = (int32_t)rec[6 * i + 4];
        mass[i] = rec[6 * i + 5];
    }
    return GG_OK;
}

GG_API int gg_volume_write_sums(gg_volume* vol, const uint32_t* emission, const int32_t* momentum, const uint32_t* mass) {
    if (!vol || !emission || !momentum || !mass)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_write_sums needs a volume and three input arrays.");
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t voxels = (uint64_t)vol->size * vol->size * vol->size;
    std::vector<uint32_t> rec(voxels * 6u);
    for (uint64_t i = 0; i < voxels; ++i) {
        rec[6 * i + 0] = emission[2 * i + 0];
        rec[6 * i + 1] = emission[2 * i + 1];
        rec[6 * i + 2] = (uint32_t)momentum[3 * i + 0];
        rec[6 * i + 3] = (uint32_t)momentum[3 * i + 1];
        rec[6 * i + 4] = (uint32_t)momentum[3 * i + 2];
        rec[6 * i + 5] = mass[i];
    }
    GG_CUDA(cudaMemcpyAsync(vol->sums, rec.data(), voxels * 24u, cudaMemcpyHostToDevice, ctx->stream), "sums upload");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "sums upload");
    return GG_OK;
}

GG_API int gg_volume_sums(gg_volume* vol, void** device_words, uint64_t* words) {
    if (!vol || !device_words || !words)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_sums needs a volume and two outputs.");
    *device_words = vol->sums;
    *words = (uint64_t)vol->size * vol->size * vol->size * 6u;
    return GG_OK;
}

static int copy_volume_array(gg_volume* vol, cudaArray_t arr, void* host, bool to_host) {
    cudaMemcpy3DParms p{};
    cudaExtent e = make_cudaExtent(vol->size, vol->size, vol->size);
    p.extent = e;
    if (to_host) {
        p.srcArray = arr;
        p.dstPtr = make_cudaPitchedPtr(host, vol->size * 8u, vol->size, vol->size);
        p.kind = cudaMemcpyDeviceToHost;
    } else {
        p.dstArray = arr;
        p.srcPtr = make_cudaPitchedPtr(host, vol->size * 8u, vol->size, vol->size);
        p.kind = cudaMemcpyHostToDevice;
    }
    GG_CUDA(cudaMemcpy3DAsync(&p, vol->ctx->stream), "volume copy");
    return GG_OK;
}

GG_API int gg_volume_read(gg_volume* vol, uint16_t* emission_half4, uint16_t* velocity_half4) {
    if (!vol) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_read needs a volume.");
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (emission_half4) GG_CHECK(copy_volume_array(vol, vol->emission, emission_half4, true));
    if (velocity_half4) GG_CHECK(copy_volume_array(vol, vol->velocity, velocity_half4, true));
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "volume readback");
    return GG_OK;
}

GG_API int gg_volume_write(gg_volume* vol, const uint16_t* emission_half4, const uint16_t* velocity_half4) {
    if (!vol) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_write needs a volume.");
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (emission_half4) GG_CHECK(copy_volume_array(vol, vol->emission, const_cast<uint16_t*>(emission_half4), false));
    if (velocity_half4) GG_CHECK(copy_volume_array(vol, vol->velocity, const_cast<uint16_t*>(velocity_half4), false));
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "volume upload");
    return GG_OK;
}

}  // extern "C"
