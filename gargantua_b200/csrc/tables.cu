// Sweep tables (Deflection.swift:14-106, DeflectionTables.swift:29-76),
// built in FP64 on the device.
//
// A ray of impact parameter b sweeps S(R, b) = integral_0^{1/R} b du /
// sqrt(1 - b^2 u^2 (1 - 2u)) in azimuth from radius R to infinity. After
// u = uMax sin^2(theta) the integrand is finite at the turning point and the
// composite midpoint rule never touches an endpoint. Three tables of
// SWEEP_TABLE_SIZE entries, sampled at b = lo + (hi - lo)(1 - (1 - t)^2):
//   sphere: S(30, b), b in [0, bMax(30)], 2048 intervals (fixed)
//   camera: S(Rc, b), b in [0, bMax(Rc)], 256 intervals
//   sky:    2 (S(rp(b), b) - S(Rc, b)) + S(Rc, b), b in [bMax(29), bMax(Rc)]
// One warp per table entry: its lanes split the midpoint sum and reduce it
// with shuffles in a fixed tree order (lane 0's total, broadcast), so a
// table is the same bits on every build. The periapsis rp(b) is a 60-step
// Newton iteration on 1 - b^2 u^2 (1 - 2u) = 0 from u = 1/b, run by every
// lane alike. One launch builds the camera and sky tables of up to
// kTableJobs camera radii (the requests a server admits together): grid x
// covers the entries, y the radii, z the two kinds.
#include "common.cuh"
#include "runtime.h"

namespace gg {

constexpr double kPiD = 3.14159265358979323846;

__device__ __forceinline__ double max_impact_parameter(double r) { return r / sqrt(1.0 - 2.0 / r); }

__device__ __forceinline__ double table_b(double lo, double hi, double t) {
    double back = 1.0 - t;
    return lo + (hi - lo) * (1.0 - back * back);
}

__device__ double periapsis(double b) {
    double u = 1.0 / b;
    for (int i = 0; i < 60; ++i) {
        double value = 1.0 - b * b * u * u * (1.0 - 2.0 * u);
        double slope = -b * b * (2.0 * u - 6.0 * u * u);
        double next = u - value / slope;
        if (fabs(next - u) < 1e-15) {
            u = next;
            break;
        }
        u = next;
    }
    return 1.0 / u;
}

// Warp-wide midpoint sum of the sweep integrand; every lane returns it.
__device__ double sweep_warp(double r, double b, int intervals, uint32_t lane) {
    const double bound = fmin(b, max_impact_parameter(r));
    const double umax = 1.0 / r;
    const double h = (kPiD / 2.0) / (double)intervals;
    double part = 0.0;
    if (b > 0.0) {
        for (int k = (int)lane; k < intervals; k += 32) {
            const double th = ((double)k + 0.5) * h;
            double sn, cs;
            sincos(th, &sn, &cs);
            const double u = umax * sn * sn;
            const double inner = 1.0 - bound * bound * u * u * (1.0 - 2.0 * u);
            if (inner > 0.0) part += bound * 2.0 * umax * sn * cs / sqrt(inner);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
    return __shfl_sync(0xffffffffu, part, 0) * h;
}

// The tables of up to kTableJobs radii: kind 0 (z = 0) is S(r, b) over
// [0, bMax(r)] into camera[j]; kind 1 (z = 1) the sky table of a camera at
// r for rays that turn outside entry_radius, into sky[j] (skipped when
// null).
constexpr int kTableJobs = 128;
constexpr int kTableWarps = 8;  // entries per block

struct TableJobs {
    int count;
    double radius[kTableJobs];
    float* camera[kTableJobs];
    float* sky[kTableJobs];
};

__global__ void __launch_bounds__(kTableWarps * 32) build_tables_kernel(TableJobs jobs, double entry_radius,
                                                                        int intervals) {
    const int j = blockIdx.y;
    const uint32_t lane = threadIdx.x & 31u;
    const int k = blockIdx.x * kTableWarps + (int)(threadIdx.x >> 5);
    if (j >= jobs.count || k >= (int)SWEEP_TABLE_SIZE) return;
    const double r = jobs.radius[j];
    const double t = (double)k / (double)(SWEEP_TABLE_SIZE - 1);
    if (blockIdx.z == 0) {
        const double b = table_b(0.0, max_impact_parameter(r), t);
        const double s = sweep_warp(r, b, intervals, lane);
        if (lane == 0) jobs.camera[j][k] = (float)s;
    } else {
        if (!jobs.sky[j]) return;
        const double b = table_b(max_impact_parameter(entry_radius), max_impact_parameter(r), t);
        const double peri = periapsis(b);
        const double sp = sweep_warp(peri, b, intervals, lane);
        const double sr = sweep_warp(r, b, intervals, lane);
        if (lane == 0) jobs.sky[j][k] = (float)(2.0 * (sp - sr) + sr);
    }
}

static int launch_tables(const TableJobs& jobs, int kinds, double entry_radius, int intervals, cudaStream_t stream) {
    if (jobs.count == 0) return GG_OK;
    dim3 grid((SWEEP_TABLE_SIZE + kTableWarps - 1) / kTableWarps, (unsigned)jobs.count, (unsigned)kinds);
    build_tables_kernel<<<grid, kTableWarps * 32, 0, stream>>>(jobs, entry_radius, intervals);
    return launch_status("sweep tables");
}

static double host_max_b(double r) { return r / std::sqrt(1.0 - 2.0 / r); }

int sweep_init(gg_context* ctx) {
    GG_CHECK(device_alloc(ctx, SWEEP_TABLE_SIZE * sizeof(float), (void**)&ctx->sphere_table, "sphere sweep table"));
    const double sphere = VOLUME_HALF_EXTENT;
    const double entry = sphere - 1.0;  // DeflectionTables.swift:35-38
    TableJobs jobs{};
    jobs.count = 1;
    jobs.radius[0] = sphere;
    jobs.camera[0] = ctx->sphere_table;
    GG_CHECK(launch_tables(jobs, 1, entry, SWEEP_SPHERE_INTERVALS, ctx->stream));
    ctx->sphere_max_b = (float)host_max_b(entry);
    ctx->sphere_table_max_b = (float)host_max_b(sphere);
    return GG_OK;
}

int sweep_build(gg_context* ctx, cudaStream_t stream, double camera_radius, gg_sweep* out) {
    return sweep_build_batch(ctx, stream, &camera_radius, &out, 1);
}

int sweep_build_batch(gg_context* ctx, cudaStream_t stream, const double* camera_radius, gg_sweep* const* out,
                      int count) {
    for (int i = 0; i < count; ++i)
        if (!(camera_radius[i] > VOLUME_HALF_EXTENT))
            return fail(GG_ERR_INVALID_ARGUMENT,
                        "The sweep tables need a camera outside the r = %.0f sphere, not r = %g.",
                        (double)VOLUME_HALF_EXTENT, camera_radius[i]);
    const double entry = (double)VOLUME_HALF_EXTENT - 1.0;
    TableJobs jobs{};
    for (int i = 0; i < count; ++i) {
        gg_sweep* o = out[i];
        // Callers may supply stream-ordered buffers; otherwise they come from the budget.
        if (!o->camera) GG_CHECK(device_alloc(ctx, SWEEP_TABLE_SIZE * sizeof(float), (void**)&o->camera, "camera sweep table"));
        if (!o->sky) GG_CHECK(device_alloc(ctx, SWEEP_TABLE_SIZE * sizeof(float), (void**)&o->sky, "sky sweep table"));
        jobs.radius[jobs.count] = camera_radius[i];
        jobs.camera[jobs.count] = o->camera;
        jobs.sky[jobs.count] = o->sky;
        ++jobs.count;
        if (jobs.count == kTableJobs || i == count - 1) {
            GG_CHECK(launch_tables(jobs, 2, entry, SWEEP_CAMERA_INTERVALS, stream));
            jobs.count = 0;
        }
        o->camera_radius = camera_radius[i];
        o->camera_max_b = (float)host_max_b(camera_radius[i]);
        o->sky_max_b = o->camera_max_b;
    }
    return GG_OK;
}

// DeflectionTables.apply (DeflectionTables.swift:68-76).
void sweep_apply(const gg_context* ctx, const gg_sweep* sweep, MarchUniforms* u) {
    u->sphereRadius = VOLUME_HALF_EXTENT;
    u->cameraRadius = (float)sweep->camera_radius;
    u->sphereMaxB = ctx->sphere_max_b;
    u->sphereTableMaxB = ctx->sphere_table_max_b;
    u->cameraMaxB = sweep->camera_max_b;
    u->skyMinB = ctx->sphere_max_b;
    u->skyMaxB = sweep->sky_max_b;
}

}  // namespace gg

extern "C" {

GG_API int gg_tables_update(gg_context* ctx, float camera_radius, MarchUniforms* inout) {
    if (!ctx || !inout) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_tables_update needs a context and uniforms.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    // DeflectionTables.update rebuilds only when the radius moved (:57-64).
    if (!ctx->sweep.camera || std::fabs((double)camera_radius - ctx->sweep.camera_radius) > 1e-6)
        GG_CHECK(gg::sweep_build(ctx, ctx->stream, (double)camera_radius, &ctx->sweep));
    gg::sweep_apply(ctx, &ctx->sweep, inout);
    return GG_OK;
}

GG_API int gg_tables_read(gg_context* ctx, float* sphere, float* camera, float* sky) {
    if (!ctx) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_tables_read needs a context.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const size_t bytes = SWEEP_TABLE_SIZE * sizeof(float);
    if (sphere) GG_CUDA(cudaMemcpyAsync(sphere, ctx->sphere_table, bytes, cudaMemcpyDeviceToHost, ctx->stream), "table readback");
    if (camera) {
        if (!ctx->sweep.camera) return gg::fail(GG_ERR_NOT_READY, "No camera table has been built yet.");
        GG_CUDA(cudaMemcpyAsync(camera, ctx->sweep.camera, bytes, cudaMemcpyDeviceToHost, ctx->stream), "table readback");
    }
    if (sky) {
        if (!ctx->sweep.sky) return gg::fail(GG_ERR_NOT_READY, "No sky table has been built yet.");
        GG_CUDA(cudaMemcpyAsync(sky, ctx->sweep.sky, bytes, cudaMemcpyDeviceToHost, ctx->stream), "table readback");
    }
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "table readback");
    return GG_OK;
}

}  // extern "C"
