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
// One CTA per table entry; its threads split the midpoint sum and reduce it
// in a fixed tree order. The periapsis rp(b) is a 60-step Newton iteration
// on 1 - b^2 u^2 (1 - 2u) = 0 from u = 1/b, run by one thread.
#include "common.cuh"
#include "runtime.h"

namespace gg {

constexpr int kTableThreads = 256;
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

// Block-wide midpoint sum of the sweep integrand; every thread returns it.
__device__ double sweep_block(double r, double b, int intervals, double* red) {
    double bound = fmin(b, max_impact_parameter(r));
    double umax = 1.0 / r;
    double h = (kPiD / 2.0) / (double)intervals;
    double part = 0.0;
    if (b > 0.0) {
        for (int k = threadIdx.x; k < intervals; k += blockDim.x) {
            double th = ((double)k + 0.5) * h;
            double s, c;
            sincos(th, &s, &c);
            double u = umax * s * s;
            double inner = 1.0 - bound * bound * u * u * (1.0 - 2.0 * u);
            if (inner > 0.0) part += bound * 2.0 * umax * s * c / sqrt(inner);
        }
    }
    red[threadIdx.x] = part;
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) red[threadIdx.x] += red[threadIdx.x + stride];
        __syncthreads();
    }
    double total = red[0] * h;
    __syncthreads();
    return total;
}

// kind 0: S(r, b) over [0, bMax(r)]; kind 1: the sky table of a camera at r
// for rays that turn outside entry_radius.
__global__ void __launch_bounds__(kTableThreads) build_table_kernel(int kind, double r, double entry_radius,
                                                                   int intervals, float* out) {
    __shared__ double red[kTableThreads];
    __shared__ double peri;
    const int k = blockIdx.x;
    const double t = (double)k / (double)(SWEEP_TABLE_SIZE - 1);
    if (kind == 0) {
        double b = table_b(0.0, max_impact_parameter(r), t);
        double s = sweep_block(r, b, intervals, red);
        if (threadIdx.x == 0) out[k] = (float)s;
    } else {
        double b = table_b(max_impact_parameter(entry_radius), max_impact_parameter(r), t);
        if (threadIdx.x == 0) peri = periapsis(b);
        __syncthreads();
        double sp = sweep_block(peri, b, intervals, red);
        double sr = sweep_block(r, b, intervals, red);
        if (threadIdx.x == 0) out[k] = (float)(2.0 * (sp - sr) + sr);
    }
}

static double host_max_b(double r) { return r / std::sqrt(1.0 - 2.0 / r); }

int sweep_init(gg_context* ctx) {
    GG_CHECK(device_alloc(ctx, SWEEP_TABLE_SIZE * sizeof(float), (void**)&ctx->sphere_table, "sphere sweep table"));
    const double sphere = VOLUME_HALF_EXTENT;
    const double entry = sphere - 1.0;  // DeflectionTables.swift:35-38
    build_table_kernel<<<SWEEP_TABLE_SIZE, kTableThreads, 0, ctx->stream>>>(0, sphere, entry, SWEEP_SPHERE_INTERVALS,
                                                                            ctx->sphere_table);
    GG_CHECK(launch_status("sphere sweep table"));
    ctx->sphere_max_b = (float)host_max_b(entry);
    ctx->sphere_table_max_b = (float)host_max_b(sphere);
    return GG_OK;
}

int sweep_build(gg_context* ctx, cudaStream_t stream, double camera_radius, gg_sweep* out) {
    if (!(camera_radius > VOLUME_HALF_EXTENT))
        return fail(GG_ERR_INVALID_ARGUMENT, "The sweep tables need a camera outside the r = %.0f sphere, not r = %g.",
                    (double)VOLUME_HALF_EXTENT, camera_radius);
    // Callers may supply stream-ordered buffers; otherwise they come from the budget.
    if (!out->camera) GG_CHECK(device_alloc(ctx, SWEEP_TABLE_SIZE * sizeof(float), (void**)&out->camera, "camera sweep table"));
    if (!out->sky) GG_CHECK(device_alloc(ctx, SWEEP_TABLE_SIZE * sizeof(float), (void**)&out->sky, "sky sweep table"));
    const double entry = (double)VOLUME_HALF_EXTENT - 1.0;
    build_table_kernel<<<SWEEP_TABLE_SIZE, kTableThreads, 0, stream>>>(0, camera_radius, entry, SWEEP_CAMERA_INTERVALS,
                                                                       out->camera);
    build_table_kernel<<<SWEEP_TABLE_SIZE, kTableThreads, 0, stream>>>(1, camera_radius, entry, SWEEP_CAMERA_INTERVALS,
                                                                       out->sky);
    GG_CHECK(launch_status("camera sweep tables"));
    out->camera_radius = camera_radius;
    out->camera_max_b = (float)host_max_b(camera_radius);
    out->sky_max_b = out->camera_max_b;
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
