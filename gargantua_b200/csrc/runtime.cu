// Context, status reporting, budgeted allocation and the FP64 host tables.
#include "runtime.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {
thread_local std::string g_last_error;
}

namespace gg {

int fail(int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return status;
}

int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return GG_OK;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(GG_ERR_OUT_OF_MEMORY, "%s: the device is out of memory.", what);
    }
    return fail(GG_ERR_DEVICE, "%s failed on the device: %s.", what, cudaGetErrorString(e));
}

int launch_status(const char* what) { return cuda_status(cudaGetLastError(), what); }

int device_alloc(gg_context* ctx, uint64_t bytes, void** out, const char* what) {
    *out = nullptr;
    if (bytes == 0) return GG_OK;
    if (ctx->used + bytes > ctx->budget) {
        return fail(GG_ERR_OVER_BUDGET,
                    "%s needs %llu bytes but the context budget has %llu of %llu bytes left.", what,
                    (unsigned long long)bytes, (unsigned long long)(ctx->budget - ctx->used),
                    (unsigned long long)ctx->budget);
    }
    GG_CUDA(cudaMalloc(out, bytes), what);
    ctx->used += bytes;
    return GG_OK;
}

void device_free(gg_context* ctx, void* ptr, uint64_t bytes) {
    if (!ptr) return;
    cudaFree(ptr);
    ctx->used -= bytes < ctx->used ? bytes : ctx->used;
}

int ensure_capacity(gg_context* ctx, void** ptr, uint64_t* capacity, uint64_t bytes, const char* what) {
    if (*capacity >= bytes) return GG_OK;
    GG_CUDA(cudaStreamSynchronize(ctx->stream), what);
    device_free(ctx, *ptr, *capacity);
    *ptr = nullptr;
    *capacity = 0;
    uint64_t grown = bytes < 4096 ? 4096 : bytes;
    GG_CHECK(device_alloc(ctx, grown, ptr, what));
    *capacity = grown;
    return GG_OK;
}

// ---------------------------------------------------------------------------
// Host tables, FP64. The steady-disk inverse CDF follows
// DiskModel.radialInverseCdf (DiskModel.swift:42-78) and the blackbody colour
// table Blackbody.table (Blackbody.swift:11-86); the host builds both once,
// as ParticleSystem.init does (ParticleSystem.swift:23-47).

static const double kPi = 3.14159265358979323846;

double disk_shape(double r, double floor) {
    double x = R_ISCO / r;
    double torque = std::fmax(1.0 - std::sqrt(x), floor);
    return std::pow(x, 0.75) * std::pow(torque, 0.25);
}

static double steady_number_density(double r) {
    const double isco = R_ISCO, outer = R_DISK_OUTER, feed = R_FEED_INNER;
    if (r <= isco || r >= outer) return 0.0;
    double flux = r <= feed ? 1.0 : (outer * outer - r * r) / (outer * outer - feed * feed);
    return 2.0 * kPi * r * (flux * (r - isco) / std::pow(r, 1.5));
}

// Inverse CDF of radius for a surface density Sigma ~ r^-p on [R_ISCO,
// R_DISK_OUTER] (number per dr ~ r^(1-p)), at u = k / (count - 1):
// r = (r0^q + u (r1^q - r0^q))^(1/q), q = 2 - p (q = 0: r0 (r1/r0)^u).
void power_law_inverse_cdf(int count, double exponent, double* table) {
    const double r0 = R_ISCO, r1 = R_DISK_OUTER, q = 2.0 - exponent;
    for (int k = 0; k < count; ++k) {
        double u = (double)k / (double)(count - 1);
        if (std::fabs(q) < 1e-12) {
            table[k] = r0 * std::pow(r1 / r0, u);
        } else {
            double a = std::pow(r0, q), b = std::pow(r1, q);
            table[k] = std::pow(a + u * (b - a), 1.0 / q);
        }
    }
    table[0] = r0;
    table[count - 1] = r1;
}

void radial_inverse_cdf(int count, int resolution, double* table) {
    const double r0 = R_ISCO, r1 = R_DISK_OUTER;
    const double dr = (r1 - r0) / resolution;
    std::vector<double> cumulative(resolution + 1, 0.0);
    double previous = steady_number_density(r0);
    for (int i = 1; i <= resolution; ++i) {
        double density = steady_number_density(r0 + i * dr);
        cumulative[i] = cumulative[i - 1] + 0.5 * (previous + density) * dr;
        previous = density;
    }
    const double total = cumulative[resolution];
    int i = 0;
    for (int k = 0; k < count; ++k) {
        double target = total * k / (count - 1);
        while (i < resolution && cumulative[i + 1] < target) ++i;
        if (i >= resolution) {
            table[k] = r1;
            continue;
        }
        double span = cumulative[i + 1] - cumulative[i];
        double t = span > 0 ? (target - cumulative[i]) / span : 0.0;
        table[k] = r0 + (i + t) * dr;
    }
    table[count - 1] = r1;
}

static double gauss_lobe(double x, double mu, double s1, double s2) {
    double t = (x - mu) / (x < mu ? s1 : s2);
    return std::exp(-0.5 * t * t);
}

void blackbody_table(int count, double tmin, double tmax, double* rgb) {
    const double c2 = 1.438776877e-2;  // second radiation constant, m K (CODATA 2018)
    for (int k = 0; k < count; ++k) {
        double t = (double)k / (count - 1);
        double temperature = std::exp(std::log(tmin) + t * (std::log(tmax) - std::log(tmin)));
        double X = 0, Y = 0, Z = 0;
        for (double nm = 380.0; nm <= 780.0; nm += 1.0) {
            // CIE 1931 matching functions, multi-lobe fit of Wyman, Sloan and Shirley 2013.
            double xb = 1.056 * gauss_lobe(nm, 599.8, 37.9, 31.0) + 0.362 * gauss_lobe(nm, 442.0, 16.0, 26.7) -
                        0.065 * gauss_lobe(nm, 501.1, 20.4, 26.2);
            double yb = 0.821 * gauss_lobe(nm, 568.8, 46.9, 40.5) + 0.286 * gauss_lobe(nm, 530.9, 16.3, 31.1);
            double zb = 1.217 * gauss_lobe(nm, 437.0, 11.8, 36.0) + 0.681 * gauss_lobe(nm, 459.0, 26.0, 13.4);
            double lambda = nm * 1e-9;
            double planck = 1.0 / (std::pow(lambda, 5.0) * (std::exp(c2 / (lambda * temperature)) - 1.0));
            X += xb * planck;
            Y += yb * planck;
            Z += zb * planck;
        }
        // XYZ to linear sRGB, D65 (IEC 61966-2-1).
        double r = std::fmax(3.2406 * X - 1.5372 * Y - 0.4986 * Z, 0.0);
        double g = std::fmax(-0.9689 * X + 1.8758 * Y + 0.0415 * Z, 0.0);
        double b = std::fmax(0.0557 * X - 0.2040 * Y + 1.0570 * Z, 0.0);
        double peak = std::fmax(r, std::fmax(g, b));
        if (peak > 0.0) {
            r /= peak;
            g /= peak;
            b /= peak;
        } else {
            r = g = b = 1.0;
        }
        rgb[3 * k + 0] = r;
        rgb[3 * k + 1] = g;
        rgb[3 * k + 2] = b;
    }
}

}  // namespace gg

// ------------------------------------------------------------- public API

extern "C" {

GG_API const char* gg_version(void) { return "gargantua-b200 0.1.0 (sm_100a)"; }

GG_API const char* gg_last_error(void) { return g_last_error.c_str(); }

GG_API const char* gg_status_name(int status) {
    switch (status) {
        case GG_OK: return "ok";
        case GG_ERR_INVALID_ARGUMENT: return "invalid argument";
        case GG_ERR_OUT_OF_MEMORY: return "out of memory";
        case GG_ERR_OVER_BUDGET: return "over budget";
        case GG_ERR_DEVICE: return "device error";
        case GG_ERR_TIMEOUT: return "timeout";
        case GG_ERR_NOT_READY: return "not ready";
        case GG_ERR_NO_DEVICE: return "no device";
        case GG_ERR_UNSUPPORTED: return "unsupported";
        case GG_ERR_CANCELLED: return "cancelled";
        default: return "unknown status";
    }
}

GG_API int gg_context_create(int device, uint64_t budget_bytes, gg_context** out) {
    if (!out) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_context_create needs an output pointer.");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return gg::fail(GG_ERR_NO_DEVICE, "No CUDA device is available.");
    }
    if (device < 0 || device >= n)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Device %d does not exist; %d devices are visible.", device, n);
    GG_CUDA(cudaSetDevice(device), "cudaSetDevice");
    cudaDeviceProp prop;
    GG_CUDA(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    if (prop.major < 10)
        return gg::fail(GG_ERR_UNSUPPORTED, "Device %d (%s, sm_%d%d) is not a Blackwell sm_100 part.", device,
                        prop.name, prop.major, prop.minor);
    gg_context* ctx = new gg_context();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    uint64_t total = prop.totalGlobalMem;
    if (budget_bytes == 0) {
        uint64_t fraction = (uint64_t)((double)total * MEMORY_BUDGET_FRACTION);
        budget_bytes = fraction < (uint64_t)MEMORY_BUDGET_CAP_BYTES ? fraction : (uint64_t)MEMORY_BUDGET_CAP_BYTES;
    }
    ctx->budget = budget_bytes;
    int s = gg::cuda_status(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (s == GG_OK) s = gg::device_alloc(ctx, sizeof(MarchCounters), (void**)&ctx->counters, "march counters");
    if (s == GG_OK) s = gg::device_alloc(ctx, 4 * sizeof(unsigned long long), (void**)&ctx->stats, "march statistics");
    if (s == GG_OK) s = gg::cuda_status(cudaMemsetAsync(ctx->stats, 0, 4 * sizeof(unsigned long long), ctx->stream), "statistics reset");
    if (s == GG_OK) s = gg::blackbody_init(ctx);
    if (s == GG_OK) s = gg::sweep_init(ctx);
    if (s == GG_OK) s = gg::cuda_status(cudaStreamSynchronize(ctx->stream), "context set-up");
    if (s != GG_OK) {
        std::string keep = g_last_error;
        gg_context_destroy(ctx);
        g_last_error = keep;
        return s;
    }
    *out = ctx;
    return GG_OK;
}

GG_API void gg_context_destroy(gg_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->sphere_table);
    cudaFree(ctx->sweep.camera);
    cudaFree(ctx->sweep.sky);
    cudaFree(ctx->blackbody);
    cudaFree(ctx->counters);
    cudaFree(ctx->stats);
    cudaFree(ctx->probe_buffer);
    cudaFree(ctx->flagged);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

GG_API int gg_context_synchronize(gg_context* ctx) {
    if (!ctx) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_context_synchronize needs a context.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "synchronize");
    return GG_OK;
}

GG_API int gg_context_memory(gg_context* ctx, uint64_t* budget, uint64_t* used) {
    if (!ctx) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_context_memory needs a context.");
    if (budget) *budget = ctx->budget;
    if (used) *used = ctx->used;
    return GG_OK;
}

GG_API void* gg_context_stream(gg_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

GG_API int gg_host_alloc(gg_context* ctx, uint64_t bytes, void** out) {
    if (!ctx || !out) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_host_alloc needs a context and an output.");
    *out = nullptr;
    if (bytes == 0) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_host_alloc needs a positive size.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const cudaError_t e = cudaHostAlloc(out, (size_t)bytes, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        *out = nullptr;
        cudaGetLastError();
        return gg::fail(GG_ERR_OUT_OF_MEMORY, "Page-locked host memory of %llu bytes is not available (%s).",
                        (unsigned long long)bytes, cudaGetErrorString(e));
    }
    return GG_OK;
}

GG_API void gg_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

}  // extern "C"
