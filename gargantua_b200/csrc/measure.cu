// Device peak measurements for the rooflines: FP32 FMA throughput, and the
// throughput of 32-bit global atomic adds in the splat's access pattern.
//
// Each thread runs kChains independent chains of dependent fused
// multiply-adds (x = x * a + b), enough independent work per warp to fill
// the FMA pipes; the grid covers every SM with several resident blocks. The
// result is what this device sustains for FP32 FMA at its current clocks:
// the denominator of the march kernel's FLOP/s fraction.
#include "runtime.h"

namespace gg {

constexpr int kChains = 8;
constexpr int kFmaIterations = 4096;

__global__ void __launch_bounds__(256) ffma_kernel(float a, float b, float* sink) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (float)(threadIdx.x + c);
    for (int i = 0; i < kFmaIterations; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 12345.678f) sink[threadIdx.x] = s;  // keeps the chains live
}

// Uniformly scattered six-word records, the splat's record layout: each
// thread adds 1 to all six words of kDeposits records drawn from an LCG, so
// the adds land on distinct sectors with negligible contention. The result
// is the device's rate of relaxed global u32 atomic adds (RED) into an
// L2-resident grid, the ceiling of the splat's deposit loop.
constexpr int kDeposits = 64;

__global__ void __launch_bounds__(256) red_kernel(uint32_t* sums, uint32_t records, uint32_t seed) {
    uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) * 0x9E3779B1u + seed;
    for (int i = 0; i < kDeposits; ++i) {
        h = h * 1664525u + 1013904223u;
        uint32_t* rec = sums + 6u * __umulhi(h, records);
        atomicAdd(rec + 0, 1u);
        atomicAdd(rec + 1, 1u);
        atomicAdd(rec + 2, 1u);
        atomicAdd(rec + 3, 1u);
        atomicAdd(rec + 4, 1u);
        atomicAdd(rec + 5, 1u);
    }
}

// The same adds into a shared-memory tile of 9^3 records (the brick splat's
// tile at edge 8) laid out as the deposit lays it out: six words and a pad,
// an odd stride, so that one word of records at random cells spreads over
// all 32 banks. The result is the device's rate of scattered shared-memory
// u32 atomic adds: the ceiling of the deposit loop.
constexpr uint32_t kTileRecords = 9u * 9u * 9u;
constexpr uint32_t kTileStride = 7u;

__global__ void __launch_bounds__(256) shared_red_kernel(uint32_t* sink, uint32_t seed) {
    __shared__ uint32_t tile[kTileRecords * kTileStride];
    for (uint32_t w = threadIdx.x; w < kTileRecords * kTileStride; w += blockDim.x) tile[w] = 0u;
    __syncthreads();
    uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) * 0x9E3779B1u + seed;
    for (int i = 0; i < kDeposits * 4; ++i) {
        h = h * 1664525u + 1013904223u;
        uint32_t* rec = tile + kTileStride * __umulhi(h, kTileRecords);
        atomicAdd(rec + 0, 1u);
        atomicAdd(rec + 1, 1u);
        atomicAdd(rec + 2, 1u);
        atomicAdd(rec + 3, 1u);
        atomicAdd(rec + 4, 1u);
        atomicAdd(rec + 5, 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0 && tile[0] == 0xFFFFFFFFu) sink[blockIdx.x] = tile[1];  // keeps the adds live
}

}  // namespace gg

extern "C" GG_API int gg_measure_shared_atomic_peak(gg_context* ctx, double* gatomics) {
    if (!ctx || !gatomics)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_measure_shared_atomic_peak needs a context and an output.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int blocks = ctx->sm_count * 8;
    uint32_t* sink = nullptr;
    GG_CHECK(gg::device_alloc(ctx, 4ull * blocks, (void**)&sink, "measurement sink"));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    int status = GG_OK;
    for (int rep = 0; rep < 6 && status == GG_OK; ++rep) {
        cudaEventRecord(e0, ctx->stream);
        gg::shared_red_kernel<<<blocks, 256, 0, ctx->stream>>>(sink, 777u + rep);
        cudaEventRecord(e1, ctx->stream);
        status = gg::cuda_status(cudaEventSynchronize(e1), "shared atomic peak measurement");
        float ms = 0.0f;
        if (status == GG_OK) cudaEventElapsedTime(&ms, e0, e1);
        double adds = 6.0 * (double)blocks * 256.0 * gg::kDeposits * 4.0;
        if (rep > 0 && ms > 0.0f) best = std::max(best, adds / (ms * 1e-3) / 1e9);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    gg::device_free(ctx, sink, 4ull * blocks);
    if (status != GG_OK) return status;
    *gatomics = best;
    return GG_OK;
}

extern "C" GG_API int gg_measure_atomic_peak(gg_context* ctx, uint32_t records, double* gatomics) {
    if (!ctx || !gatomics || records == 0)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_measure_atomic_peak needs a context, records and an output.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    uint32_t* sums = nullptr;
    const uint64_t bytes = (uint64_t)records * 24u;
    GG_CHECK(gg::device_alloc(ctx, bytes, (void**)&sums, "atomic measurement grid"));
    int status = gg::cuda_status(cudaMemsetAsync(sums, 0, bytes, ctx->stream), "atomic measurement grid");
    const int blocks = ctx->sm_count * 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    for (int rep = 0; rep < 6 && status == GG_OK; ++rep) {
        cudaEventRecord(e0, ctx->stream);
        gg::red_kernel<<<blocks, 256, 0, ctx->stream>>>(sums, records, 12345u + rep);
        cudaEventRecord(e1, ctx->stream);
        status = gg::cuda_status(cudaEventSynchronize(e1), "atomic peak measurement");
        float ms = 0.0f;
        if (status == GG_OK) cudaEventElapsedTime(&ms, e0, e1);
        double adds = 6.0 * (double)blocks * 256.0 * gg::kDeposits;
        if (rep > 0 && ms > 0.0f) best = std::max(best, adds / (ms * 1e-3) / 1e9);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    gg::device_free(ctx, sums, bytes);
    if (status != GG_OK) return status;
    *gatomics = best;
    return GG_OK;
}

extern "C" GG_API int gg_measure_fp32_peak(gg_context* ctx, double* tflops) {
    if (!ctx || !tflops) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_measure_fp32_peak needs a context and an output.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    float* sink = nullptr;
    GG_CHECK(gg::device_alloc(ctx, 1024, (void**)&sink, "measurement sink"));
    const int blocks = ctx->sm_count * 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    int status = GG_OK;
    for (int rep = 0; rep < 6 && status == GG_OK; ++rep) {
        cudaEventRecord(e0, ctx->stream);
        gg::ffma_kernel<<<blocks, 256, 0, ctx->stream>>>(0.999999f, 1e-7f, sink);
        cudaEventRecord(e1, ctx->stream);
        status = gg::cuda_status(cudaEventSynchronize(e1), "FP32 peak measurement");
        float ms = 0.0f;
        if (status == GG_OK) cudaEventElapsedTime(&ms, e0, e1);
        double flops = 2.0 * (double)blocks * 256.0 * gg::kChains * gg::kFmaIterations;
        if (rep > 0 && ms > 0.0f) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    gg::device_free(ctx, sink, 1024);
    if (status != GG_OK) return status;
    *tflops = best;
    return GG_OK;
}
