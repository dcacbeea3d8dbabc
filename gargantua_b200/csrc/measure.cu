// Device peak measurement for the rooflines: FP32 FMA throughput.
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

}  // namespace gg

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
