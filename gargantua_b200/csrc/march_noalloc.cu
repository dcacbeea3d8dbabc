// gg_march_compensated_noalloc: the compensated image march for callers
// that must not allocate device memory while they render.
//
// Some hosts cannot call cudaMalloc once they are running: a renderer that
// hands the whole device to its own pool or caching allocator up front, a
// frame loop with a hard latency budget (cudaFree synchronises the whole
// device, and an allocation that fails mid-frame has no good recovery), or a
// plugin living inside another program that owns the memory budget. The
// regular gg_march grows its FP64 re-integration list with cudaMalloc the
// first time it sees a larger target; this variant keeps that list in a
// fixed array that is part of the library's image, so a call allocates
// nothing.
//
// The scratch is one file-scope __device__ array of NOALLOC_MAX_PIXELS + 64
// words (about 8 MiB); every GPU that loads the library holds it until the
// process exits. Host code cannot pass the array's name to a kernel (on the
// host it names a host-side stand-in, not device memory), so each call, with
// its device current, asks the runtime for the array's device address with
// cudaGetSymbolAddress. The first such lookup on a device loads the array
// (set-up); make that first call before any stream capture. While the
// context's stream is being captured the address recorded by the last
// uncaptured call on that device is used instead, so a capture never does
// the set-up; looking the address up again on the other calls keeps it
// right after a cudaDeviceReset, which may place the array elsewhere.
// Every call on a device shares the
// array and reuses what the last call left in it: each call zeroes the list
// counter on its stream before the march, and two calls whose work overlaps
// on the GPU (different streams or contexts on one device) race on the
// array, so serialise them.
#include <mutex>

#include "../../include/gargantua.h"
#include "march.cuh"
#include "runtime.h"

namespace gg {

MarchParams make_params(gg_context* ctx, const gg_volume* vol, const MarchUniforms& u, const gg_sweep* sweep);
int check_uniforms(gg_context* ctx, const MarchUniforms* u, const char* what);
int launch_compensated_image(const MarchParams& p, cudaStream_t stream, int sm_count);

// Largest target (width x height) the fixed list can serve: 1920x1080 fits.
constexpr uint32_t kNoAllocMaxPixels = NOALLOC_MAX_PIXELS;

// word 0: list length; words 64..: flagged target-local pixel indices.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocMaxPixels + 64];

constexpr int kMaxDevices = 64;
static std::mutex g_noalloc_mu;
static uint32_t* g_noalloc_address[kMaxDevices] = {};

// The array's device address on `device` (current). Looked up on every call
// made outside a stream capture; a call made while `stream` is capturing
// reuses the address the last uncaptured call on the device recorded.
static int noalloc_scratch(int device, cudaStream_t stream, uint32_t** out) {
    if (device < 0 || device >= kMaxDevices)
        return fail(GG_ERR_UNSUPPORTED, "Device %d is beyond the %d devices the fixed scratch tracks.", device, kMaxDevices);
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    GG_CUDA(cudaStreamIsCapturing(stream, &capture), "fixed scratch: capture status");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (capture == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "fixed scratch address");
        g_noalloc_address[device] = static_cast<uint32_t*>(p);
    } else if (!g_noalloc_address[device]) {
        return fail(GG_ERR_UNSUPPORTED,
                    "gg_march_compensated_noalloc: the first call on device %d must come before any stream capture.",
                    device);
    }
    *out = g_noalloc_address[device];
    return GG_OK;
}

}  // namespace gg

extern "C" GG_API int gg_march_compensated_noalloc(gg_context* ctx, const gg_volume* vol, const MarchUniforms* u,
                                                   gg_targets* targets, MarchCounters* counters) {
    if (!ctx || !targets) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_march_compensated_noalloc needs a context and targets.");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    GG_CHECK(gg::check_uniforms(ctx, u, "gg_march_compensated_noalloc"));
    if (vol && vol->ctx != ctx) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_march_compensated_noalloc: volume from another context.");
    const uint64_t pixels = (uint64_t)targets->width * targets->height;
    if (pixels > gg::kNoAllocMaxPixels)
        return gg::fail(GG_ERR_INVALID_ARGUMENT,
                        "gg_march_compensated_noalloc serves targets of at most %u pixels; %ux%u is %llu.",
                        gg::kNoAllocMaxPixels, targets->width, targets->height, (unsigned long long)pixels);
    uint32_t* scratch = nullptr;
    GG_CHECK(gg::noalloc_scratch(ctx->device, ctx->stream, &scratch));
    gg::MarchParams p = gg::make_params(ctx, vol, *u, &ctx->sweep);
    p.color = targets->color;
    p.debug = targets->debug;
    p.depth = targets->depth;
    p.motion = targets->motion;
    p.target_width = targets->width;
    p.target_height = targets->height;
    p.counters = ctx->counters;
    p.stats = ctx->stats;
    p.flagged_count = scratch;
    p.flagged = scratch + 64;
    p.flagged_capacity = (uint32_t)pixels;
    // The array keeps the previous call's contents: reset the list length.
    GG_CUDA(cudaMemsetAsync(scratch, 0, sizeof(uint32_t), ctx->stream), "fixed scratch reset");
    GG_CUDA(cudaMemsetAsync(ctx->counters, 0, sizeof(MarchCounters), ctx->stream), "counter reset");
    GG_CUDA(cudaMemsetAsync(ctx->stats, 0, 4 * sizeof(unsigned long long), ctx->stream), "stats reset");
    GG_CHECK(gg::launch_compensated_image(p, ctx->stream, ctx->sm_count));
    if (counters) {
        GG_CUDA(cudaMemcpyAsync(counters, ctx->counters, sizeof(MarchCounters), cudaMemcpyDeviceToHost, ctx->stream),
                "counter readback");
        GG_CUDA(cudaStreamSynchronize(ctx->stream), "gg_march_compensated_noalloc");
    }
    return GG_OK;
}
