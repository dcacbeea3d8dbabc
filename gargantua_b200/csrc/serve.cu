// Serving: continuous batching of still requests onto the device.
//
// Device side. A wave is one persistent launch over a queue of ray chunks
// (chunk_rays consecutive pixels of one request) packed from every admitted
// request, with one queue per metric: Schwarzschild rays and Kerr rays run
// different integrators, so a warp works one queue at a time (half the
// warps start on each, then take the other). Each warp steals chunks with
// one atomic per chunk and keeps its 32 lanes busy: a lane whose ray ended
// is refilled from the warp's chunk (ballot + popc ranks the idle lanes) as
// soon as a quarter of the warp is idle, so long and short rays share warps
// without the 8x8-tile tail of the per-request kernel. Ray state stays in
// registers for the whole ray. Per-request counters are aggregated across
// the lanes of a warp that finish together (match_any + reduce) before one
// atomic per request. Rays over their drift budget after passing inside
// r = 4 are queued for an FP64 re-integration kernel that runs after the
// wave. The wave (counter reset, persistent kernel, FP64 pass) is captured
// once per slot into a CUDA graph and replayed; only the wave's descriptors
// are copied in before each replay.
//
// Host side. A scheduler thread admits submitted requests in arrival order
// while their device footprint fits the server's memory (the HBM admission
// the reference's MemoryBudget does before allocating, Budget.swift:6-22),
// builds their sweep tables in FP64 on a side stream, forms waves
// round-robin across admitted requests (so a small request that arrives
// behind a large one is packed into the next wave rather than queued behind
// it), keeps up to max_waves_in_flight waves on alternating streams so one
// wave's tail overlaps the next wave's start, and copies each finished
// request's pixels to its host buffer on a copy stream.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include "lanes.cuh"
#include "runtime.h"

namespace gg {

MarchParams make_params(gg_context* ctx, const gg_volume* vol, const MarchUniforms& u, const gg_sweep* sweep);
int launch_plain_image(const MarchParams& p, cudaStream_t stream, bool as_written);
int launch_bake_walk(const MarchParams& bake, const MarchParams& walk, ushort4* samples, BakedRay* headers,
                     uint32_t* overflow, unsigned long long* stats, cudaStream_t stream);

struct ServeRequest {
    MarchUniforms u;
    const float* camera_table;
    const float* sky_table;
    ushort4* color;
    ushort4* debug;
    unsigned long long* stats;  // steps, samples, fp64, rays, over budget, exhausted, captured, spare
    cudaTextureObject_t emission;  // the request's volume (0: no gas)
    cudaTextureObject_t velocity;
    uint32_t pad[2];
};
static_assert(sizeof(ServeRequest) == 256, "ServeRequest");

struct ServeChunk {
    uint32_t request, first, count, pad;
};

struct WaveHeader {
    uint32_t chunk_count[2];
    uint32_t heads[2];
    uint32_t flagged_count;
    uint32_t request_count;
    uint32_t pad[10];
};
static_assert(sizeof(WaveHeader) == 64, "WaveHeader");

struct WaveArgs {
    WaveHeader* header;
    const ServeRequest* requests;
    const ServeChunk* chunks0;
    const ServeChunk* chunks1;
    unsigned long long* flagged;
    uint32_t flagged_capacity;
    const float* sphere_table;
    const float4* blackbody;
    uint32_t fp64_all;         // GG_FP64_ALL_FLAGGED
    uint32_t steps_per_round;  // RK4 steps between refill checks
    uint32_t refill_idle;      // refill once this many lanes of a warp are idle
};

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kMaxRounds = 1u << 28;  // bound on a warp's rounds (each consumes work or a step)
constexpr uint32_t kMaxFillsPerRound = 64;
constexpr int kServeThreads = 128;

__device__ __forceinline__ void write_result(const ServeRequest& R, uint32_t pixel, const PixelResult& r) {
    R.color[pixel] = pack_half4(r.color.x, r.color.y, r.color.z, 1.0f);
    if (R.debug) R.debug[pixel] = pack_half4(r.drift, (float)r.steps, (float)r.outcome, 1.0f);
}

// Warp-aggregated per-request counters for the lanes that finished a ray
// this iteration. Every lane of the warp calls it.
__device__ __forceinline__ void account(const WaveArgs& a, bool finished, uint32_t req, const PixelResult& r,
                                        float budget, uint32_t lane) {
    unsigned fin = __ballot_sync(kFull, finished);
    if (!finished) return;
    unsigned peers = __match_any_sync(fin, req);
    uint32_t steps = __reduce_add_sync(peers, r.steps);
    uint32_t samples = __reduce_add_sync(peers, r.samples);
    uint32_t rays = __popc(peers);
    uint32_t over = __reduce_add_sync(peers, r.drift > budget ? 1u : 0u);
    uint32_t exhausted = __reduce_add_sync(peers, r.outcome == RayExhausted ? 1u : 0u);
    uint32_t captured = __reduce_add_sync(peers, r.outcome == RayCaptured ? 1u : 0u);
    if ((int)lane == __ffs(peers) - 1) {
        unsigned long long* st = a.requests[req].stats;
        if (steps) atomicAdd(st + 0, (unsigned long long)steps);
        if (samples) atomicAdd(st + 1, (unsigned long long)samples);
        atomicAdd(st + 3, (unsigned long long)rays);
        if (over) atomicAdd(st + 4, (unsigned long long)over);
        if (exhausted) atomicAdd(st + 5, (unsigned long long)exhausted);
        if (captured) atomicAdd(st + 6, (unsigned long long)captured);
    }
}

// Write a finished ray, or queue it for FP64 re-integration.
__device__ __forceinline__ void complete(const WaveArgs& a, uint32_t req, uint32_t pixel, const PixelResult& r) {
    const ServeRequest& R = a.requests[req];
    if (needs_fp64(R.u, r, a.fp64_all != 0u)) {
        uint32_t slot = atomicAdd(&a.header->flagged_count, 1u);
        if (slot < a.flagged_capacity) {
            a.flagged[slot] = ((unsigned long long)req << 32) | pixel;
            return;
        }
    }
    write_result(R, pixel, r);
}

template <int Kind> struct LaneOf;
template <> struct LaneOf<0> { typedef SLane<float> type; };
template <> struct LaneOf<1> { typedef KLane<float> type; };

template <int Kind>
__device__ void serve_queue(const WaveArgs& a, uint32_t lane) {
    const ServeChunk* chunks = Kind == 0 ? a.chunks0 : a.chunks1;
    const uint32_t nchunks = a.header->chunk_count[Kind];
    uint32_t* head = &a.header->heads[Kind];
    const unsigned lower = (1u << lane) - 1u;
    typename LaneOf<Kind>::type L;
    bool active = false;
    uint32_t req = 0, pixel = 0;
    uint32_t cursor = 0, chunk_end = 0, chunk_req = 0;
    bool drained = false;
    for (uint32_t round = 0; round < kMaxRounds; ++round) {
        // Refill idle lanes from the warp's chunk, stealing new chunks.
        for (uint32_t fill = 0; fill < kMaxFillsPerRound && !drained; ++fill) {
            unsigned idle = __ballot_sync(kFull, !active);
            if (idle == 0u) break;
            if (cursor >= chunk_end) {
                uint32_t c = 0;
                if (lane == 0) c = atomicAdd(head, 1u);
                c = __shfl_sync(kFull, c, 0);
                if (c >= nchunks) {
                    drained = true;
                    break;
                }
                ServeChunk ch = chunks[c];
                cursor = ch.first;
                chunk_end = ch.first + ch.count;
                chunk_req = ch.request;
            }
            uint32_t take = min((uint32_t)__popc(idle), chunk_end - cursor);
            uint32_t rank = __popc(idle & lower);
            bool sky_done = false;
            PixelResult r{};
            if (!active && rank < take) {
                req = chunk_req;
                pixel = cursor + rank;
                const ServeRequest& R = a.requests[req];
                uint32_t w = R.u.resolution.x;
                float3 dir = camera_direction(R.u, pixel % w, pixel / w);
                float3 origin = to_f3(R.u.cameraPosition);
                if constexpr (Kind == 0) {
                    float3 sky;
                    SweepTables t{a.sphere_table, R.camera_table, R.sky_table};
                    if (s_init(L, origin, dir, R.u, t, &sky)) {
                        r = sky_only_result(sky, R.u, a.blackbody);
                        write_result(R, pixel, r);
                        sky_done = true;
                    } else {
                        active = true;
                    }
                } else {
                    k_init(L, origin, dir, R.u);
                    active = true;
                }
            }
            account(a, sky_done, req, r, 1e30f, lane);
            cursor += take;
        }
        unsigned act = __ballot_sync(kFull, active);
        if (act == 0u) {
            if (drained) break;
            continue;
        }
        // Advance every active lane, a few steps per round.
        for (uint32_t it = 0; it < a.steps_per_round; ++it) {
            bool finished = false;
            PixelResult r{};
            float budget = 0.0f;
            if (active) {
                const ServeRequest& R = a.requests[req];
                if constexpr (Kind == 0) {
                    finished = s_step(L, R.u, R.emission, R.velocity, R.emission != 0);
                    if (finished) {
                        SweepTables t{a.sphere_table, R.camera_table, R.sky_table};
                        r = s_finish(L, R.u, t, a.blackbody);
                    }
                } else {
                    finished = k_step(L, R.u, R.emission, R.velocity, R.emission != 0);
                    if (finished) r = k_finish(L, R.u, a.blackbody);
                }
                budget = R.u.driftBudget;
                if (finished) {
                    complete(a, req, pixel, r);
                    active = false;
                }
            }
            account(a, finished, req, r, budget, lane);
            act = __ballot_sync(kFull, active);
            if (act == 0u) break;
            if (!drained && (uint32_t)__popc(~act) >= a.refill_idle) break;
        }
    }
}

// The chunk schedule (GG_SCHEDULE_CHUNKS): a warp steals a chunk, gives
// each lane one of its rays (32 at a time) and runs every lane to the end of
// its ray with no warp-level operation inside the step loop, like a
// thread-per-pixel image kernel; one warp-aggregated account per 32 rays.
// The request's uniforms are copied to registers once per chunk, so the
// step loop reads them as it would read kernel parameters.
template <int Kind>
__device__ void serve_chunks(const WaveArgs& a, uint32_t lane) {
    const ServeChunk* chunks = Kind == 0 ? a.chunks0 : a.chunks1;
    const uint32_t nchunks = a.header->chunk_count[Kind];
    uint32_t* head = &a.header->heads[Kind];
    for (uint32_t round = 0; round < kMaxRounds; ++round) {
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(head, 1u);
        c = __shfl_sync(kFull, c, 0);
        if (c >= nchunks) break;
        const ServeChunk ch = chunks[c];
        const ServeRequest& R = a.requests[ch.request];
        const MarchUniforms u = R.u;
        const cudaTextureObject_t em = R.emission, vel = R.velocity;
        for (uint32_t base = 0; base < ch.count; base += 32u) {
            const uint32_t k = base + lane;
            const bool has = k < ch.count;
            PixelResult r{};
            if (has) {
                const uint32_t pixel = ch.first + k;
                const uint32_t w = u.resolution.x;
                float3 dir = camera_direction(u, pixel % w, pixel / w);
                float3 origin = to_f3(u.cameraPosition);
                typename LaneOf<Kind>::type L;
                if constexpr (Kind == 0) {
                    float3 sky;
                    SweepTables t{a.sphere_table, R.camera_table, R.sky_table};
                    if (s_init(L, origin, dir, u, t, &sky)) {
                        r = sky_only_result(sky, u, a.blackbody);
                        write_result(R, pixel, r);
                    } else {
                        for (uint32_t s = 0; s <= STEP_CAP_STILL; ++s)
                            if (s_step(L, u, em, vel, em != 0)) break;
                        r = s_finish(L, u, t, a.blackbody);
                        complete(a, ch.request, pixel, r);
                    }
                } else {
                    k_init(L, origin, dir, u);
                    for (uint32_t s = 0; s <= STEP_CAP_STILL; ++s)
                        if (k_step(L, u, em, vel, em != 0)) break;
                    r = k_finish(L, u, a.blackbody);
                    complete(a, ch.request, pixel, r);
                }
            }
            account(a, has, ch.request, r, u.driftBudget, lane);
        }
    }
}

// One persistent kernel per metric and schedule; a wave runs the two
// metrics side by side. All four are held to 7 blocks per SM (at most 72
// registers, with a few dozen bytes of spills): the step is bound by
// instruction issue, and more warps per SM keep the issue slots fuller.
// Measured on the mixed stream (64 requests, A/B on one box): 4 blocks per
// SM 76.9 G ray-steps/s, 5 78.7, 6 79.6, 7 80.4, 8 78.1 (its spills grow to
// 80 bytes); the compiler unbounded picks 119 registers, 4 blocks. Compiling
// every schedule under the same bound keeps their arithmetic, and so their
// pixels, identical.
constexpr int kServeBlocksPerSM = 7;

__global__ void __launch_bounds__(kServeThreads, kServeBlocksPerSM) serve_schwarzschild_kernel(WaveArgs a) {
    serve_queue<0>(a, threadIdx.x & 31u);
}

__global__ void __launch_bounds__(kServeThreads, kServeBlocksPerSM) serve_kerr_kernel(WaveArgs a) {
    serve_queue<1>(a, threadIdx.x & 31u);
}

__global__ void __launch_bounds__(kServeThreads, kServeBlocksPerSM) serve_schwarzschild_chunks_kernel(WaveArgs a) {
    serve_chunks<0>(a, threadIdx.x & 31u);
}

__global__ void __launch_bounds__(kServeThreads, kServeBlocksPerSM) serve_kerr_chunks_kernel(WaveArgs a) {
    serve_chunks<1>(a, threadIdx.x & 31u);
}

// FP64 re-integration of the wave's flagged rays.
__global__ void __launch_bounds__(128) serve_reintegrate_kernel(WaveArgs a) {
    const uint32_t n = min(a.header->flagged_count, a.flagged_capacity);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned long long e = a.flagged[i];
        uint32_t req = (uint32_t)(e >> 32), pixel = (uint32_t)e;
        const ServeRequest& R = a.requests[req];
        MarchParams p{};
        p.u = R.u;
        p.tables = SweepTables{a.sphere_table, R.camera_table, R.sky_table};
        p.emission = R.emission;
        p.velocity = R.velocity;
        p.blackbody = a.blackbody;
        uint32_t w = R.u.resolution.x;
        PixelResult r = shade_pixel_lane<double>(p, pixel % w, pixel / w);
        write_result(R, pixel, r);
        atomicAdd(R.stats + 2, 1ull);
    }
}

// ------------------------------------------------------------------- host

static double now_seconds() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// MarchPass.uniforms (MarchPass.swift:67-98) for a request, with the orbit
// camera's basis in float as Camera.swift computes it.
static MarchUniforms request_uniforms(const gg_request& q) {
    MarchUniforms u{};
    float c = cosf(q.elevation);
    float px = q.distance * (c * cosf(q.azimuth)), py = q.distance * (c * sinf(q.azimuth)), pz = q.distance * sinf(q.elevation);
    float inv = 1.0f / sqrtf(px * px + py * py + pz * pz);
    float fx = -px * inv, fy = -py * inv, fz = -pz * inv;
    // right = normalize(cross(forward, z)), up = cross(right, forward)
    float rx = fy, ry = -fx, rz = 0.0f;
    float rn = 1.0f / sqrtf(rx * rx + ry * ry);
    rx *= rn;
    ry *= rn;
    float ux = ry * fz - rz * fy, uy = rz * fx - rx * fz, uz = rx * fy - ry * fx;
    u.cameraPosition = {px, py, pz, 0.0f};
    u.cameraRight = {rx, ry, rz, 0.0f};
    u.cameraUp = {ux, uy, uz, 0.0f};
    u.cameraForward = {fx, fy, fz, 0.0f};
    float t = tanf(q.fov_y * 0.5f);
    u.tanHalfFov = {t * (float)q.width / (float)q.height, t};
    u.resolution = {q.width, q.height};
    u.tileOrigin = {0u, 0u};
    u.volumeHalfExtent = VOLUME_HALF_EXTENT;
    u.opacityScale = VOLUME_OPACITY;
    u.starBrightness = (q.flags & GG_REQUEST_NO_STARS) ? 0.0f : STAR_BRIGHTNESS;
    const bool interactive = q.step_cap <= STEP_CAP_INTERACTIVE;
    u.driftBudget = interactive ? DRIFT_BUDGET_INTERACTIVE : DRIFT_BUDGET_STILL;
    u.starSeed = q.star_seed;
    u.redshift = (q.flags & GG_REQUEST_NO_REDSHIFT) ? 0u : 1u;
    u.bakeSpacing = 0.0f;
    u.bakeCapacity = BAKE_SAMPLES;
    u.spin = q.spin;
    u.jitter = {0.0f, 0.0f};
    GeodesicSettings& g = u.geodesic;
    g.stepFactor = STEP_RADIUS_FACTOR;
    g.stepMin = STEP_MIN;
    g.stepMax = STEP_MAX;
    g.captureRadius = R_CAPTURE;
    g.escapeRadius = R_ESCAPE;
    // Kerr has no sphere jump; a camera beyond R_ESCAPE would escape on its
    // first step, so its escape radius moves out with it.
    if (q.spin > 0.0f) g.escapeRadius = fmaxf(R_ESCAPE, q.distance + 10.0f);
    g.stepCap = q.step_cap;
    g.emptyStepFactor = interactive ? STEP_FACTOR_EMPTY_INTERACTIVE : STEP_FACTOR_EMPTY_STILL;
    g.emptyStepMax = interactive ? STEP_MAX_EMPTY_INTERACTIVE : STEP_MAX_EMPTY_STILL;
    return u;
}

struct ServedRequest {
    uint64_t ticket = 0;
    gg_request q{};
    MarchUniforms u{};
    gg_sweep sweep;
    ushort4* d_color = nullptr;
    ushort4* d_debug = nullptr;
    // GG_REQUEST_BAKE: the bake storage (BakePass.swift:31-38), its
    // overflow count, and whether the bake and walk were launched.
    bool bake = false;
    ushort4* d_samples = nullptr;
    BakedRay* d_headers = nullptr;
    uint32_t* d_overflow = nullptr;
    cudaEvent_t baked = nullptr;
    unsigned long long* d_stats = nullptr;  // 8 u64 then a MarchCounters
    uint64_t footprint = 0;
    uint32_t rays = 0;
    uint32_t next_ray = 0;
    int waves_pending = 0;
    bool copying = false;
    bool done = false;
    cudaEvent_t copied = nullptr;
    unsigned long long host_stats[10] = {};
    gg_request_result result{};
};

struct WaveSlot {
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;   // second branch of the wave graph
    cudaStream_t fp64 = nullptr;   // the FP64 re-integration pass
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaEvent_t fp64_done = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
    cudaGraphExec_t graph = nullptr;
    char* device = nullptr;  // header, requests, chunks0, chunks1, flagged
    char* host = nullptr;    // pinned staging for the descriptors
    bool busy = false;
    std::vector<std::shared_ptr<ServedRequest>> members;
    WaveArgs args{};
};

}  // namespace gg

struct gg_server {
    gg_context* ctx = nullptr;
    const gg_volume* vol = nullptr;
    gg_server_config cfg{};
    uint32_t max_requests = 1024;
    uint32_t max_chunks = 0;
    uint32_t flagged_capacity = 0;
    uint64_t slot_bytes = 0;
    int grid_s = 0, grid_k = 0;
    cudaStream_t build = nullptr, copy = nullptr, plain = nullptr;
    // The server's own stream-ordered pool, keeping up to memory_bytes mapped
    // between requests so freeing one request's targets and allocating the
    // next costs no page mapping at synchronisation points.
    cudaMemPool_t pool = nullptr;
    cudaEvent_t built = nullptr, origin = nullptr;
    std::vector<gg::WaveSlot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<gg::ServedRequest>> pending;
    std::vector<std::shared_ptr<gg::ServedRequest>> admitted;
    std::map<uint64_t, std::shared_ptr<gg::ServedRequest>> all;
    uint64_t next_ticket = 1;
    uint64_t memory_used = 0;
    bool stop = false;
    int fatal = GG_OK;
    std::string fatal_sentence;
    int injected = GG_OK;  // gg_server_inject_fault: the next device call "fails" with this status
    std::thread worker;
    // total_launches: kernels launched (each wave's two persistent kernels and
    // its FP64 pass, one sweep-table build per admission round (per 128
    // Schwarzschild requests), two per bake request, one
    // image kernel per request in the plain modes).
    uint64_t total_requests = 0, total_steps = 0, total_launches = 0;
    std::vector<std::pair<double, double>> intervals;  // wave device intervals, seconds after `origin`
    int next_slot = 0;
};

namespace gg {

static uint64_t slot_offset_requests() { return sizeof(WaveHeader); }
static uint64_t slot_offset_chunks0(const gg_server* s) { return slot_offset_requests() + (uint64_t)s->max_requests * sizeof(ServeRequest); }
static uint64_t slot_offset_chunks1(const gg_server* s) { return slot_offset_chunks0(s) + (uint64_t)s->max_chunks * sizeof(ServeChunk); }
static uint64_t slot_offset_flagged(const gg_server* s) { return slot_offset_chunks1(s) + (uint64_t)s->max_chunks * sizeof(ServeChunk); }

// The wave graph: fork, the Schwarzschild and Kerr persistent kernels side
// by side, join. The FP64 pass is launched outside the graph on its own
// stream so it overlaps the next wave.
static int capture_wave_graph(gg_server* s, WaveSlot& w) {
    cudaGraph_t g = nullptr;
    GG_CUDA(cudaStreamBeginCapture(w.stream, cudaStreamCaptureModeThreadLocal), "wave capture");
    GG_CUDA(cudaEventRecord(w.fork, w.stream), "wave capture");
    GG_CUDA(cudaStreamWaitEvent(w.side, w.fork, 0), "wave capture");
    if (s->cfg.schedule == GG_SCHEDULE_LANE_REFILL) {
        serve_schwarzschild_kernel<<<s->grid_s, kServeThreads, 0, w.side>>>(w.args);
        serve_kerr_kernel<<<s->grid_k, kServeThreads, 0, w.stream>>>(w.args);
    } else {
        serve_schwarzschild_chunks_kernel<<<s->grid_s, kServeThreads, 0, w.side>>>(w.args);
        serve_kerr_chunks_kernel<<<s->grid_k, kServeThreads, 0, w.stream>>>(w.args);
    }
    GG_CUDA(cudaEventRecord(w.join, w.side), "wave capture");
    GG_CUDA(cudaStreamWaitEvent(w.stream, w.join, 0), "wave capture");
    cudaError_t e = cudaStreamEndCapture(w.stream, &g);
    GG_CUDA(e, "wave capture");
    e = cudaGraphInstantiate(&w.graph, g, 0);
    cudaGraphDestroy(g);
    GG_CUDA(e, "wave graph instantiate");
    return GG_OK;
}

// The volume a request marches: its own, or the server's.
static const gg_volume* request_volume(const gg_server* s, const ServedRequest& r) {
    return r.q.volume ? r.q.volume : s->vol;
}

// The per-request baselines: one request at a time through an image kernel.
static bool serial(const gg_server* s) { return s->cfg.mode != GG_SERVE_BATCHED; }

static int admit(gg_server* s, const std::shared_ptr<ServedRequest>& r) {
    gg::Range range("serve: admit");
    const uint64_t px = r->rays;
    GG_CUDA(cudaMallocFromPoolAsync((void**)&r->d_color, px * 8u, s->pool, s->build), "request target");
    if (r->q.debug_output)
        GG_CUDA(cudaMallocFromPoolAsync((void**)&r->d_debug, px * 8u, s->pool, s->build), "request debug target");
    GG_CUDA(cudaMallocFromPoolAsync((void**)&r->d_stats, 128, s->pool, s->build), "request counters");
    GG_CUDA(cudaMemsetAsync(r->d_stats, 0, 128, s->build), "request counters");
    if (r->bake) {
        GG_CUDA(cudaMallocFromPoolAsync((void**)&r->d_samples, px * BAKE_SAMPLES * 8u, s->pool, s->build),
                "request bake samples");
        GG_CUDA(cudaMallocFromPoolAsync((void**)&r->d_headers, px * 16u, s->pool, s->build), "request bake headers");
        GG_CUDA(cudaMallocFromPoolAsync((void**)&r->d_overflow, 4u, s->pool, s->build), "request bake overflow");
        GG_CUDA(cudaMemsetAsync(r->d_overflow, 0, 4u, s->build), "request bake overflow");
        // The walk writes colour only: the debug target, if asked for, stays zero.
        if (r->d_debug) GG_CUDA(cudaMemsetAsync(r->d_debug, 0, px * 8u, s->build), "request debug target");
    }
    if (r->q.spin == 0.0f) {
        GG_CUDA(cudaMallocFromPoolAsync((void**)&r->sweep.camera, SWEEP_TABLE_SIZE * sizeof(float), s->pool, s->build),
                "camera table");
        GG_CUDA(cudaMallocFromPoolAsync((void**)&r->sweep.sky, SWEEP_TABLE_SIZE * sizeof(float), s->pool, s->build),
                "sky table");
        // Its tables are built with those of the other requests admitted
        // in the same round (build_admitted_tables).
    }
    r->result.admitted = now_seconds();
    return GG_OK;
}

// The camera and sky tables of every Schwarzschild request admitted in one
// round, in one launch on the build stream (per 128 requests), then each
// request's uniforms take its tables (DeflectionTables.apply).
static int build_admitted_tables(gg_server* s, const std::vector<std::shared_ptr<ServedRequest>>& round) {
    std::vector<double> radii;
    std::vector<gg_sweep*> sweeps;
    for (auto& r : round)
        if (r->q.spin == 0.0f) {
            radii.push_back((double)r->q.distance);
            sweeps.push_back(&r->sweep);
        }
    if (radii.empty()) return GG_OK;
    GG_CHECK(sweep_build_batch(s->ctx, s->build, radii.data(), sweeps.data(), (int)radii.size()));
    s->total_launches += (radii.size() + 127u) / 128u;
    for (auto& r : round)
        if (r->q.spin == 0.0f) sweep_apply(s->ctx, &r->sweep, &r->u);
    return GG_OK;
}

static void release(gg_server* s, ServedRequest& r) {
    if (r.bake) {
        // An admission that failed part-way leaves some of these null.
        if (r.d_samples) cudaFreeAsync(r.d_samples, s->copy);
        if (r.d_headers) cudaFreeAsync(r.d_headers, s->copy);
        if (r.d_overflow) cudaFreeAsync(r.d_overflow, s->copy);
        r.d_samples = nullptr;
        r.d_headers = nullptr;
        r.d_overflow = nullptr;
        if (r.baked) cudaEventDestroy(r.baked);
        r.baked = nullptr;
    }
    cudaFreeAsync(r.d_color, s->copy);
    if (r.d_debug) cudaFreeAsync(r.d_debug, s->copy);
    cudaFreeAsync(r.d_stats, s->copy);
    r.d_color = nullptr;
    r.d_debug = nullptr;
    r.d_stats = nullptr;
    if (r.sweep.camera) {
        cudaFreeAsync(r.sweep.camera, s->copy);
        cudaFreeAsync(r.sweep.sky, s->copy);
        r.sweep.camera = r.sweep.sky = nullptr;
    }
}

// Start the copy of a request whose rays are all done.
static int start_copy(gg_server* s, ServedRequest& r, cudaEvent_t after) {
    if (after) GG_CUDA(cudaStreamWaitEvent(s->copy, after, 0), "copy ordering");
    const uint64_t px = r.rays;
    GG_CUDA(cudaMemcpyAsync(r.q.output, r.d_color, px * 8u, cudaMemcpyDeviceToHost, s->copy), "request readback");
    if (r.d_debug)
        GG_CUDA(cudaMemcpyAsync(r.q.debug_output, r.d_debug, px * 8u, cudaMemcpyDeviceToHost, s->copy), "request readback");
    GG_CUDA(cudaMemcpyAsync(r.host_stats, r.d_stats, 80, cudaMemcpyDeviceToHost, s->copy), "request counters");
    GG_CUDA(cudaEventCreateWithFlags(&r.copied, cudaEventDisableTiming), "copy event");
    GG_CUDA(cudaEventRecord(r.copied, s->copy), "copy event");
    r.copying = true;
    return GG_OK;
}

// A GG_REQUEST_BAKE request: the bake of every row at the request's step
// policy and BakePass.spacing (BakePass.swift:50-52) for its volume's size,
// then the walk through that volume into its colour target, on `stream`
// after the tables are built; its copy follows. Its rays join no wave.
static int launch_bake(gg_server* s, ServedRequest& r, cudaStream_t stream, cudaEvent_t* done) {
    gg_context* ctx = s->ctx;
    const gg_volume* vol = request_volume(s, r);
    GG_CUDA(cudaStreamWaitEvent(stream, s->built, 0), "bake ordering");
    MarchUniforms ub = r.u;
    ub.bakeSpacing = (float)(2.0 * VOLUME_HALF_EXTENT / (double)(vol ? vol->size : 128u) * BAKE_SPACING_VOXELS);
    ub.bakeCapacity = BAKE_SAMPLES;
    MarchParams pb = make_params(ctx, nullptr, ub, &r.sweep);
    MarchParams pw = make_params(ctx, vol, ub, nullptr);
    pw.color = r.d_color;
    GG_CHECK(launch_bake_walk(pb, pw, r.d_samples, r.d_headers, r.d_overflow, r.d_stats, stream));
    GG_CUDA(cudaEventCreateWithFlags(&r.baked, cudaEventDisableTiming), "bake event");
    GG_CUDA(cudaEventRecord(r.baked, stream), "bake event");
    r.next_ray = r.rays;
    *done = r.baked;
    return GG_OK;
}

// Pack the next wave into slot w from the admitted requests, round-robin.
static bool form_wave(gg_server* s, WaveSlot& w) {
    std::vector<std::shared_ptr<ServedRequest>> cands;
    for (auto& r : s->admitted)
        if (r->next_ray < r->rays) cands.push_back(r);
    if (cands.empty()) return false;
    WaveHeader* hdr = reinterpret_cast<WaveHeader*>(w.host);
    std::memset(hdr, 0, sizeof *hdr);
    ServeRequest* reqs = reinterpret_cast<ServeRequest*>(w.host + slot_offset_requests());
    ServeChunk* c0 = reinterpret_cast<ServeChunk*>(w.host + slot_offset_chunks0(s));
    ServeChunk* c1 = reinterpret_cast<ServeChunk*>(w.host + slot_offset_chunks1(s));
    const uint32_t chunk = s->cfg.chunk_rays;
    uint64_t budget = s->cfg.wave_rays;
    w.members.clear();
    std::vector<uint32_t> local(cands.size(), UINT32_MAX);
    bool progress = true;
    while (budget > 0 && progress) {
        progress = false;
        const uint64_t share = std::max<uint64_t>(chunk, budget / cands.size());
        for (size_t i = 0; i < cands.size() && budget > 0; ++i) {
            ServedRequest& r = *cands[i];
            if (r.next_ray >= r.rays) continue;
            if (local[i] == UINT32_MAX) {
                if (hdr->request_count >= s->max_requests) continue;
                local[i] = hdr->request_count++;
                ServeRequest& d = reqs[local[i]];
                std::memset(&d, 0, sizeof d);
                d.u = r.u;
                d.camera_table = r.sweep.camera;
                d.sky_table = r.sweep.sky;
                d.color = r.d_color;
                d.debug = r.d_debug;
                d.stats = r.d_stats;
                const gg_volume* vol = request_volume(s, r);
                d.emission = vol ? vol->emission_tex : 0;
                d.velocity = vol ? vol->velocity_tex : 0;
                w.members.push_back(cands[i]);
                r.waves_pending += 1;
            }
            const int kind = r.u.spin > 0.0f ? 1 : 0;
            uint64_t take = std::min<uint64_t>({share, budget, (uint64_t)(r.rays - r.next_ray)});
            while (take > 0 && hdr->chunk_count[kind] < s->max_chunks) {
                uint32_t n = (uint32_t)std::min<uint64_t>(chunk, take);
                ServeChunk& ch = (kind ? c1 : c0)[hdr->chunk_count[kind]++];
                ch.request = local[i];
                ch.first = r.next_ray;
                ch.count = n;
                ch.pad = 0;
                r.next_ray += n;
                take -= n;
                budget -= n;
                progress = true;
            }
        }
    }
    return hdr->request_count > 0;
}

static int launch_wave(gg_server* s, WaveSlot& w) {
    gg::Range range("serve: launch wave");
    WaveHeader* hdr = reinterpret_cast<WaveHeader*>(w.host);
    GG_CUDA(cudaStreamWaitEvent(w.stream, s->built, 0), "wave ordering");
    GG_CUDA(cudaMemcpyAsync(w.device, w.host, sizeof(WaveHeader) + hdr->request_count * sizeof(ServeRequest),
                            cudaMemcpyHostToDevice, w.stream),
            "wave upload");
    if (hdr->chunk_count[0])
        GG_CUDA(cudaMemcpyAsync(w.device + slot_offset_chunks0(s), w.host + slot_offset_chunks0(s),
                                hdr->chunk_count[0] * sizeof(ServeChunk), cudaMemcpyHostToDevice, w.stream),
                "wave upload");
    if (hdr->chunk_count[1])
        GG_CUDA(cudaMemcpyAsync(w.device + slot_offset_chunks1(s), w.host + slot_offset_chunks1(s),
                                hdr->chunk_count[1] * sizeof(ServeChunk), cudaMemcpyHostToDevice, w.stream),
                "wave upload");
    GG_CUDA(cudaEventRecord(w.start, w.stream), "wave event");
    GG_CUDA(cudaGraphLaunch(w.graph, w.stream), "wave launch");
    GG_CUDA(cudaEventRecord(w.stop, w.stream), "wave event");
    // FP64 pass after the wave, on its own stream: it overlaps the next wave.
    GG_CUDA(cudaStreamWaitEvent(w.fp64, w.stop, 0), "FP64 ordering");
    serve_reintegrate_kernel<<<s->ctx->sm_count * 2, 128, 0, w.fp64>>>(w.args);
    GG_CHECK(launch_status("FP64 re-integration"));
    GG_CUDA(cudaEventRecord(w.fp64_done, w.fp64), "wave event");
    w.busy = true;
    s->total_launches += 3;
    return GG_OK;
}

static int finish_wave(gg_server* s, WaveSlot& w) {
    gg::Range range("serve: finish wave");
    // The wave's device interval runs from its start to the end of its FP64
    // pass, which may overlap the next wave.
    float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f;
    GG_CUDA(cudaEventElapsedTime(&t0, s->origin, w.start), "wave timing");
    GG_CUDA(cudaEventElapsedTime(&t1, s->origin, w.stop), "wave timing");
    GG_CUDA(cudaEventElapsedTime(&t2, s->origin, w.fp64_done), "wave timing");
    t1 = std::max(t1, t2);
    s->intervals.emplace_back((double)t0 * 1e-3, (double)t1 * 1e-3);
    for (auto& r : w.members) {
        r->waves_pending -= 1;
        if (r->waves_pending == 0 && r->next_ray >= r->rays && !r->copying) GG_CHECK(start_copy(s, *r, w.fp64_done));
    }
    w.members.clear();
    w.busy = false;
    return GG_OK;
}

// The per-request baseline: one request at a time, plain FP32 image kernel.
// Runs with the server's mutex released, so it touches no shared server
// state: the launch's device interval is returned in *interval and the
// caller records it (and the launch count) once it holds the mutex again.
static int run_plain(gg_server* s, ServedRequest& r, std::pair<double, double>* interval) {
    gg::Range range("serve: per-request launch");
    gg_context* ctx = s->ctx;
    if (r.bake) {
        GG_CUDA(cudaEventRecord(s->slots[0].start, s->plain), "plain event");
        cudaEvent_t done = nullptr;
        GG_CHECK(launch_bake(s, r, s->plain, &done));
        GG_CUDA(cudaEventRecord(s->slots[0].stop, s->plain), "plain event");
        GG_CHECK(start_copy(s, r, s->slots[0].stop));
        GG_CUDA(cudaEventSynchronize(r.copied), "plain bake");
        float t0 = 0.0f, t1 = 0.0f;
        GG_CUDA(cudaEventElapsedTime(&t0, s->origin, s->slots[0].start), "plain timing");
        GG_CUDA(cudaEventElapsedTime(&t1, s->origin, s->slots[0].stop), "plain timing");
        *interval = std::make_pair((double)t0 * 1e-3, (double)t1 * 1e-3);
        return GG_OK;
    }
    GG_CUDA(cudaStreamWaitEvent(s->plain, s->built, 0), "plain ordering");
    MarchParams p = make_params(ctx, request_volume(s, r), r.u, r.q.spin == 0.0f ? &r.sweep : nullptr);
    p.color = r.d_color;
    p.debug = r.d_debug;
    p.target_width = r.q.width;
    p.target_height = r.q.height;
    p.counters = reinterpret_cast<MarchCounters*>(r.d_stats + 8);
    p.stats = r.d_stats;
    GG_CUDA(cudaEventRecord(s->slots[0].start, s->plain), "plain event");
    GG_CHECK(launch_plain_image(p, s->plain, s->cfg.mode == GG_SERVE_SERIAL_PLAIN_AS_WRITTEN));
    GG_CUDA(cudaEventRecord(s->slots[0].stop, s->plain), "plain event");
    r.next_ray = r.rays;
    GG_CHECK(start_copy(s, r, s->slots[0].stop));
    // Serial: the next request starts after this one's pixels are home.
    GG_CUDA(cudaEventSynchronize(r.copied), "plain march");
    float t0 = 0.0f, t1 = 0.0f;
    GG_CUDA(cudaEventElapsedTime(&t0, s->origin, s->slots[0].start), "plain timing");
    GG_CUDA(cudaEventElapsedTime(&t1, s->origin, s->slots[0].stop), "plain timing");
    *interval = std::make_pair((double)t0 * 1e-3, (double)t1 * 1e-3);
    return GG_OK;
}

static void complete_request(gg_server* s, ServedRequest& r) {
    r.result.finished = now_seconds();
    r.result.ray_steps = r.host_stats[0];
    r.result.samples = r.host_stats[1];
    r.result.fp64_rays = r.host_stats[2];
    if (serial(s) && !r.bake) {
        std::memcpy(&r.result.counters, &r.host_stats[8], sizeof(MarchCounters));
    } else if (r.bake) {
        r.result.counters.rays = r.rays;
        r.result.counters.exhausted = (uint32_t)r.host_stats[5];
        r.result.counters.captured = (uint32_t)r.host_stats[6];
    } else {
        r.result.counters.rays = (uint32_t)r.host_stats[3];
        r.result.counters.overDriftBudget = (uint32_t)r.host_stats[4];
        r.result.counters.exhausted = (uint32_t)r.host_stats[5];
        r.result.counters.captured = (uint32_t)r.host_stats[6];
    }
    r.result.status = GG_OK;
    cudaEventDestroy(r.copied);
    r.copied = nullptr;
    release(s, r);
    s->memory_used -= r.footprint;
    s->total_requests += 1;
    s->total_steps += r.result.ray_steps;
    r.done = true;
}

static void worker_loop(gg_server* s) {
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lock(s->mu);
    // Runs for the server's lifetime: until destroy() asks it to stop and
    // every submitted request has completed, or a device error.
    for (bool running = true; running;) {
        int status = GG_OK;
        // Admission in arrival order while the footprint fits.
        std::vector<std::shared_ptr<ServedRequest>> round;
        while (!s->pending.empty() && s->memory_used + s->pending.front()->footprint <= s->cfg.memory_bytes &&
               (!serial(s) || s->admitted.empty())) {
            auto r = s->pending.front();
            s->pending.pop_front();
            s->memory_used += r->footprint;
            status = admit(s, r);
            if (status != GG_OK) break;
            s->admitted.push_back(r);
            round.push_back(r);
        }
        if (status == GG_OK && !round.empty()) status = build_admitted_tables(s, round);
        if (status == GG_OK && !round.empty()) status = cuda_status(cudaEventRecord(s->built, s->build), "admission");
        // Launch work.
        if (status == GG_OK) {
            if (serial(s)) {
                for (auto& r : s->admitted)
                    if (r->next_ray < r->rays && status == GG_OK) {
                        std::pair<double, double> interval(0.0, 0.0);
                        lock.unlock();
                        status = run_plain(s, *r, &interval);
                        lock.lock();
                        if (status == GG_OK) {
                            s->total_launches += 1;
                            s->intervals.push_back(interval);
                        }
                    }
            } else {
                // Bake requests run beside the waves on their own stream.
                for (auto& r : s->admitted) {
                    if (!r->bake || r->baked || status != GG_OK) continue;
                    cudaEvent_t done = nullptr;
                    status = launch_bake(s, *r, s->plain, &done);
                    if (status == GG_OK) status = start_copy(s, *r, done);
                    if (status == GG_OK) s->total_launches += 2;
                }
                for (uint32_t k = 0; k < s->slots.size() && status == GG_OK; ++k) {
                    WaveSlot& w = s->slots[(s->next_slot + k) % s->slots.size()];
                    if (w.busy) continue;
                    if (!form_wave(s, w)) break;
                    status = launch_wave(s, w);
                    s->next_slot = (int)((&w - &s->slots[0]) + 1) % (int)s->slots.size();
                }
            }
        }
        // Retire finished waves and copies.
        bool any_busy = false;
        for (auto& w : s->slots) {
            if (!w.busy || status != GG_OK) continue;
            cudaError_t q = cudaEventQuery(w.fp64_done);
            if (q == cudaSuccess) status = finish_wave(s, w);
            else if (q != cudaErrorNotReady) status = cuda_status(q, "wave");
            else any_busy = true;
        }
        bool finished_any = false;
        for (auto it = s->admitted.begin(); it != s->admitted.end() && status == GG_OK;) {
            ServedRequest& r = **it;
            if (r.copying) {
                cudaError_t q = cudaEventQuery(r.copied);
                if (q == cudaSuccess) {
                    complete_request(s, r);
                    finished_any = true;
                    it = s->admitted.erase(it);
                    continue;
                }
                if (q != cudaErrorNotReady) status = cuda_status(q, "request readback");
            }
            ++it;
        }
        if (status == GG_OK && s->injected != GG_OK)
            status = fail(s->injected, "Injected fault: the scheduler's device call reported status %d.", s->injected);
        if (status != GG_OK) {
            s->fatal = status;
            s->fatal_sentence = gg_last_error();
            s->cv_done.notify_all();
            return;
        }
        if (finished_any) s->cv_done.notify_all();
        bool work_left = !s->pending.empty() || !s->admitted.empty() || any_busy;
        if (s->stop && !work_left) {
            running = false;
        } else if (work_left) {
            // Devices run asynchronously; poll at a short interval.
            s->cv_work.wait_for(lock, std::chrono::microseconds(50));
        } else {
            s->cv_work.wait(lock, [s] { return s->stop || !s->pending.empty(); });
        }
    }
}

}  // namespace gg

namespace gg {
void release_server_resources(gg_server* s);
}

using namespace gg;

extern "C" {

GG_API int gg_server_create(gg_context* ctx, const gg_volume* vol, const gg_server_config* config, gg_server** out) {
    if (!ctx || !out) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_server_create needs a context and an output.");
    *out = nullptr;
    if (vol && vol->ctx != ctx) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_server_create: volume from another context.");
    std::lock_guard<std::recursive_mutex> clock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    // Until it is handed out, a failure releases whatever was created.
    auto discard = [](gg_server* p) {
        gg::release_server_resources(p);
        delete p;
    };
    std::unique_ptr<gg_server, decltype(discard)> s(new gg_server(), discard);
    s->ctx = ctx;
    s->vol = vol;
    if (config) s->cfg = *config;
    if (s->cfg.mode != GG_SERVE_BATCHED && s->cfg.mode != GG_SERVE_SERIAL_PLAIN &&
        s->cfg.mode != GG_SERVE_SERIAL_PLAIN_AS_WRITTEN)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Unknown serving mode %d.", s->cfg.mode);
    if (s->cfg.steps_per_round == 0) s->cfg.steps_per_round = 8;
    if (s->cfg.refill_idle == 0) s->cfg.refill_idle = 8;
    if (s->cfg.steps_per_round > 64 || s->cfg.refill_idle > 32)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "steps_per_round %u or refill_idle %u is outside 1..64 / 1..32.",
                        s->cfg.steps_per_round, s->cfg.refill_idle);
    if (s->cfg.fp64_policy != GG_FP64_ESCAPING && s->cfg.fp64_policy != GG_FP64_ALL_FLAGGED)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Unknown FP64 policy %u.", s->cfg.fp64_policy);
    if (s->cfg.schedule != GG_SCHEDULE_CHUNKS && s->cfg.schedule != GG_SCHEDULE_LANE_REFILL)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Unknown schedule %u.", s->cfg.schedule);
    if (s->cfg.memory_bytes == 0) s->cfg.memory_bytes = (ctx->budget - ctx->used) / 4;
    if (ctx->used + s->cfg.memory_bytes > ctx->budget)
        return gg::fail(GG_ERR_OVER_BUDGET, "The server asks for %llu bytes but the budget has %llu left.",
                        (unsigned long long)s->cfg.memory_bytes, (unsigned long long)(ctx->budget - ctx->used));
    if (s->cfg.wave_rays == 0) s->cfg.wave_rays = 4u << 20;
    if (s->cfg.chunk_rays == 0) s->cfg.chunk_rays = 32;
    if (s->cfg.max_waves_in_flight == 0) s->cfg.max_waves_in_flight = 6;
    if (s->cfg.max_waves_in_flight > 8) s->cfg.max_waves_in_flight = 8;
    if (s->cfg.chunk_rays < 32 || s->cfg.chunk_rays > 65536)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "chunk_rays %u is outside 32..65536.", s->cfg.chunk_rays);
    s->max_chunks = s->cfg.wave_rays / s->cfg.chunk_rays + 1024;
    s->flagged_capacity = s->cfg.wave_rays / 8;
    s->slot_bytes = gg::slot_offset_flagged(s.get()) + (uint64_t)s->flagged_capacity * 8u;
    int blocks = 0;
    const bool refill = s->cfg.schedule == GG_SCHEDULE_LANE_REFILL;
    GG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &blocks, refill ? (const void*)gg::serve_schwarzschild_kernel : (const void*)gg::serve_schwarzschild_chunks_kernel,
                gg::kServeThreads, 0),
            "occupancy");
    s->grid_s = std::max(1, blocks) * ctx->sm_count;
    GG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &blocks, refill ? (const void*)gg::serve_kerr_kernel : (const void*)gg::serve_kerr_chunks_kernel,
                gg::kServeThreads, 0),
            "occupancy");
    s->grid_k = std::max(1, blocks) * ctx->sm_count;
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ctx->device;
        GG_CUDA(cudaMemPoolCreate(&s->pool, &props), "server memory pool");
        uint64_t keep = s->cfg.memory_bytes;
        GG_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep), "server memory pool");
    }
    GG_CUDA(cudaStreamCreateWithFlags(&s->build, cudaStreamNonBlocking), "server streams");
    GG_CUDA(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking), "server streams");
    GG_CUDA(cudaStreamCreateWithFlags(&s->plain, cudaStreamNonBlocking), "server streams");
    GG_CUDA(cudaEventCreateWithFlags(&s->built, cudaEventDisableTiming), "server events");
    GG_CUDA(cudaEventCreate(&s->origin), "server events");
    GG_CUDA(cudaEventRecord(s->built, s->build), "server events");
    GG_CUDA(cudaEventRecord(s->origin, s->build), "server events");
    const int nslots = serial(s.get()) ? 1 : (int)s->cfg.max_waves_in_flight;
    s->slots.resize(nslots);
    for (auto& w : s->slots) {
        GG_CUDA(cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking), "wave stream");
        GG_CUDA(cudaStreamCreateWithFlags(&w.side, cudaStreamNonBlocking), "wave stream");
        GG_CUDA(cudaStreamCreateWithFlags(&w.fp64, cudaStreamNonBlocking), "wave stream");
        GG_CUDA(cudaEventCreateWithFlags(&w.fork, cudaEventDisableTiming), "wave events");
        GG_CUDA(cudaEventCreateWithFlags(&w.join, cudaEventDisableTiming), "wave events");
        GG_CUDA(cudaEventCreate(&w.fp64_done), "wave events");
        GG_CUDA(cudaEventCreate(&w.start), "wave events");
        GG_CUDA(cudaEventCreate(&w.stop), "wave events");
        if (serial(s.get())) continue;
        GG_CHECK(gg::device_alloc(ctx, s->slot_bytes, (void**)&w.device, "wave descriptors"));
        GG_CUDA(cudaHostAlloc((void**)&w.host, gg::slot_offset_flagged(s.get()), cudaHostAllocDefault), "wave staging");
        w.args.header = reinterpret_cast<gg::WaveHeader*>(w.device);
        w.args.requests = reinterpret_cast<const gg::ServeRequest*>(w.device + gg::slot_offset_requests());
        w.args.chunks0 = reinterpret_cast<const gg::ServeChunk*>(w.device + gg::slot_offset_chunks0(s.get()));
        w.args.chunks1 = reinterpret_cast<const gg::ServeChunk*>(w.device + gg::slot_offset_chunks1(s.get()));
        w.args.flagged = reinterpret_cast<unsigned long long*>(w.device + gg::slot_offset_flagged(s.get()));
        w.args.flagged_capacity = s->flagged_capacity;
        w.args.sphere_table = ctx->sphere_table;
        w.args.blackbody = ctx->blackbody;
        w.args.fp64_all = s->cfg.fp64_policy == GG_FP64_ALL_FLAGGED ? 1u : 0u;
        w.args.steps_per_round = s->cfg.steps_per_round;
        w.args.refill_idle = s->cfg.refill_idle;
        GG_CHECK(gg::capture_wave_graph(s.get(), w));
    }
    GG_CUDA(cudaStreamSynchronize(s->build), "server set-up");
    ctx->used += s->cfg.memory_bytes;  // reserved for admitted requests
    s->worker = std::thread(gg::worker_loop, s.get());
    *out = s.release();
    return GG_OK;
}

GG_API void gg_server_destroy(gg_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    gg::release_server_resources(s);
    s->ctx->used -= std::min(s->ctx->used, s->cfg.memory_bytes);
    delete s;
}

}  // extern "C"

namespace gg {

// The device and host resources a server holds, whichever of them exist
// (a server whose creation failed part way holds some).
void release_server_resources(gg_server* s) {
    gg_context* ctx = s->ctx;
    cudaSetDevice(ctx->device);
    for (auto& w : s->slots) {
        if (w.stream) cudaStreamSynchronize(w.stream);
        if (w.fp64) cudaStreamSynchronize(w.fp64);  // the FP64 pass reads the slot's flagged list
        if (w.graph) cudaGraphExecDestroy(w.graph);
        if (w.device) gg::device_free(ctx, w.device, s->slot_bytes);
        if (w.host) cudaFreeHost(w.host);
        if (w.start) cudaEventDestroy(w.start);
        if (w.stop) cudaEventDestroy(w.stop);
        if (w.fork) cudaEventDestroy(w.fork);
        if (w.join) cudaEventDestroy(w.join);
        if (w.fp64_done) cudaEventDestroy(w.fp64_done);
        if (w.side) cudaStreamDestroy(w.side);
        if (w.fp64) cudaStreamDestroy(w.fp64);
        if (w.stream) cudaStreamDestroy(w.stream);
    }
    if (s->copy) cudaStreamSynchronize(s->copy);
    if (s->build) cudaStreamSynchronize(s->build);
    for (auto& r : s->admitted) gg::release(s, *r);
    if (s->copy) cudaStreamSynchronize(s->copy);
    if (s->built) cudaEventDestroy(s->built);
    if (s->origin) cudaEventDestroy(s->origin);
    if (s->build) cudaStreamDestroy(s->build);
    if (s->copy) cudaStreamDestroy(s->copy);
    if (s->plain) cudaStreamDestroy(s->plain);
    if (s->pool) cudaMemPoolDestroy(s->pool);
}

}  // namespace gg

extern "C" {

GG_API int gg_server_submit(gg_server* s, const gg_request* req, uint64_t* ticket) {
    if (!s || !req || !ticket) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_server_submit needs a server, a request and a ticket.");
    if (req->width == 0 || req->height == 0 || req->width > 16384 || req->height > 16384 ||
        (uint64_t)req->width * req->height > (1ull << 31))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Request size %ux%u is outside 1..16384.", req->width, req->height);
    if (req->step_cap == 0 || req->step_cap > STEP_CAP_STILL)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Step cap %u is outside 1..%u.", req->step_cap, STEP_CAP_STILL);
    if (!(req->spin >= 0.0f && req->spin < 1.0f))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Spin %g is outside [0, 1).", (double)req->spin);
    if (!(req->distance > VOLUME_HALF_EXTENT) || !(req->distance < 1e4f))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Camera distance %g is outside (%g, 1e4).", (double)req->distance,
                        (double)VOLUME_HALF_EXTENT);
    if (!(req->fov_y > 0.0f && req->fov_y < 3.1f)) return gg::fail(GG_ERR_INVALID_ARGUMENT, "Field of view %g is invalid.", (double)req->fov_y);
    if (!req->output) return gg::fail(GG_ERR_INVALID_ARGUMENT, "The request has no output buffer.");
    if (req->volume && req->volume->ctx != s->ctx)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "The request's volume belongs to another context.");
    const bool bake = (req->flags & GG_REQUEST_BAKE) != 0u;
    if (bake && req->spin != 0.0f)
        return gg::fail(GG_ERR_UNSUPPORTED, "The bake strategy is Schwarzschild only; spin %g was given.", (double)req->spin);
    auto r = std::make_shared<gg::ServedRequest>();
    r->q = *req;
    r->u = gg::request_uniforms(*req);
    r->rays = req->width * req->height;
    r->bake = bake;
    r->footprint = (uint64_t)r->rays * (req->debug_output ? 16u : 8u) + 128u + 2u * SWEEP_TABLE_SIZE * 4u;
    if (bake) r->footprint += (uint64_t)r->rays * (BAKE_SAMPLES * 8u + 16u) + 4u;
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->fatal != GG_OK) return gg::fail(s->fatal, "The server stopped after a device error: %s", s->fatal_sentence.c_str());
    if (r->footprint > s->cfg.memory_bytes)
        return gg::fail(GG_ERR_OVER_BUDGET, "A %ux%u request needs %llu bytes but the server has %llu.", req->width,
                        req->height, (unsigned long long)r->footprint, (unsigned long long)s->cfg.memory_bytes);
    r->ticket = s->next_ticket++;
    r->result.submitted = gg::now_seconds();
    s->pending.push_back(r);
    s->all[r->ticket] = r;
    *ticket = r->ticket;
    s->cv_work.notify_one();
    return GG_OK;
}

GG_API int gg_server_inject_fault(gg_server* s, int status) {
    if (!s || status == GG_OK) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_server_inject_fault needs a server and a status.");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->injected = status;
    }
    s->cv_work.notify_all();
    return GG_OK;
}

GG_API int gg_server_cancel(gg_server* s, uint64_t ticket) {
    if (!s) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_server_cancel needs a server.");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return gg::fail(GG_ERR_INVALID_ARGUMENT, "Unknown ticket %llu.", (unsigned long long)ticket);
    auto r = it->second;
    auto p = std::find(s->pending.begin(), s->pending.end(), r);
    if (p == s->pending.end())
        return gg::fail(GG_ERR_NOT_READY, "Request %llu is %s; it completes.", (unsigned long long)ticket,
                        r->done ? "already done" : "admitted and on the device");
    s->pending.erase(p);
    r->result.status = GG_ERR_CANCELLED;
    r->result.finished = gg::now_seconds();
    r->done = true;
    s->cv_done.notify_all();
    return GG_OK;
}

GG_API int gg_server_poll(gg_server* s, uint64_t ticket, int* done) {
    if (!s || !done) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_server_poll needs a server and an output.");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return gg::fail(GG_ERR_INVALID_ARGUMENT, "Unknown ticket %llu.", (unsigned long long)ticket);
    if (s->fatal != GG_OK) return gg::fail(s->fatal, "The server stopped after a device error: %s", s->fatal_sentence.c_str());
    *done = it->second->done ? 1 : 0;
    return GG_OK;
}

GG_API int gg_server_wait(gg_server* s, uint64_t ticket, double timeout_s, gg_request_result* result) {
    if (!s) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_server_wait needs a server.");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return gg::fail(GG_ERR_INVALID_ARGUMENT, "Unknown ticket %llu.", (unsigned long long)ticket);
    auto r = it->second;
    bool ok = s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s),
                                  [&] { return r->done || s->fatal != GG_OK; });
    if (s->fatal != GG_OK) return gg::fail(s->fatal, "The server stopped after a device error: %s", s->fatal_sentence.c_str());
    if (!ok) return gg::fail(GG_ERR_TIMEOUT, "Request %llu is not done after %g s.", (unsigned long long)ticket, timeout_s);
    if (result) *result = r->result;
    s->all.erase(it);
    if (r->result.status == GG_ERR_CANCELLED)
        return gg::fail(GG_ERR_CANCELLED, "Request %llu was cancelled before admission.", (unsigned long long)ticket);
    return GG_OK;
}

GG_API int gg_server_totals(gg_server* s, int reset, uint64_t* requests, uint64_t* ray_steps, uint64_t* launches,
                            double* busy_seconds, double* span_seconds) {
    if (!s) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_server_totals needs a server.");
    std::lock_guard<std::mutex> lock(s->mu);
    if (requests) *requests = s->total_requests;
    if (ray_steps) *ray_steps = s->total_steps;
    if (launches) *launches = s->total_launches;
    // Union of the launch intervals: waves on different streams overlap.
    std::vector<std::pair<double, double>> iv = s->intervals;
    std::sort(iv.begin(), iv.end());
    double busy = 0.0, end = -1e300, first = 1e300, last = -1e300;
    for (auto& p : iv) {
        double a = std::max(p.first, end);
        if (p.second > a) busy += p.second - a;
        end = std::max(end, p.second);
        first = std::min(first, p.first);
        last = std::max(last, p.second);
    }
    if (busy_seconds) *busy_seconds = busy;
    if (span_seconds) *span_seconds = iv.empty() ? 0.0 : last - first;
    if (reset) {
        s->total_requests = s->total_steps = s->total_launches = 0;
        s->intervals.clear();
    }
    return GG_OK;
}

}  // extern "C"
