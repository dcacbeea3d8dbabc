// gargantua: the command-line host over the C ABI (include/gargantua.h),
// the same options, refusals and exit codes as gargantua's own executable
// (Options.swift:36-154, Program.swift, Exit.swift:5-18): 64 for a usage
// error, 2 for an operational one, 0 on success.
//
//   gargantua --still out.png [--width W --height H] [--spin a]
//             [--camera az,el,d] [--seed S] [--preset small|default|max]
//             [--particles N] [--volume 96|128|192|256] [--sequence N]
//   gargantua bench [--preset p] [--spin a] [--strategy march|bake]
//   gargantua version | constants
//
// --still settles the disk (Still.swift:36-46), splats it exactly, serves
// the still as one request through the batched server (compensated FP32,
// 4096-step still policy), tone-maps it on the device and writes a PNG;
// --sequence adds N 960x540 interactive frames with the simulation
// advancing and the stochastic deposit (Still.swift:67-90). bench times
// every pass of the preset's scene, each call waited to completion
// (Bench.swift:27-45: 5 warm-ups, 30 timed; mean, p50, max), as one JSON
// object. validate holds the device to the goldens (Validate.swift:17-55)
// and prints their table: exit 0 when every golden it runs passes, 1 when
// one fails. The interactive window needs a display and has no counterpart
// here.
#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstdarg>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "gargantua.h"
#include "gargantua_constants.h"

namespace {

const char* kVersion = "0.1.0";
const char* kUsage =
    "usage: gargantua [--preset small|default|max] [--particles N] [--volume 96|128|192|256] [--seed S] "
    "[--strategy march|bake] [--fps-cap 30|60] [--no-upscale] [--still out.png --width W --height H] [--spin a] "
    "[--camera az,el,d] [--sequence N] | bench | validate | version | constants";

const char* kConstants =
#include "constants_text.h"
    ;

struct UsageError {
    std::string sentence;
};

struct OperationalError {
    std::string sentence;
};

struct Preset {
    const char* name;
    uint32_t particles, volume, march_w, march_h;
};

// Presets.swift:72-93.
const Preset kPresets[] = {{"small", 250000, 96, 640, 360},
                           {"default", 1000000, 128, 960, 540},
                           {"max", 4000000, 256, 960, 540}};

struct Options {
    std::string command = "interactive";
    std::string still_path;
    const Preset* preset = &kPresets[1];
    uint32_t particles = 0, volume = 0;  // 0: the preset's
    uint64_t seed = 1;
    std::string strategy = "march";
    uint32_t fps_cap = 60;
    bool upscale = true;
    uint32_t width = 3840, height = 2160;
    uint32_t sequence = 0;
    bool has_camera = false;
    double azimuth = 0.6, elevation = 0.32, distance = 52.0;
    double spin = 0.0;
};

bool parse_positive(const std::string& text, uint64_t* out) {
    if (text.empty() || text.size() > 19) return false;
    for (char c : text)
        if (c < '0' || c > '9') return false;
    *out = std::strtoull(text.c_str(), nullptr, 10);
    return *out > 0;
}

// Options.parse (Options.swift:60-154).
Options parse(int argc, char** argv) {
    Options o;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto value = [&](const std::string& flag) -> std::string {
            if (++i >= argc) throw UsageError{flag + " needs a value. " + kUsage};
            return argv[i];
        };
        auto integer = [&](const std::string& flag) -> uint32_t {
            const std::string text = value(flag);
            uint64_t n = 0;
            if (!parse_positive(text, &n) || n > 0xffffffffull)
                throw UsageError{flag + " needs a positive integer, not " + text + "."};
            return (uint32_t)n;
        };
        if (a == "bench" || a == "validate" || a == "version" || a == "constants") {
            o.command = a;
        } else if (a == "--preset") {
            const std::string name = value(a);
            o.preset = nullptr;
            for (const Preset& p : kPresets)
                if (name == p.name) o.preset = &p;
            if (!o.preset) throw UsageError{"unknown preset " + name + "; choose small, default or max."};
        } else if (a == "--particles") {
            o.particles = integer(a);
        } else if (a == "--volume") {
            const uint32_t v = integer(a);
            if (v != 96 && v != 128 && v != 192 && v != 256) throw UsageError{"volume must be 96, 128, 192 or 256."};
            o.volume = v;
        } else if (a == "--seed") {
            const std::string text = value(a);
            bool digits = !text.empty() && text.size() <= 20;
            for (char c : text) digits = digits && c >= '0' && c <= '9';
            errno = 0;
            const unsigned long long s = digits ? std::strtoull(text.c_str(), nullptr, 10) : 0;
            if (!digits || errno == ERANGE)
                throw UsageError{"seed must be an unsigned 64 bit integer, not " + text + "."};
            o.seed = s;
        } else if (a == "--strategy") {
            const std::string name = value(a);
            if (name != "march" && name != "bake") throw UsageError{"unknown strategy " + name + "; choose march or bake."};
            o.strategy = name;
        } else if (a == "--fps-cap") {
            const uint32_t cap = integer(a);
            if (cap != 30 && cap != 60) throw UsageError{"fps cap must be 30 or 60."};
            o.fps_cap = cap;
        } else if (a == "--no-upscale") {
            o.upscale = false;
        } else if (a == "--still") {
            o.command = "still";
            o.still_path = value(a);
        } else if (a == "--width") {
            o.width = integer(a);
        } else if (a == "--height") {
            o.height = integer(a);
        } else if (a == "--sequence") {
            o.sequence = integer(a);
        } else if (a == "--spin") {
            const std::string text = value(a);
            char* end = nullptr;
            const double s = std::strtod(text.c_str(), &end);
            if (end == text.c_str() || *end != '\0' || !(s >= 0.0 && s <= 0.998))
                throw UsageError{"spin must be between 0 and 0.998."};
            o.spin = s;
        } else if (a == "--camera") {
            const std::string text = value(a);
            std::vector<double> parts;
            size_t start = 0;
            while (start <= text.size()) {
                size_t comma = text.find(',', start);
                if (comma == std::string::npos) comma = text.size();
                const std::string piece = text.substr(start, comma - start);
                char* end = nullptr;
                const double v = std::strtod(piece.c_str(), &end);
                if (!piece.empty() && end != piece.c_str() && *end == '\0') parts.push_back(v);
                start = comma + 1;
            }
            if (parts.size() != 3 || !(parts[2] > 2.5 && parts[2] < 60.0))
                throw UsageError{"camera needs azimuth,elevation,distance with distance between 2.5 and 60."};
            o.has_camera = true;
            o.azimuth = parts[0];
            o.elevation = std::min(std::max(parts[1], -1.5), 1.5);  // OrbitCamera.from (Camera.swift:5-13)
            o.distance = parts[2];
        } else {
            throw UsageError{"unknown argument " + a + ". " + kUsage};
        }
    }
    return o;
}

void check(int status) {
    if (status != GG_OK) throw OperationalError{gg_last_error()};
}

// The orbit camera's basis in float, as the Swift host's SIMD3<Float>
// (Camera.swift:4-33), and MarchPass.uniforms (MarchPass.swift:67-98).
MarchUniforms march_uniforms(const Options& o, uint32_t w, uint32_t h, bool still, float drift_budget) {
    const float az = (float)o.azimuth, el = (float)o.elevation, d = (float)o.distance;
    const float c = std::cos(el);
    const float pos[3] = {d * (c * std::cos(az)), d * (c * std::sin(az)), d * std::sin(el)};
    const float len = std::sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
    const float fwd[3] = {-pos[0] / len, -pos[1] / len, -pos[2] / len};
    float right[3] = {fwd[1], -fwd[0], 0.0f};  // fwd x (0, 0, 1)
    const float rl = std::sqrt(right[0] * right[0] + right[1] * right[1]);
    right[0] /= rl;
    right[1] /= rl;
    const float up[3] = {right[1] * fwd[2] - right[2] * fwd[1], right[2] * fwd[0] - right[0] * fwd[2],
                         right[0] * fwd[1] - right[1] * fwd[0]};
    MarchUniforms u;
    std::memset(&u, 0, sizeof u);
    u.cameraPosition = {pos[0], pos[1], pos[2], 0.0f};
    u.cameraRight = {right[0], right[1], right[2], 0.0f};
    u.cameraUp = {up[0], up[1], up[2], 0.0f};
    u.cameraForward = {fwd[0], fwd[1], fwd[2], 0.0f};
    const float tan_half = std::tan((float)(50.0 * M_PI / 180.0) * 0.5f);
    u.tanHalfFov = {tan_half * (float)w / (float)h, tan_half};
    u.resolution = {w, h};
    u.tileOrigin = {0u, 0u};
    u.volumeHalfExtent = VOLUME_HALF_EXTENT;
    u.opacityScale = VOLUME_OPACITY;
    u.starBrightness = STAR_BRIGHTNESS;
    u.driftBudget = drift_budget;
    u.starSeed = (uint32_t)o.seed;
    u.redshift = 1u;
    u.bakeCapacity = BAKE_SAMPLES;
    u.spin = (float)o.spin;
    // Schwarzschild.Settings .interactive / .still (Schwarzschild.swift:167-172).
    u.geodesic = {STEP_RADIUS_FACTOR, STEP_MIN, STEP_MAX, R_CAPTURE, R_ESCAPE,
                  still ? STEP_CAP_STILL : STEP_CAP_INTERACTIVE,
                  still ? STEP_FACTOR_EMPTY_STILL : STEP_FACTOR_EMPTY_INTERACTIVE,
                  still ? STEP_MAX_EMPTY_STILL : STEP_MAX_EMPTY_INTERACTIVE};
    return u;
}

SplatUniforms splat_uniforms(uint32_t size, uint32_t particles, uint64_t seed, uint32_t frame, bool exact) {
    SplatUniforms u;
    std::memset(&u, 0, sizeof u);
    u.volumeSize = size;
    u.particleCount = particles;
    u.halfExtent = VOLUME_HALF_EXTENT;
    u.peakTemperature = T_PEAK_DEFAULT;
    u.emissionScale = EMISSION_SCALE;
    u.frame = frame;
    u.exactDeposit = exact ? 1u : 0u;
    u.seed = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    return u;
}

// Owned handles, released in reverse order.
struct Scene {
    gg_context* ctx = nullptr;
    gg_particles* ps = nullptr;
    gg_volume* vol = nullptr;
    uint32_t particles = 0, size = 0, frame = 0;
    ~Scene() {
        gg_volume_destroy(vol);
        gg_particles_destroy(ps);
        gg_context_destroy(ctx);
    }
    void splat(uint64_t seed, bool exact) {
        SplatUniforms u = splat_uniforms(size, particles, seed, frame++, exact);
        check(gg_splat(ps, vol, &u));
    }
};

// The settled disk of the preset: seed, STILL_SETTLE_STEPS substeps, an
// exact splat (Still.swift:36-46).
void settle(Scene& s, const Options& o) {
    s.particles = o.particles ? o.particles : o.preset->particles;
    s.size = o.volume ? o.volume : o.preset->volume;
    check(gg_context_create(0, 0, &s.ctx));
    check(gg_particles_create(s.ctx, s.particles, o.seed, PotentialPaczynskiWiita, &s.ps));
    std::printf("settling %u particles for %u substeps\n", s.particles, STILL_SETTLE_STEPS);
    std::fflush(stdout);
    check(gg_particles_seed(s.ps));
    check(gg_particles_step(s.ps, STILL_SETTLE_STEPS / SIM_SUBSTEPS));
    check(gg_volume_create(s.ctx, s.size, &s.vol));
    s.splat(o.seed, true);
    check(gg_context_synchronize(s.ctx));
}

double seconds_now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void write_tonemapped(gg_targets* t, uint32_t w, uint32_t h, float drift_budget, const std::string& path) {
    PresentUniforms pu;
    std::memset(&pu, 0, sizeof pu);
    pu.exposure = 1.0f;
    pu.driftBudget = drift_budget;
    std::vector<uint8_t> rgba((size_t)w * h * 4);
    check(gg_tonemap(t, &pu, rgba.data()));
    check(gg_write_png(path.c_str(), rgba.data(), w, h));
}

std::string folder_of(const std::string& path) {
    const size_t slash = path.find_last_of('/');
    return slash == std::string::npos ? std::string(".") : path.substr(0, slash);
}

// The HUD's validation line (Renderer.swift:133-137) for one frame's
// counters, printed per served still and sequence frame.
void print_counters(const MarchCounters& c) {
    if (c.rays == 0) return;
    std::printf("drift over budget %.2f percent, %u exhausted, %u captured\n",
                100.0 * (double)c.overDriftBudget / (double)c.rays, c.exhausted, c.captured);
}

// Still.render (Still.swift:8-98), the march served as one request.
void still(const Options& o) {
    Scene s;
    settle(s, o);
    gg_server_config cfg;
    std::memset(&cfg, 0, sizeof cfg);
    cfg.mode = GG_SERVE_BATCHED;
    gg_server* server = nullptr;
    check(gg_server_create(s.ctx, s.vol, &cfg, &server));
    // The result copies into page-locked memory at the link's rate.
    const size_t halves = (size_t)o.width * o.height * 4;
    void* block = nullptr;
    int status = gg_host_alloc(s.ctx, halves * sizeof(uint16_t), &block);
    if (status != GG_OK) gg_server_destroy(server);
    check(status);
    std::unique_ptr<uint16_t, void (*)(uint16_t*)> pixels(static_cast<uint16_t*>(block),
                                                          [](uint16_t* p) { gg_host_free(p); });
    gg_request q;
    std::memset(&q, 0, sizeof q);
    q.azimuth = (float)o.azimuth;
    q.elevation = (float)o.elevation;
    q.distance = (float)o.distance;
    q.fov_y = (float)(50.0 * M_PI / 180.0);
    q.width = o.width;
    q.height = o.height;
    q.step_cap = STEP_CAP_STILL;
    q.spin = (float)o.spin;
    q.star_seed = (uint32_t)o.seed;
    q.output = pixels.get();
    uint64_t ticket = 0;
    gg_request_result res;
    const double t0 = seconds_now();
    status = gg_server_submit(server, &q, &ticket);
    if (status == GG_OK) status = gg_server_wait(server, ticket, 3600.0, &res);
    const double wall = seconds_now() - t0;
    uint64_t requests = 0, steps = 0, launches = 0;
    double busy = 0.0, span = 0.0;
    if (status == GG_OK) status = gg_server_totals(server, 1, &requests, &steps, &launches, &busy, &span);
    gg_server_destroy(server);
    check(status);
    span = std::max(span, 1e-12);
    std::printf("served %u by %u: %llu ray steps, %llu rays re-integrated in FP64, device %.2f ms (%.2f G ray-steps/s), "
                "wall %.1f ms\n",
                o.width, o.height, (unsigned long long)res.ray_steps, (unsigned long long)res.fp64_rays, span * 1e3,
                (double)res.ray_steps / span / 1e9, wall * 1e3);
    print_counters(res.counters);
    gg_targets* t = nullptr;
    check(gg_targets_create(s.ctx, o.width, o.height, &t));
    status = gg_targets_write(t, pixels.get(), nullptr);
    if (status == GG_OK) {
        try {
            write_tonemapped(t, o.width, o.height, DRIFT_BUDGET_STILL, o.still_path);
        } catch (...) {
            gg_targets_destroy(t);
            throw;
        }
    }
    gg_targets_destroy(t);
    check(status);
    if (o.sequence) {
        gg_targets* ft = nullptr;
        check(gg_targets_create(s.ctx, 960, 540, &ft));
        try {
            for (uint32_t frame = 0; frame < o.sequence; ++frame) {
                check(gg_particles_step(s.ps, 1));
                s.splat(o.seed, false);
                MarchUniforms u = march_uniforms(o, 960, 540, false, DRIFT_BUDGET_INTERACTIVE);
                if (o.spin == 0.0) check(gg_tables_update(s.ctx, (float)o.distance, &u));
                MarchCounters counters;
                check(gg_march(s.ctx, s.vol, &u, ft, GG_PRECISION_PLAIN, &counters));
                print_counters(counters);
                char name[32];
                std::snprintf(name, sizeof name, "/seq-%03u.png", frame);
                write_tonemapped(ft, 960, 540, DRIFT_BUDGET_INTERACTIVE, folder_of(o.still_path) + name);
            }
        } catch (...) {
            gg_targets_destroy(ft);
            throw;
        }
        gg_targets_destroy(ft);
        std::printf("sequence of %u frames beside the still\n", o.sequence);
    }
    std::printf("still %s\n", o.still_path.c_str());
}

// Bench.time (Bench.swift:34-44): each call waited to completion, host
// clock; mean, p50 and max of the timed calls in ms.
std::string timing(const char* name, gg_context* ctx, const std::function<void()>& fn, int iterations = 30) {
    std::vector<double> samples;
    for (int k = 0; k < 5 + iterations; ++k) {
        const double t0 = seconds_now();
        fn();
        check(gg_context_synchronize(ctx));
        if (k >= 5) samples.push_back(seconds_now() - t0);
    }
    std::sort(samples.begin(), samples.end());
    double mean = 0.0;
    for (double v : samples) mean += v;
    mean /= samples.size();
    char buf[160];
    std::snprintf(buf, sizeof buf, "\"%s\": {\"mean_ms\": %.4f, \"p50_ms\": %.4f, \"max_ms\": %.4f}", name, mean * 1e3,
                  samples[samples.size() / 2] * 1e3, samples.back() * 1e3);
    return buf;
}

void bench(const Options& o) {
    Scene s;
    settle(s, o);
    const uint32_t mw = o.preset->march_w, mh = o.preset->march_h;
    std::vector<std::string> fields;
    char head[200];
    std::snprintf(head, sizeof head, "\"preset\": \"%s\", \"particles\": %u, \"volume\": %u, \"march\": [%u, %u], \"spin\": %g",
                  o.preset->name, s.particles, s.size, mw, mh, o.spin);
    fields.push_back(head);
    fields.push_back(timing("sim_step", s.ctx, [&] { check(gg_particles_step(s.ps, 1)); }));
    fields.push_back(timing("splat_exact", s.ctx, [&] { s.splat(o.seed, true); }));
    fields.push_back(timing("splat_stochastic", s.ctx, [&] { s.splat(o.seed, false); }));
    gg_targets* t = nullptr;
    check(gg_targets_create(s.ctx, mw, mh, &t));
    try {
        MarchUniforms ui = march_uniforms(o, mw, mh, false, DRIFT_BUDGET_INTERACTIVE);
        MarchUniforms us = march_uniforms(o, mw, mh, true, DRIFT_BUDGET_STILL);
        if (o.spin == 0.0) {
            check(gg_tables_update(s.ctx, (float)o.distance, &ui));
            check(gg_tables_update(s.ctx, (float)o.distance, &us));
        }
        fields.push_back(timing("march_interactive", s.ctx,
                                [&] { check(gg_march(s.ctx, s.vol, &ui, t, GG_PRECISION_PLAIN, nullptr)); }));
        fields.push_back(timing("march_still_compensated", s.ctx,
                                [&] { check(gg_march(s.ctx, s.vol, &us, t, GG_PRECISION_COMPENSATED, nullptr)); }, 10));
        fields.push_back(timing("march_still_as_written", s.ctx,
                                [&] { check(gg_march(s.ctx, s.vol, &us, t, GG_PRECISION_PLAIN_AS_WRITTEN, nullptr)); },
                                10));
        std::vector<uint8_t> rgba((size_t)mw * mh * 4);
        PresentUniforms pu;
        std::memset(&pu, 0, sizeof pu);
        pu.exposure = 1.0f;
        pu.driftBudget = DRIFT_BUDGET_INTERACTIVE;
        fields.push_back(timing("present", s.ctx, [&] { check(gg_tonemap(t, &pu, rgba.data())); }));
        if (o.strategy == "bake") {
            gg_bake* b = nullptr;
            check(gg_bake_create(s.ctx, mw, mh, &b));
            try {
                // The bake strategy is Schwarzschild only (BakePass.swift): its
                // rays are the spin-0 camera's, with the sphere jump.
                Options o0 = o;
                o0.spin = 0.0;
                MarchUniforms ub = march_uniforms(o0, mw, mh, false, DRIFT_BUDGET_INTERACTIVE);
                check(gg_tables_update(s.ctx, (float)o.distance, &ub));
                ub.bakeSpacing = (float)(2.0 * VOLUME_HALF_EXTENT / s.size * BAKE_SPACING_VOXELS);  // BakePass.swift:50-52
                auto bake_full = [&] {  // BAKE_FRAMES chunks of rows (BakePass.swift:55-84)
                    const uint32_t rows = std::max(1u, mh / BAKE_FRAMES);
                    for (uint32_t r = 0; r < mh; r += rows) check(gg_bake_rows(b, &ub, r, std::min(mh, r + rows)));
                };
                fields.push_back(timing("bake_full", s.ctx, bake_full, 5));
                uint32_t truncated = 0;
                check(gg_bake_overflow(b, &truncated, 1));
                bake_full();
                check(gg_context_synchronize(s.ctx));
                check(gg_bake_overflow(b, &truncated, 0));
                fields.push_back("\"bake_truncated_rays\": " + std::to_string(truncated));
                fields.push_back(timing("walk", s.ctx, [&] { check(gg_walk(b, s.vol, &ub, t)); }));
            } catch (...) {
                gg_bake_destroy(b);
                throw;
            }
            gg_bake_destroy(b);
        }
    } catch (...) {
        gg_targets_destroy(t);
        throw;
    }
    gg_targets_destroy(t);
    std::string line = "{";
    for (size_t i = 0; i < fields.size(); ++i) line += (i ? ", " : "") + fields[i];
    std::printf("%s}\n", line.c_str());
}

// ------------------------------------------------------------- validate

// A golden (Golden.swift:5-59): a claim, a kind of bar, the expected value
// and tolerance, and named numeric parameters, embedded from the goldens'
// JSON files at build time.
struct GoldenFile {
    const char* name;
    const char* json;
};

const GoldenFile kGoldens[] = {
#include "goldens_text.h"
};

// The text after `"key":` in a JSON object's text, or npos.
size_t json_value_at(const std::string& text, const std::string& key) {
    const std::string quoted = "\"" + key + "\"";
    size_t at = text.find(quoted);
    if (at == std::string::npos) return at;
    at = text.find(':', at + quoted.size());
    if (at == std::string::npos) return at;
    ++at;
    while (at < text.size() && (text[at] == ' ' || text[at] == '\n' || text[at] == '\t' || text[at] == '\r')) ++at;
    return at;
}

struct Golden {
    std::string name, claim, kind, parameters;
    double expected = 0.0, tolerance = 0.0;

    double number(const std::string& text, const std::string& key) const {
        const size_t at = json_value_at(text, key);
        char* end = nullptr;
        const double v = at == std::string::npos ? 0.0 : std::strtod(text.c_str() + at, &end);
        if (at == std::string::npos || end == text.c_str() + at)
            throw OperationalError{"Golden " + name + " has no number " + key + "."};
        return v;
    }
    std::string string(const std::string& text, const std::string& key) const {
        const size_t at = json_value_at(text, key);
        if (at == std::string::npos || text[at] != '"') throw OperationalError{"Golden " + name + " has no " + key + "."};
        const size_t close = text.find('"', at + 1);
        return text.substr(at + 1, close - at - 1);
    }
    double parameter(const std::string& key) const { return number(parameters, key); }
    // Golden.passes (Golden.swift:47-53).
    bool passes(double measured) const {
        if (kind == "relative") return std::fabs(measured - expected) / std::fabs(expected) <= tolerance;
        if (kind == "absolute") return std::fabs(measured - expected) <= tolerance;
        return measured == expected;
    }
    std::string tolerance_text() const {
        char buf[64];
        if (kind == "relative") std::snprintf(buf, sizeof buf, "%.1f percent", tolerance * 100.0);
        else if (kind == "absolute") std::snprintf(buf, sizeof buf, "%g", tolerance);
        else std::snprintf(buf, sizeof buf, "bitwise");
        return buf;
    }
};

Golden load_golden(const std::string& name) {
    for (const GoldenFile& f : kGoldens) {
        if (name != f.name) continue;
        Golden g;
        g.name = name;
        const std::string text = f.json;
        g.claim = g.string(text, "claim");
        g.kind = g.string(text, "kind");
        g.expected = g.number(text, "expected");
        g.tolerance = g.number(text, "tolerance");
        const size_t at = json_value_at(text, "parameters");
        if (at == std::string::npos) throw OperationalError{"Golden " + name + " has no parameters."};
        g.parameters = text.substr(at, text.find('}', at) - at + 1);
        return g;
    }
    throw OperationalError{"Golden " + name + " is missing from the embedded goldens."};
}

struct Row {
    Golden golden;
    std::string measured;
    bool passed;
    bool run;
};

std::string format(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
std::string format(const char* fmt, ...) {
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return buf;
}

// Probes.run's uniforms (Probes.swift:39-40): one-pixel image, no gas, no
// redshift, no sphere jump; `still` picks the step policy.
MarchUniforms probe_uniforms(bool still, float spin) {
    Options cam;
    MarchUniforms u = march_uniforms(cam, 1, 1, still, 1.0f);
    u.redshift = 0u;
    u.starSeed = 0u;
    u.spin = spin;
    return u;
}

RayProbe probe_of(const double origin[3], const double direction[3]) {
    RayProbe p;
    p.origin = {(float)origin[0], (float)origin[1], (float)origin[2]};
    p.direction = {(float)direction[0], (float)direction[1], (float)direction[2]};
    return p;
}

// Probes.aimed (Probes.swift:46-49): from `radius` on the x axis toward the
// hole with impact parameter b.
RayProbe aimed(double radius, double b, double direction_out[3] = nullptr) {
    const double f = 1.0 - 2.0 / radius;
    const double dphi = b * std::sqrt(f) / radius;
    const double dr = -std::sqrt(std::max(0.0, 1.0 - dphi * dphi));
    const double origin[3] = {radius, 0.0, 0.0}, direction[3] = {dr, dphi, 0.0};
    if (direction_out) std::memcpy(direction_out, direction, sizeof direction);
    return probe_of(origin, direction);
}

// Probes.cameraGrid (Probes.swift:52-66) for the default orbit camera.
std::vector<RayProbe> camera_grid(uint32_t columns, uint32_t rows, double aspect) {
    Options cam;
    const MarchUniforms u = march_uniforms(cam, 1, 1, true, 1.0f);
    const double tan_half = (double)std::tan((float)(50.0 * M_PI / 180.0) * 0.5f);
    const double origin[3] = {u.cameraPosition.x, u.cameraPosition.y, u.cameraPosition.z};
    std::vector<RayProbe> out;
    for (uint32_t row = 0; row < rows; ++row)
        for (uint32_t col = 0; col < columns; ++col) {
            const double x = (2.0 * (col + 0.5) / columns - 1.0) * tan_half * aspect;
            const double y = (1.0 - 2.0 * (row + 0.5) / rows) * tan_half;
            double d[3] = {u.cameraForward.x + x * u.cameraRight.x + y * u.cameraUp.x,
                           u.cameraForward.y + x * u.cameraRight.y + y * u.cameraUp.y,
                           u.cameraForward.z + x * u.cameraRight.z + y * u.cameraUp.z};
            const double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            for (double& c : d) c /= len;
            out.push_back(probe_of(origin, d));
        }
    return out;
}

std::vector<RayProbeResult> run_probes(gg_context* ctx, const MarchUniforms& u, const std::vector<RayProbe>& probes) {
    std::vector<RayProbeResult> out(probes.size());
    check(gg_probe(ctx, &u, probes.data(), out.data(), (uint32_t)probes.size(), GG_PRECISION_PLAIN));
    return out;
}

// DiskEdge.innerEdge (DiskEdge.swift:14-43): Sigma r^(3/2) binned over the
// fit window, a least-squares line, extrapolated to zero.
double disk_inner_edge(const std::vector<double>& radii, double width, double inner, double outer) {
    const int count = (int)std::lround((outer - inner) / width);
    std::vector<double> counts(count, 0.0);
    for (double r : radii)
        if (r >= inner && r < outer) counts[std::min((int)((r - inner) / width), count - 1)] += 1.0;
    double sx = 0.0, sy = 0.0, sxx = 0.0, sxy = 0.0;
    for (int k = 0; k < count; ++k) {
        const double x = inner + (k + 0.5) * width;
        const double y = counts[k] / (2.0 * M_PI * x * width) * std::pow(x, 1.5);
        sx += x;
        sy += y;
        sxx += x * x;
        sxy += x * y;
    }
    const double n = count;
    const double slope = (n * sxy - sx * sy) / (n * sxx - sx * sx);
    const double intercept = (sy - slope * sx) / n;
    return -intercept / slope;
}

uint64_t settled_checksum(gg_context* ctx, const Options& o, uint32_t particles, uint32_t dispatches) {
    gg_particles* ps = nullptr;
    check(gg_particles_create(ctx, particles, o.seed, PotentialPaczynskiWiita, &ps));
    uint64_t sum = 0;
    int status = gg_particles_seed(ps);
    if (status == GG_OK) status = gg_particles_step(ps, dispatches);
    if (status == GG_OK) status = gg_particles_checksum(ps, &sum);
    gg_particles_destroy(ps);
    check(status);
    return sum;
}

// An IEEE binary16 value (the march targets' rgba16f words).
double half_to_double(uint16_t h) {
    const int exponent = (h >> 10) & 0x1f, mantissa = h & 0x3ff;
    const double sign = (h & 0x8000) ? -1.0 : 1.0;
    if (exponent == 0) return sign * std::ldexp((double)mantissa, -24);
    if (exponent == 31) return mantissa ? NAN : sign * INFINITY;
    return sign * std::ldexp((double)(mantissa | 0x400), exponent - 25);
}

// Validate.jump's render (Validate.swift:320-347): still policy, no stars,
// with or without the sphere jump; luminance per pixel.
std::vector<double> render_luminance(Scene& s, uint32_t w, uint32_t h, bool jump) {
    Options cam;
    MarchUniforms u = march_uniforms(cam, w, h, true, DRIFT_BUDGET_STILL);
    u.starBrightness = 0.0f;
    u.starSeed = 0u;
    if (jump) check(gg_tables_update(s.ctx, (float)cam.distance, &u));
    gg_targets* t = nullptr;
    check(gg_targets_create(s.ctx, w, h, &t));
    std::vector<uint16_t> color((size_t)w * h * 4);
    int status = gg_march(s.ctx, s.vol, &u, t, GG_PRECISION_PLAIN, nullptr);
    if (status == GG_OK) status = gg_targets_read(t, color.data(), nullptr, nullptr, nullptr);
    gg_targets_destroy(t);
    check(status);
    std::vector<double> lum((size_t)w * h);
    for (size_t i = 0; i < lum.size(); ++i) {
        double rgb[3];
        for (int c = 0; c < 3; ++c) rgb[c] = half_to_double(color[4 * i + c]);
        lum[i] = 0.2126 * rgb[0] + 0.7152 * rgb[1] + 0.0722 * rgb[2];
    }
    return lum;
}

// The Kerr shadow's equatorial edge on one side, as L / E of the launch at
// the boundary: the reference's bisection through single-ray probes
// (Validate.swift:352-365), and the same boundary bisected in FP64 on the
// device (gg_capture_boundary).
double kerr_xi_of(gg_context* ctx, const MarchUniforms& u, double radius, double side, double aim) {
    const double origin[3] = {radius, 0.0, 0.0}, direction[3] = {-1.0, side * aim, 0.0};
    const RayProbeResult r = run_probes(ctx, u, {probe_of(origin, direction)})[0];
    return (double)r.angularMomentum / (double)r.energy;
}

double kerr_xi_probes(gg_context* ctx, const MarchUniforms& u, double radius, double side, int iterations) {
    double low = 0.0, high = 12.0 / radius;
    for (int i = 0; i < iterations; ++i) {
        const double aim = 0.5 * (low + high);
        const double origin[3] = {radius, 0.0, 0.0}, direction[3] = {-1.0, side * aim, 0.0};
        const RayProbeResult r = run_probes(ctx, u, {probe_of(origin, direction)})[0];
        if (r.outcome == RayCaptured) low = aim;
        else high = aim;
    }
    return kerr_xi_of(ctx, u, radius, side, 0.5 * (low + high));
}

double kerr_xi_fp64(gg_context* ctx, const MarchUniforms& u, double radius, double side) {
    const double origin[3] = {radius, 0.0, 0.0}, base[3] = {-1.0, 0.0, 0.0}, axis[3] = {0.0, side, 0.0};
    double t = 0.0;
    check(gg_capture_boundary(ctx, &u, origin, base, axis, 0.0, 12.0 / radius, 1024, 4, &t));
    return kerr_xi_of(ctx, u, radius, side, t);
}

// Validate.run (Validate.swift:19-55): the default preset's disk settled for
// the isco golden, then each golden in the reference's order. Parity,
// beaming and sky compare against the FP64 oracle, which is test
// infrastructure here and is not linked into this program: those rows
// report that the test suite runs them (tests/test_goldens_gpu.py) and do
// not decide the exit code.
int validate(const Options& o) {
    Scene s;
    s.particles = o.particles ? o.particles : o.preset->particles;
    s.size = o.volume ? o.volume : o.preset->volume;
    check(gg_context_create(0, 0, &s.ctx));
    const Golden isco = load_golden("isco");
    check(gg_particles_create(s.ctx, s.particles, o.seed, PotentialPaczynskiWiita, &s.ps));
    check(gg_particles_seed(s.ps));
    check(gg_particles_step(s.ps, (uint32_t)isco.parameter("settlingSteps") / SIM_SUBSTEPS));
    check(gg_volume_create(s.ctx, s.size, &s.vol));
    const char* order[] = {"isco", "determinism", "shadow", "deflection", "conservation_interactive",
                           "conservation_still", "parity", "beaming", "sky", "jump", "shadow_kerr"};
    std::vector<Row> rows;
    for (const char* name : order) {
        const Golden g = load_golden(name);
        const std::string n = name;
        if (n == "isco") {
            std::vector<Particle> parts(s.particles);
            check(gg_particles_read(s.ps, parts.data(), s.particles));
            std::vector<double> radii(parts.size());
            for (size_t i = 0; i < parts.size(); ++i)
                radii[i] = std::sqrt((double)parts[i].position.x * parts[i].position.x +
                                     (double)parts[i].position.y * parts[i].position.y);
            const double edge =
                disk_inner_edge(radii, g.parameter("binWidth"), g.parameter("fitInner"), g.parameter("fitOuter"));
            rows.push_back({g, format("r = %.3f", edge), g.passes(edge), true});
        } else if (n == "determinism") {
            const uint32_t d = (uint32_t)g.parameter("steps") / SIM_SUBSTEPS;
            const uint64_t a = settled_checksum(s.ctx, o, s.particles, d), b = settled_checksum(s.ctx, o, s.particles, d);
            rows.push_back({g, format("%016llx vs %016llx", (unsigned long long)a, (unsigned long long)b), a == b, true});
        } else if (n == "shadow") {
            double low = g.parameter("bracketLow"), high = g.parameter("bracketHigh");
            const double radius = g.parameter("launchRadius");
            const int per = (int)g.parameter("raysPerRound");
            const MarchUniforms u = probe_uniforms(true, 0.0f);
            double measured = -1.0;
            for (int round = 0; round < (int)g.parameter("rounds") && measured < 0.0; ++round) {
                std::vector<double> values;
                std::vector<RayProbe> probes;
                for (int i = 0; i < per; ++i) {
                    values.push_back(low + (high - low) * ((i + 0.5) / per));
                    probes.push_back(aimed(radius, values.back()));
                }
                const std::vector<RayProbeResult> res = run_probes(s.ctx, u, probes);
                int exhausted = -1, escaped = per;
                for (int i = per - 1; i >= 0; --i) {
                    if (res[i].outcome == RayExhausted) exhausted = i;
                    if (res[i].outcome == RayEscaped) escaped = i;
                }
                if (exhausted >= 0) {
                    measured = values[exhausted];
                    break;
                }
                const double new_low = escaped > 0 ? values[escaped - 1] : low;
                const double new_high = escaped < per ? values[escaped] : high;
                low = new_low;
                high = new_high;
            }
            const double critical = measured >= 0.0 ? measured : 0.5 * (low + high);
            rows.push_back({g, format("b = %.4f", critical), g.passes(critical), true});
        } else if (n == "deflection") {
            const double radius = g.parameter("launchRadius");
            MarchUniforms u = probe_uniforms(true, 0.0f);
            u.geodesic.stepMax = INFINITY;
            u.geodesic.escapeRadius = (float)radius;
            double a[3];
            const RayProbe launch = aimed(radius, g.parameter("impactParameter"), a);
            const RayProbeResult r = run_probes(s.ctx, u, {launch})[0];
            const double d[3] = {r.direction.x, r.direction.y, r.direction.z};
            const double c[3] = {a[1] * d[2] - a[2] * d[1], a[2] * d[0] - a[0] * d[2], a[0] * d[1] - a[1] * d[0]};
            const double angle =
                std::atan2(std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]), a[0] * d[0] + a[1] * d[1] + a[2] * d[2]);
            const bool escaped = r.outcome == RayEscaped;
            rows.push_back({g, format("%.6f rad%s", angle, escaped ? "" : " (ray did not escape)"),
                            g.passes(angle) && escaped, true});
        } else if (n == "conservation_interactive" || n == "conservation_still") {
            const bool still = n == "conservation_still";
            const std::vector<RayProbe> grid =
                camera_grid((uint32_t)g.parameter("columns"), (uint32_t)g.parameter("rows"), 960.0 / 540.0);
            const std::vector<RayProbeResult> res = run_probes(s.ctx, probe_uniforms(still, 0.0f), grid);
            double worst = 0.0;
            int exhausted = 0;
            for (const RayProbeResult& r : res) {
                worst = std::max(worst, (double)r.drift);
                exhausted += r.outcome == RayExhausted ? 1 : 0;
            }
            rows.push_back({g, format("max drift %.2e, %d of %zu rays exhausted", worst, exhausted, res.size()),
                            g.passes(worst), true});
        } else if (n == "jump") {
            // The volume as the reference's run leaves it before the jump
            // golden: the settled disk, splatted exactly (Validate.swift:262-266).
            s.splat(o.seed, true);
            const uint32_t w = (uint32_t)g.parameter("width"), h = (uint32_t)g.parameter("height");
            const std::vector<double> full = render_luminance(s, w, h, false), jumped = render_luminance(s, w, h, true);
            double difference = 0.0, total = 0.0;
            for (size_t i = 0; i < full.size(); ++i) {
                difference += std::fabs(full[i] - jumped[i]);
                total += full[i];
            }
            const double measured = total > 0.0 ? difference / total : 1.0;
            rows.push_back({g, format("mean relative difference %.2e", measured), g.passes(measured), true});
        } else if (n == "shadow_kerr") {
            const double spin = g.parameter("spin"), radius = g.parameter("launchRadius");
            const MarchUniforms u = probe_uniforms(true, (float)spin);
            const int iterations = (int)g.parameter("iterations");
            const double gpu = std::fabs(kerr_xi_probes(s.ctx, u, radius, -1.0, iterations) /
                                         kerr_xi_probes(s.ctx, u, radius, 1.0, iterations));
            const double fp64 = std::fabs(kerr_xi_fp64(s.ctx, u, radius, -1.0) / kerr_xi_fp64(s.ctx, u, radius, 1.0));
            const double measured = gpu / fp64;
            rows.push_back({g, format("gpu %.4f vs FP64 bisection %.4f, ratio %.4f", gpu, fp64, measured),
                            g.passes(measured), true});
        } else {
            rows.push_back({g, "needs the FP64 oracle: run by the test suite", true, false});
        }
    }
    // Validate.print (Validate.swift:388-397).
    size_t wn = 6, wc = 5, wm = 8;
    for (const Row& r : rows) {
        wn = std::max(wn, r.golden.name.size());
        wc = std::max(wc, r.golden.claim.size());
        wm = std::max(wm, r.measured.size());
    }
    auto pad = [](const std::string& t, size_t w) { return t + std::string(w > t.size() ? w - t.size() : 0, ' '); };
    std::printf("validation on CUDA device 0\n");
    std::printf("%s  %s  %s  tolerance    status\n", pad("golden", wn).c_str(), pad("claim", wc).c_str(),
                pad("measured", wm).c_str());
    bool all = true;
    for (const Row& r : rows) {
        all = all && r.passed;
        std::printf("%s  %s  %s  %s  %s\n", pad(r.golden.name, wn).c_str(), pad(r.golden.claim, wc).c_str(),
                    pad(r.measured, wm).c_str(), pad(r.golden.tolerance_text(), 11).c_str(),
                    !r.run ? "skipped" : (r.passed ? "pass" : "FAIL"));
    }
    return all ? 0 : 1;
}

int run(const Options& o) {
    if (o.command == "version") {
        std::printf("gargantua-b200 %s\n", kVersion);
    } else if (o.command == "constants") {
        std::fputs(kConstants, stdout);
    } else if (o.command == "still") {
        still(o);
    } else if (o.command == "bench") {
        bench(o);
    } else if (o.command == "validate") {
        return validate(o);
    } else {
        throw OperationalError{"The interactive window needs a display; use --still or bench."};
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    try {
        o = parse(argc, argv);
    } catch (const UsageError& e) {
        std::fprintf(stderr, "%s\n", e.sentence.c_str());
        return 64;
    }
    try {
        return run(o);
    } catch (const OperationalError& e) {
        std::fprintf(stderr, "%s\n", e.sentence.c_str());
        return 2;
    }
}
