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
// object. The interactive window needs a display and has no counterpart
// here; validate runs as the GPU test suite, where the FP64 oracle lives.
#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
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

// Still.render (Still.swift:8-98), the march served as one request.
void still(const Options& o) {
    Scene s;
    settle(s, o);
    gg_server_config cfg;
    std::memset(&cfg, 0, sizeof cfg);
    cfg.mode = GG_SERVE_BATCHED;
    gg_server* server = nullptr;
    check(gg_server_create(s.ctx, s.vol, &cfg, &server));
    std::vector<uint16_t> pixels((size_t)o.width * o.height * 4);
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
    q.output = pixels.data();
    uint64_t ticket = 0;
    gg_request_result res;
    const double t0 = seconds_now();
    int status = gg_server_submit(server, &q, &ticket);
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
    gg_targets* t = nullptr;
    check(gg_targets_create(s.ctx, o.width, o.height, &t));
    status = gg_targets_write(t, pixels.data(), nullptr);
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
                check(gg_march(s.ctx, s.vol, &u, ft, GG_PRECISION_PLAIN, nullptr));
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
        throw OperationalError{"validate compares against the FP64 oracle, which ships with the tests: "
                               "run python -m pytest tests -m gpu."};
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
