"""Benchmark: ray-steps/s of the served, compensated-FP32 march on the mixed
request stream, against the plain per-request FP32 march; p50/p99 latency.

Workload (one GPU): the served mixed request stream -- still requests with
Poisson arrivals at 40 req/s, resolution from {320x180, 640x360, 960x540,
1920x1080, 3840x2160}, step budget from {256, 4096}, spin from {0, 0.5,
0.9}, camera radius uniform in [40, 120], inclination uniform in [10, 90]
degrees, azimuth uniform -- all sharing one resident default-preset disk
(1M particles settled for 600 substeps, exact splat into 128^3). The stream
is generated from a fixed seed (synthetic data; the reference ships none).

A step serves one slice of `--requests-per-step` consecutive requests of the
stream, all submitted at once (closed loop), through gg_server_* with pinned
host output buffers:
  value  ray steps / device time: the span from the first to the last launch
         of the step on the device clock (CUDA events), inputs resident;
  e2e    ray steps / wall time from the first submit to the last result in
         host memory (device-to-host copies included).
Two per-request baselines serve the same slices one request at a time
through a thread-per-pixel image kernel: `plain_per_request` with the
reference's step arithmetic as written (march.metal), and
`plain_lane_per_request` with this library's plain FP32 step arithmetic,
which isolates what batching and the persistent kernel add. Latency p50/p99
come from a separate open-loop replay of the stream's arrivals at 40 req/s.
`passes` times the particle step and the splat alone against their
rooflines.

--impl reference times the reference's CPU path, the FP64 oracle's
integrators (oracle/, a C restatement of gargantua's Swift oracle), on a
bounded sample of each slice's rays with every host core.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RESOLUTIONS = [(320, 180), (640, 360), (960, 540), (1920, 1080), (3840, 2160)]
STEP_CAPS = [256, 4096]
SPINS = [0.0, 0.5, 0.9]
ARRIVAL_RATE = 40.0
STREAM_LENGTH = 512

# Algorithmic FP32 operations per unit of work, from running the reference
# algorithm on a counting scalar type (oracle/opcount.cpp; a CPU test keeps
# these equal to its output): add/sub/mul/div/sqrt/transcendental = 1.
FLOPS_SCHWARZSCHILD_STEP = 192  # RK4 165 + position 14 + step policy 3 + path 10
FLOPS_KERR_STEP = 515           # RK4 436 + step policy, position, path, Carter and null gauges 79
FLOPS_SAMPLE = 111              # in-slab gather 67 + static-observer direction 44
# DRAM bytes of one serve_kerr_chunks_kernel launch (ncu, 1920x1080 4096-step Kerr still): the
# march reads only its descriptors and tables from HBM; pixels stay in L2 until the copy-out.
SERVE_KERR_TRAFFIC_BYTES = 5836288


def stream_length(warmup: int, steps: int, per_step: int, latency_requests: int) -> int:
    """Requests the run needs: every warm-up and timed slice full, then the
    open-loop latency replay's requests after them (at least 512)."""
    return max(STREAM_LENGTH, (warmup + steps) * per_step + latency_requests)


def make_stream(seed: int, count: int = STREAM_LENGTH):
    """The seeded request stream: arrival time and request parameters. The
    first `n` requests are the same for every count >= n: requests are drawn
    in blocks of 512 (STREAM_LENGTH), block b from its own generator
    (seed, b), arrivals continuing from the previous block's last."""
    out = []
    for block in range((count + STREAM_LENGTH - 1) // STREAM_LENGTH):
        out.extend(_stream_block(seed, block, out[-1]["t"] if out else 0.0, len(out)))
    return out[:count]


def _stream_block(seed: int, block: int, t0: float, first: int):
    rng = np.random.default_rng(seed if block == 0 else [seed, block])
    arrivals = t0 + np.cumsum(rng.exponential(1.0 / ARRIVAL_RATE, size=STREAM_LENGTH))
    out = []
    for j in range(STREAM_LENGTH):
        k = first + j
        w, h = RESOLUTIONS[rng.integers(len(RESOLUTIONS))]
        cap = STEP_CAPS[rng.integers(len(STEP_CAPS))]
        spin = SPINS[rng.integers(len(SPINS))]
        r = rng.uniform(40.0, 120.0)
        inclination = math.radians(rng.uniform(10.0, 90.0))
        azimuth = rng.uniform(0.0, 2.0 * math.pi)
        out.append({"t": float(arrivals[j]), "width": w, "height": h, "step_cap": cap, "spin": spin,
                    "distance": float(r), "elevation": math.pi / 2.0 - inclination, "azimuth": float(azimuth),
                    "seed": seed * 100003 + k})
    return out


def spec_of(q):
    import gargantua_b200 as g

    return g.RequestSpec(q["width"], q["height"], q["step_cap"], q["spin"], azimuth=q["azimuth"],
                         elevation=q["elevation"], distance=q["distance"], star_seed=q["seed"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.reader.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def flops_of(q, result) -> float:
    per_step = FLOPS_KERR_STEP if q["spin"] > 0.0 else FLOPS_SCHWARZSCHILD_STEP
    return float(result.ray_steps) * per_step + float(result.samples) * FLOPS_SAMPLE


def serve_slice(server, slice_, pinned):
    """Submit a slice closed-loop; returns (results, wall seconds, device span
    seconds, device busy seconds, launches)."""
    server.totals(reset=True)
    t0 = time.perf_counter()
    tickets = [server.submit(spec_of(q), output=out) for q, out in zip(slice_, pinned)]
    results = [server.wait(t)[2] for t in tickets]
    wall = time.perf_counter() - t0
    tot = server.totals(reset=True)
    return results, wall, tot["span_seconds"], tot["busy_seconds"], tot["launches"]


def pinned_outputs(ctx, slice_):
    """The slice's output arrays in page-locked host memory, from the
    library's own allocator (gargantua_b200.pinned_array, gg_host_alloc), as
    a host serving many requests would pass them."""
    import gargantua_b200 as g

    return [g.pinned_array(ctx, (q["width"] * q["height"], 4), np.float16) for q in slice_]


def latency_replay(server, stream):
    """Open loop: submit each request at its arrival time; latency is result
    ready minus arrival (gg_request_result.finished - submitted)."""
    pinned = pinned_outputs(server.ctx, stream)
    t0 = time.perf_counter()
    base = stream[0]["t"]
    tickets = []
    for q, out in zip(stream, pinned):
        delay = (q["t"] - base) - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        tickets.append(server.submit(spec_of(q), output=out))
    lat = []
    for t in tickets:
        r = server.wait(t)[2]
        lat.append((r.finished - r.submitted) * 1e3)
    return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))


# Request classes of the per-class table: every resolution and step budget,
# Schwarzschild (spin 0) and Kerr (spin 0.5 or 0.9), with the stream's camera
# distribution. A class serves about CLASS_PIXELS pixels (2 to 32 requests).
CLASS_PIXELS = 2 * 1920 * 1080


def class_requests(width: int, height: int, cap: int, kerr: bool, seed: int):
    rng = np.random.default_rng(seed)
    n = int(min(32, max(2, round(CLASS_PIXELS / (width * height)))))
    out = []
    for k in range(n):
        spin = float(rng.choice([0.5, 0.9])) if kerr else 0.0
        r = rng.uniform(40.0, 120.0)
        inclination = math.radians(rng.uniform(10.0, 90.0))
        azimuth = rng.uniform(0.0, 2.0 * math.pi)
        out.append({"t": 0.0, "width": width, "height": height, "step_cap": cap, "spin": spin, "distance": float(r),
                    "elevation": math.pi / 2.0 - inclination, "azimuth": float(azimuth), "seed": seed * 1009 + k})
    return out


def class_table(servers: dict) -> list:
    """Each class served closed-loop by every server in `servers` (name ->
    Server): ray steps / device span, in G ray-steps/s, and the served
    server's ratio over each per-request one. Each class is served once
    untimed first (the servers' pools map the class's target sizes)."""
    rows = []
    seed = 500
    for (w, h) in RESOLUTIONS:
        for cap in STEP_CAPS:
            for kerr in (False, True):
                seed += 1
                reqs = class_requests(w, h, cap, kerr, seed)
                pins = pinned_outputs(next(iter(servers.values())).ctx, reqs)
                row = {"class": f"{w}x{h}/{cap}/{'kerr' if kerr else 'schw'}", "requests": len(reqs)}
                for name, server in servers.items():
                    serve_slice(server, reqs, pins)
                    results, wall, span, _, _ = serve_slice(server, reqs, pins)
                    steps = sum(r.ray_steps for r in results)
                    row[name] = round(steps / max(span, 1e-12) / 1e9, 3)
                    row[name + "_e2e"] = round(steps / max(wall, 1e-12) / 1e9, 3)
                for name in servers:
                    if name != "served":
                        row["x_" + name] = round(row["served"] / max(row[name], 1e-12), 2)
                rows.append(row)
    return rows


def cpu_sample(slices, seconds: float, threads: int):
    """The oracle's FP64 integrators on a bounded sample of the slices' rays:
    returns (ray steps per second, rays, steps, seconds, description)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi as O

    import gargantua_b200 as g

    rng = np.random.default_rng(7)
    total_steps, total_rays, elapsed = 0, 0, 0.0
    per_request = 256
    flat = [q for s in slices for q in s]
    k = 0
    while elapsed < seconds and k < 4 * len(flat):
        q = flat[k % len(flat)]
        k += 1
        cam = g.OrbitCamera(q["azimuth"], q["elevation"], q["distance"])
        launches = g.camera_grid(cam, 64, 36, q["width"] / q["height"])
        pick = rng.choice(len(launches), size=min(per_request, len(launches)), replace=False)
        probes = np.array([np.concatenate([launches[i].origin, launches[i].direction]) for i in pick])
        escape = max(60.0, q["distance"] + 10.0)
        t0 = time.perf_counter()
        if q["spin"] > 0.0:
            st = O.KerrSettings(0.02, 0.005, 0.5, 0.05, escape, q["step_cap"])
            res = O.kerr_integrate_batch(q["spin"], probes, st, threads)
        else:
            interactive = q["step_cap"] <= 256
            st = O.Settings(0.02, 0.02, 0.5, 2.02, escape, q["step_cap"], 0.1 if interactive else 0.06,
                            3.0 if interactive else 1.5)
            res = O.integrate_batch(probes, st, threads)
        elapsed += time.perf_counter() - t0
        total_steps += int(res[:, 8].sum())
        total_rays += len(probes)
    desc = (f"FP64 oracle integrators, {total_rays} rays ({per_request} per request from a 64x36 grid of each "
            f"request's camera) over {k} requests of the timed slices, {threads} threads")
    return total_steps / max(elapsed, 1e-9), total_rays, total_steps, elapsed, desc


def drift_vs_oracle(ctx, slices, per_request: int = 64, max_requests: int = 24) -> dict:
    """4096-step rays of the timed requests, 64 per request from a 64x36 grid
    of its camera: drift of the compensated FP32 march (gg_probe, the served
    arithmetic, FP64 re-integration off) beside the FP64 oracle's drift for
    the same rays (Schwarzschild: E and L; Kerr: Carter constant and null
    residual, each the maximum over the ray's steps as the reference
    defines it)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi as O

    import gargantua_b200 as g

    rng = np.random.default_rng(11)
    picked = [q for s in slices for q in s if q["step_cap"] == 4096][:max_requests]
    out = {}
    for kind in ("schwarzschild", "kerr"):
        gpu, ref = [], []
        for q in picked:
            if (q["spin"] > 0.0) != (kind == "kerr"):
                continue
            cam = g.OrbitCamera(q["azimuth"], q["elevation"], q["distance"])
            launches = g.camera_grid(cam, 64, 36, q["width"] / q["height"])
            pick = rng.choice(len(launches), size=per_request, replace=False)
            sel = [g.as_float32_launch(launches[i]) for i in pick]
            escape = max(60.0, q["distance"] + 10.0)
            st = g.Settings.still()
            st.escape_radius = escape
            u = g.uniforms(cam, 1, 1, st, 1.0, False, 0, spin=q["spin"])  # budget 1: no FP64 pass
            gpu.append(ctx.probe(sel, u, g.types.PRECISION_COMPENSATED)["drift"].astype(np.float64))
            probes = np.array([np.concatenate([l.origin, l.direction]) for l in sel])
            if kind == "kerr":
                res = O.kerr_integrate_batch(q["spin"], probes, O.KerrSettings(0.02, 0.005, 0.5, 0.05, escape, 4096))
            else:
                res = O.integrate_batch(probes, O.Settings(0.02, 0.02, 0.5, 2.02, escape, 4096, 0.06, 1.5))
            ref.append(res[:, 6])
        if not gpu:
            continue
        a, b = np.concatenate(gpu), np.concatenate(ref)
        edges = [0.0] + [10.0 ** e for e in range(-12, 1)] + [np.inf]

        def summary(x):
            hist, _ = np.histogram(x, bins=edges)
            return {"p50": float(np.median(x)), "p99": float(np.quantile(x, 0.99)), "under_1e-5": float(np.mean(x < 1e-5)),
                    "histogram": {"upper_edges": [f"{e:g}" for e in edges[1:]], "counts": hist.tolist()}}

        out[kind] = {"rays": int(a.size), "fp32_compensated": summary(a), "fp64_oracle": summary(b)}
    return out


def measured_peaks() -> dict:
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return json.load(fh)
    except OSError:
        return {}


def cpu_timed(fn, seconds: float = 1.0) -> float:
    """Mean seconds of fn() over repeats totalling about `seconds` (at least 1)."""
    t0 = time.perf_counter()
    fn()
    once = time.perf_counter() - t0
    reps = max(1, min(20, int(seconds / max(once, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    return (time.perf_counter() - t0) / reps


def cpu_pass_baseline(kind: str, fn_of_threads, units: float, unit: str, sample: str) -> dict:
    """The FP32 CPU replica of a pass (oracle/replica.c, built with
    -ffp-contract=off, bit-exact with the kernel) on one host thread and on
    every host core: `units` of work per call."""
    cores = os.cpu_count() or 1
    one = cpu_timed(lambda: fn_of_threads(1))
    every = cpu_timed(lambda: fn_of_threads(cores))
    return {"value": units / every, "unit": unit, "cores": cores, "kind": "port",
            "single_thread": units / one, "sample": sample + f"; FP32 replica, 1 and {cores} threads"}


def measure_passes(ctx, g, torch) -> dict:
    """The particle step and the splat, each timed alone with CUDA events on
    the library's stream, L2 flushed before every launch by reading a 256 MB
    buffer (a read leaves clean lines, so no write-back of the flush lands
    inside the timed launch).

    sim: the max preset's 4M particles, one dispatch (SIM_SUBSTEPS = 2
    substeps) reads and writes 32 B per particle: 64 B algorithmic traffic
    per particle-dispatch, bound by HBM. splat: the default preset's 1M
    settled particles into 128^3, the shape (brick edge, chunk) picked by
    gg_splat_autotune; the bin's work is 6 u32 atomic adds per deposit
    (exact: one per corner), bound by the device's scattered shared-memory
    atomic rate for the brick deposit (gg_measure_shared_atomic_peak), or
    the global one for direct atomics (gg_measure_atomic_peak); the resolve
    reads 24 B, zeroes 24 B and writes 16 B per voxel, bound by HBM."""
    lib = g.lib()
    ext = torch.cuda.ExternalStream(lib.gg_context_stream(ctx.handle))
    flush = torch.ones(64 << 20, dtype=torch.int32, device="cuda")
    sink = torch.empty((), dtype=torch.int64, device="cuda")

    def timed(fn, pre=None, iters=20, warm=3):
        pairs = []
        for k in range(warm + iters):
            if pre is not None:
                pre()
            with torch.cuda.stream(ext):
                torch.sum(flush, dim=0, out=sink)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            fn()
            e1.record(ext)
            if k >= warm:
                pairs.append((e0, e1))
        ext.synchronize()
        return sum(a.elapsed_time(b) for a, b in pairs) / len(pairs) * 1e-3

    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    hbm_src = "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"
    out = {}

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi as O

    big = g.Particles(ctx, 4_000_000, seed=1)
    big.advance(10, seed_first=True)
    t = timed(lambda: big.step(1))
    gbs = 64.0 * big.count / t / 1e9
    su, cdf = big.uniforms(), big.inverse_cdf()
    cpu_parts = big.read()[:1_000_000].copy()

    def cpu_step(threads):
        O.step32(cpu_parts, 1, 1, cdf, su.dt, su.alpha, su.temperatureScale, 1, threads)

    out["sim"] = {"workload": "4M particles (max preset), one dispatch of 2 substeps", "us": t * 1e6,
                  "value": 2 * big.count / t, "unit": "particle-steps/s",
                  "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                               "bytes_per_launch": 64 * big.count, "peak_source": hbm_src},
                  "cpu_baseline": cpu_pass_baseline("sim", cpu_step, 2.0 * len(cpu_parts), "particle-steps/s",
                                                    "1M of the 4M particles, one dispatch of 2 substeps")}
    big.close()

    ps = g.Particles(ctx, 1_000_000, seed=1)
    ps.advance(300, seed_first=True)
    parts = ps.read()
    unit = (parts[:, :3] + np.float32(30.0)) / np.float32(60.0)  # splat.metal:52-53, in float32
    inside = int(np.all((unit >= 0.0) & (unit < 1.0), axis=1).sum())
    vol = g.Volume(ctx, 128)
    atom_peak = ctx.atomic_peak_gadds(128 ** 3)
    shared_peak = ctx.shared_atomic_peak_gadds()
    for exact in (True, False):
        edge, chunk, _ = vol.autotune(ps, exact)
        deposits = inside * (8 if exact else 1)
        t = timed(lambda: vol.bin(ps, exact), pre=vol.clear)
        rate = 6.0 * deposits / t / 1e9
        peak, src = ((shared_peak, "gg_measure_shared_atomic_peak: scattered u32 shared atomics into a 9^3 "
                                   "tile of six-word records padded to seven (all 32 banks)") if edge else
                     (atom_peak, "gg_measure_atomic_peak: scattered u32 REDs into a 128^3 six-word grid"))
        out["splat_bin_exact" if exact else "splat_bin_stochastic"] = {
            "workload": "1M settled particles (default preset) into 128^3", "us": t * 1e6,
            "value": deposits / t, "unit": "deposits/s",
            "shape": {"brick_edge": edge, "chunk": chunk, "chosen_by": "gg_splat_autotune"},
            "roofline": {"bound": "shared atomics" if edge else "global atomics", "achieved": rate, "peak": peak,
                         "unit": "G u32 atomic adds/s", "frac": rate / peak, "peak_source": src,
                         "global_atomic_peak": atom_peak},
            "cpu_baseline": cpu_pass_baseline(
                "splat", lambda threads, ex=exact: O.deposit32(parts, 128, 0, ex, 1, threads=threads), deposits,
                "deposits/s", "the same 1M particles into 128^3 (sums allocated and zeroed per call)")}
    vol.bin(ps, True)
    sums = vol.read_sums()
    bb = ctx.blackbody()[:, :3].copy()
    t = timed(vol.resolve, pre=lambda: vol.bin(ps, True))
    gbs = 64.0 * 128 ** 3 / t / 1e9
    out["splat_resolve"] = {"workload": "128^3 resolve + clear", "us": t * 1e6, "value": 128 ** 3 / t,
                            "unit": "voxels/s",
                            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                                         "frac": gbs / hbm, "bytes_per_launch": 64 * 128 ** 3,
                                         "peak_source": hbm_src},
                            "cpu_baseline": cpu_pass_baseline(
                                "resolve", lambda threads: O.resolve32(*sums, 128, bb, threads=threads), 128 ** 3,
                                "voxels/s", "the same 128^3 sums (no clear)")}
    vol.close()
    ps.close()

    # The max preset's contention workload: 4M particles, 70 % seeded from a
    # power-law surface density ~ r^-3 (concentrating deposits near r = 6),
    # settled 600 substeps, exact splat into 256^3 with the autotuned shape.
    mx = g.Particles(ctx, 4_000_000, seed=1)
    mx.seed_profile(0.7, 3.0)
    mx.advance(300, seed_first=True)
    parts = mx.read()
    unit = (parts[:, :3] + np.float32(30.0)) / np.float32(60.0)
    inside = int(np.all((unit >= 0.0) & (unit < 1.0), axis=1).sum())
    big_vol = g.Volume(ctx, 256)
    edge, chunk, _ = big_vol.autotune(mx, True)
    t = timed(lambda: big_vol.bin(mx, True), pre=big_vol.clear)
    rate = 6.0 * 8 * inside / t / 1e9
    peak, src = ((shared_peak, "gg_measure_shared_atomic_peak") if edge else (atom_peak, "gg_measure_atomic_peak"))
    out["splat_bin_exact_max_preset"] = {
        "workload": "4M particles, 70 % from Sigma ~ r^-3, into 256^3 (max preset contention case)", "us": t * 1e6,
        "value": 8 * inside / t, "unit": "deposits/s",
        "shape": {"brick_edge": edge, "chunk": chunk, "chosen_by": "gg_splat_autotune"},
        "roofline": {"bound": "shared atomics" if edge else "global atomics", "achieved": rate, "peak": peak,
                     "unit": "G u32 atomic adds/s", "frac": rate / peak, "peak_source": src}}
    t = timed(big_vol.resolve, pre=lambda: big_vol.bin(mx, True))
    gbs = 64.0 * 256 ** 3 / t / 1e9
    out["splat_resolve_max_preset"] = {"workload": "256^3 resolve + clear", "us": t * 1e6, "value": 256 ** 3 / t,
                                       "unit": "voxels/s",
                                       "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                                                    "frac": gbs / hbm, "bytes_per_launch": 64 * 256 ** 3,
                                                    "peak_source": hbm_src}}
    big_vol.close()
    mx.close()
    del flush, sink
    return out


def setup_world(device: int, world: int):
    import gargantua_b200 as g

    # A server-sized budget: the reference's 3 GB cap is a laptop rule.
    ctx = g.Context(device, budget_bytes=48 << 30)
    if world > 1:
        # The disk's particles are sharded over the ranks and their grids
        # summed over NCCL, so every rank serves the same volume.
        from gargantua_b200 import parallel

        disk = parallel.ShardedDisk(ctx, 1_000_000, 128, seed=1)
        disk.advance(300, seed_first=True)  # STILL_SETTLE_STEPS = 600 substeps
        disk.splat(exact=True)
        ctx.synchronize()
        return ctx, disk, disk.volume
    ps = g.Particles(ctx, 1_000_000, seed=1)
    ps.advance(300, seed_first=True)  # STILL_SETTLE_STEPS = 600 substeps
    vol = g.Volume(ctx, 128)
    vol.splat(ps, exact=True)
    ctx.synchronize()
    return ctx, ps, vol


def drift_summary(d) -> dict | None:
    """The 4096-step drift figures that carry the metric's precision bar."""
    if not d:
        return None
    out = {}
    for kind, label in (("schwarzschild", "E/L"), ("kerr", "Q/null residual")):
        if kind in d:
            a, b = d[kind]["fp32_compensated"], d[kind]["fp64_oracle"]
            out[kind] = {"gauge": label, "p99": a["p99"], "under_1e-5": a["under_1e-5"], "fp64_oracle_p99": b["p99"],
                         "fp64_oracle_under_1e-5": b["under_1e-5"]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--requests-per-step", type=int, default=32)
    ap.add_argument("--latency-requests", type=int, default=48)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-classes", action="store_true", help="skip the per-class served-vs-per-request table")
    ap.add_argument("--no-passes", action="store_true", help="skip the separate sim and splat timings")
    ap.add_argument("--no-tune", action="store_true", help="serve with the default wave shape")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    B = args.requests_per_step
    nslices = args.warmup + args.steps
    count = stream_length(args.warmup, args.steps, B, args.latency_requests)

    if args.impl == "reference":
        # The reference's CPU path on rank 0 only; other ranks do no work.
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        stream = make_stream(1, count)
        slices = [stream[i * B:(i + 1) * B] for i in range(nslices)]
        budget = max(3.0, args.cpu_seconds / 2)
        for s in slices[:args.warmup]:
            cpu_sample([s], 0.2, threads)
        vals, steps_total, secs_total, rays_total = [], 0, 0.0, 0
        for s in slices[args.warmup:]:
            v, rays, steps, secs, desc = cpu_sample([s], budget / max(args.steps, 1), threads)
            vals.append(v)
            steps_total += steps
            secs_total += secs
            rays_total += rays
        value = steps_total / secs_total
        line = {
            "metric": "ray-steps/s, served mixed request stream (4096-step E/L drift < 1e-5), p50/p99 ms",
            "value": value, "unit": "ray-steps/s", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * secs_total / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "served mixed request stream, 40 req/s Poisson, 1M-particle 128^3 disk",
                       "requests_per_step": B, "stream_seed": 1},
            "cpu_baseline": {"value": value, "unit": "ray-steps/s", "cores": threads, "kind": "port",
                             "sample": desc},
            "e2e": {"value": value, "unit": "ray-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import gargantua_b200 as g

    ctx, ps, vol = setup_world(local, world)
    peak = ctx.fp32_peak_tflops()
    # Weak scaling: every rank serves its own stream (seed 1 + rank).
    stream = make_stream(1 + rank, count)
    slices = [stream[i * B:(i + 1) * B] for i in range(nslices)]
    assert all(len(sl) == B for sl in slices), "every slice is full"
    lat_stream = stream[nslices * B:nslices * B + args.latency_requests]
    shape = {"chunk_rays": 32, "wave_rays": 4 << 20, "max_waves_in_flight": 6, "steps_per_round": 8, "refill_idle": 8,
             "schedule": 0,
             "chosen_by": "defaults"}
    if not args.no_tune:
        # Untimed: the server's wave shape from a sample of other requests
        # with the same mix (a different stream seed).
        from gargantua_b200 import autotune

        sample = [spec_of(q) for q in make_stream(1000 + rank)[:16]]
        tuned = autotune.tune_server(ctx, vol, sample)
        shape = {k: tuned[k] for k in ("chunk_rays", "wave_rays", "max_waves_in_flight", "steps_per_round",
                                         "refill_idle", "schedule")}
        shape["chosen_by"] = "gargantua_b200.autotune.tune_server on 16 requests of stream seed 1000"
    batched = g.Server(ctx, vol, g.types.SERVE_BATCHED,
                       **{k: v for k, v in shape.items() if k != "chosen_by"})

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for s in slices[:args.warmup]:
        serve_slice(batched, s, pinned_outputs(ctx, s))
    timed = slices[args.warmup:]
    pins = [pinned_outputs(ctx, s) for s in timed]
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    span = busy = wall = 0.0
    steps_total = flops_total = 0.0
    launches = 0
    d2h = 0
    drift_over = rays_total = 0
    served_per_step = []
    for s, pin in zip(timed, pins):
        results, w, sp, bu, la = serve_slice(batched, s, pin)
        wall += w
        span += sp
        busy += bu
        launches += la
        served_per_step.append(sum(r.ray_steps for r in results) / max(sp, 1e-12))
        for q, r in zip(s, results):
            steps_total += r.ray_steps
            flops_total += flops_of(q, r)
            d2h += q["width"] * q["height"] * 8
            rays_total += r.counters.rays
            drift_over += r.counters.overDriftBudget
    barrier()
    clock_info = clocks.stop()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    span_max = max_over_ranks(span)
    wall_max = max_over_ranks(wall)
    steps_all = sum_over_ranks(steps_total)
    value = steps_all / span_max
    e2e = steps_all / wall_max

    # The per-request baselines on the same slices: the reference's march as
    # written, and this library's plain FP32 step arithmetic launched per
    # request (what batching and compensation add over it).
    def plain_baseline(server_plain):
        serve_slice(server_plain, slices[0], pinned_outputs(ctx, slices[0]))
        barrier()
        sampler = ClockSampler(local)
        sampler.start()
        p_span = p_wall = p_steps = 0.0
        per_step = []
        for s, pin in zip(timed, pins):
            results, w, sp, bu, la = serve_slice(server_plain, s, pin)
            steps = sum(r.ray_steps for r in results)
            p_span += sp
            p_wall += w
            p_steps += steps
            per_step.append(steps / max(sp, 1e-12))
        barrier()
        p_clocks = sampler.stop()
        p_span, p_wall, p_steps = max_over_ranks(p_span), max_over_ranks(p_wall), sum_over_ranks(p_steps)
        out = {"value": p_steps / p_span, "e2e": p_steps / p_wall, "unit": "ray-steps/s",
               "served_over_plain": value / (p_steps / p_span),
               "served_over_plain_e2e": e2e / (p_steps / p_wall),
               "per_step": {"min": min(per_step), "median": statistics.median(per_step), "max": max(per_step)},
               "clocks": p_clocks,
               "served_over_plain_median": statistics.median(served_per_step) / statistics.median(per_step)}
        if len(lat_stream) >= 8:
            out["p50_ms"], out["p99_ms"] = latency_replay(server_plain, lat_stream)
        return out

    plain = plain_lane = None
    plain_servers = {}
    if not args.no_plain:
        plain_servers = {"as_written": g.Server(ctx, vol, g.types.SERVE_SERIAL_PLAIN_AS_WRITTEN),
                         "plain": g.Server(ctx, vol, g.types.SERVE_SERIAL_PLAIN)}
        plain = plain_baseline(plain_servers["as_written"])
        plain["kernel"] = "per-request image kernel, the reference's step arithmetic as written (march.metal)"
        plain_lane = plain_baseline(plain_servers["plain"])
        plain_lane["kernel"] = "per-request image kernel, this library's plain FP32 step arithmetic"

    p50 = p99 = None
    if len(lat_stream) >= 8:
        p50, p99 = latency_replay(batched, lat_stream)

    classes = None
    if not args.no_classes and plain_servers:
        classes = class_table({"served": batched, **plain_servers})
    for server in plain_servers.values():
        server.close()

    passes = measure_passes(ctx, g, torch) if not args.no_passes else None

    drift_oracle = drift_vs_oracle(ctx, timed) if (rank == 0 and world == 1) else None

    cpu = None
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        cv, crays, csteps, csecs, desc = cpu_sample(timed, args.cpu_seconds, threads)
        # The reference's oracle renders serially (Sources/Oracle/LensedRender.swift:3-5):
        # the same integrators on one thread, a shorter bounded sample.
        sv, srays, ssteps, ssecs, sdesc = cpu_sample(timed, max(1.0, args.cpu_seconds / 4), 1)
        cpu = {"value": cv, "unit": "ray-steps/s", "cores": threads, "kind": "port", "sample": desc,
               "single_thread": sv, "single_thread_sample": sdesc}

    achieved = flops_total / busy / 1e12
    summary = {
        "served_G_ray_steps_s": round(value / 1e9, 2),
        "served_over_plain_as_written": round(plain["served_over_plain"], 3) if plain else None,
        "served_over_plain_lane": round(plain_lane["served_over_plain"], 3) if plain_lane else None,
        "p50_ms": p50, "p99_ms": p99,
        "plain_as_written_p50_p99_ms": [plain.get("p50_ms"), plain.get("p99_ms")] if plain else None,
        "timed_requests": len(timed) * B, "latency_requests": len(lat_stream),
        "drift_4096": drift_summary(drift_oracle),
        "classes_x_as_written_x_plain": ({r["class"]: [r.get("x_as_written"), r.get("x_plain")] for r in classes}
                                         if classes else None),
    }
    line = {
        "metric": "ray-steps/s, served mixed request stream (4096-step E/L drift < 1e-5), p50/p99 ms",
        "value": value,
        "unit": "ray-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * span_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "served mixed request stream (configs: 40 req/s Poisson; 320x180..3840x2160; "
                               "256/4096 steps; spin 0/0.5/0.9; r 40-120; 1M-particle settled disk, 128^3)",
                   "requests_per_step": B, "stream_seed": 1, "stream_requests": count,
                   "precision": "compensated FP32 + FP64 re-integration",
                   "server_shape": shape,
                   "l2": "inputs larger than L2 (outputs up to 66 MB per request, 8-200 MB per step)"},
        "p50_ms": p50,
        "p99_ms": p99,
        "per_step": {"min": min(served_per_step), "median": statistics.median(served_per_step),
                     "max": max(served_per_step)},
        "plain_per_request": plain,
        "plain_lane_per_request": plain_lane,
        "classes": classes,
        "drift": {"rays": rays_total, "over_budget": drift_over, "vs_fp64_oracle": drift_oracle},
        "e2e": {"value": e2e, "unit": "ray-steps/s", "h2d_bytes_per_step": int(B * 64),
                "d2h_bytes_per_step": int(d2h / max(args.steps, 1))},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": SERVE_KERR_TRAFFIC_BYTES,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                       "serve_kerr_chunks_kernel launch serving a 1920x1080 4096-step Kerr still",
                     "peak_source": "measured FP32 FMA microbenchmark (gg_measure_fp32_peak) on this GPU",
                     "kernel": "serve_kerr_chunks_kernel + serve_schwarzschild_chunks_kernel (persistent, "
                               "work-stealing)",
                     "device_busy_fraction": busy / max(span, 1e-12)},
        "cpu_baseline": cpu,
        "passes": passes,
        "clocks": clock_info,
        # Kernels the server launched in the timed steps (gg_server_totals).
        "gpu_launches": int(sum_over_ranks(launches)),
        "summary": summary,
    }
    batched.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
