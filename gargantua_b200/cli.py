"""Command line: `python -m gargantua_b200 ...`, the options of gargantua's
own executable (Options.swift:36-154) over this library.

Parsing is pure (parse() raises UsageError, exit 64) so it runs without a
GPU. Commands:

* `--still out.png [--width W --height H] [--spin a] [--camera az,el,d]
  [--seed S] [--preset p] [--particles N] [--volume n] [--sequence N]`:
  settle the disk (Still.swift:36-46), splat it exactly, serve the still as
  one request through the batched server (compensated FP32 with FP64
  re-integration, 4096-step still policy), tone-map on the device and write
  a PNG. --sequence adds N frames of 960x540 interactive marches with the
  simulation advancing (Still.swift:67-90).
* `bench`: per-pass device timings on the preset's scene (Bench.swift:27-45:
  5 warm-ups, 30 timed, mean / p50 / max), printed as one JSON object.
* `version`, `constants` (the constant table as a C header).

* `validate`: the goldens the device can be held to without the FP64
  oracle, run by the C++ host (gargantua_b200/cli/gargantua validate, the
  same library): exit 0 when all pass, 1 when one fails.

The interactive window (MTKView, HUD, MetalFX) needs a display and has no
counterpart here; running without a command says so and exits 2.
"""
from __future__ import annotations

import json
import os
import sys
import time
from dataclasses import dataclass

VERSION = "0.1.0"

USAGE = ("usage: python -m gargantua_b200 [--preset small|default|max] [--particles N] [--volume 96|128|192|256] "
         "[--seed S] [--strategy march|bake] [--fps-cap 30|60] [--no-upscale] [--still out.png --width W --height H] "
         "[--spin a] [--camera az,el,d] [--sequence N] | bench | validate | version | constants")

PRESETS = {  # Presets.swift:72-93
    "small": (250_000, 96, 640, 360),
    "default": (1_000_000, 128, 960, 540),
    "max": (4_000_000, 256, 960, 540),
}


class UsageError(Exception):
    """A command line the program cannot run: one sentence, exit 64."""


class OperationalError(Exception):
    """A failure while running: one sentence, exit 2."""


@dataclass
class Options:
    command: str = "interactive"
    still_path: str | None = None
    preset: str = "default"
    particles: int | None = None
    volume: int | None = None
    seed: int = 1
    strategy: str = "march"
    fps_cap: int = 60
    upscale: bool = True
    width: int = 3840
    height: int = 2160
    sequence: int | None = None
    camera: tuple[float, float, float] | None = None
    spin: float = 0.0

    @property
    def configuration(self) -> tuple[int, int, int, int]:
        particles, volume, mw, mh = PRESETS[self.preset]
        return (self.particles or particles, self.volume or volume, mw, mh)


def parse(argv: list[str]) -> Options:
    """Options.parse (Options.swift:60-154): same flags, same refusals."""
    o = Options()
    i = 0

    def value(flag: str) -> str:
        nonlocal i
        i += 1
        if i >= len(argv):
            raise UsageError(f"{flag} needs a value. {USAGE}")
        return argv[i]

    def integer(flag: str) -> int:
        text = value(flag)
        try:
            n = int(text)
        except ValueError:
            n = 0
        if n <= 0:
            raise UsageError(f"{flag} needs a positive integer, not {text}.")
        return n

    while i < len(argv):
        a = argv[i]
        if a in ("bench", "validate", "version", "constants"):
            o.command = a
        elif a == "--preset":
            name = value(a)
            if name not in PRESETS:
                raise UsageError(f"unknown preset {name}; choose small, default or max.")
            o.preset = name
        elif a == "--particles":
            o.particles = integer(a)
        elif a == "--volume":
            v = integer(a)
            if v not in (96, 128, 192, 256):
                raise UsageError("volume must be 96, 128, 192 or 256.")
            o.volume = v
        elif a == "--seed":
            text = value(a)
            if not text.isdigit() or int(text) >= 1 << 64:
                raise UsageError(f"seed must be an unsigned 64 bit integer, not {text}.")
            o.seed = int(text)
        elif a == "--strategy":
            name = value(a)
            if name not in ("march", "bake"):
                raise UsageError(f"unknown strategy {name}; choose march or bake.")
            o.strategy = name
        elif a == "--fps-cap":
            cap = integer(a)
            if cap not in (30, 60):
                raise UsageError("fps cap must be 30 or 60.")
            o.fps_cap = cap
        elif a == "--no-upscale":
            o.upscale = False
        elif a == "--still":
            o.command = "still"
            o.still_path = value(a)
        elif a == "--width":
            o.width = integer(a)
        elif a == "--height":
            o.height = integer(a)
        elif a == "--sequence":
            o.sequence = integer(a)
        elif a == "--spin":
            text = value(a)
            try:
                spin = float(text)
            except ValueError:
                spin = -1.0
            if not 0.0 <= spin <= 0.998:
                raise UsageError("spin must be between 0 and 0.998.")
            o.spin = spin
        elif a == "--camera":
            parts = []
            for p in value(a).split(","):
                try:
                    parts.append(float(p))
                except ValueError:
                    pass
            if len(parts) != 3 or not 2.5 < parts[2] < 60:
                raise UsageError("camera needs azimuth,elevation,distance with distance between 2.5 and 60.")
            o.camera = (parts[0], parts[1], parts[2])
        else:
            raise UsageError(f"unknown argument {a}. {USAGE}")
        i += 1
    return o


def orbit_camera(o: Options):
    """OrbitCamera.from (Camera.swift:5-13): elevation clamped to +-1.5."""
    from . import host as H

    cam = H.OrbitCamera()
    if o.camera:
        cam.azimuth = o.camera[0]
        cam.elevation = min(max(o.camera[1], -1.5), 1.5)
        cam.distance = min(max(o.camera[2], 2.5), 60.0)
    return cam


def _settled_disk(ctx, o: Options):
    from . import host as H
    from . import types as T

    particles, size, _, _ = o.configuration
    ps = H.Particles(ctx, particles, o.seed, T.POTENTIAL_PACZYNSKI_WIITA)
    print(f"settling {particles} particles for 600 substeps", flush=True)
    ps.advance(600 // 2, seed_first=True)
    vol = H.Volume(ctx, size)
    vol.splat(ps, exact=True)
    ctx.synchronize()
    return ps, vol


def still(o: Options) -> None:
    """Still.render (Still.swift:8-98), the march served as one request."""
    from . import host as H

    ctx = H.Context()
    ps, vol = _settled_disk(ctx, o)
    cam = orbit_camera(o)
    server = H.Server(ctx, vol)
    spec = H.RequestSpec(o.width, o.height, 4096, o.spin, cam.azimuth, cam.elevation, cam.distance, cam.fov_y,
                         star_seed=o.seed & 0xFFFFFFFF)
    t0 = time.perf_counter()
    pixels, _, res = server.wait(server.submit(spec), timeout_s=3600.0)
    wall = time.perf_counter() - t0
    if res.status != 0:
        raise OperationalError(f"The still failed: {H.lib().gg_status_name(res.status).decode()}.")
    totals = server.totals(reset=True)
    span = max(totals["span_seconds"], 1e-12)
    print(f"served {o.width} by {o.height}: {res.ray_steps} ray steps, {res.fp64_rays} rays re-integrated in FP64, "
          f"device {span * 1e3:.2f} ms ({res.ray_steps / span / 1e9:.2f} G ray-steps/s), wall {wall * 1e3:.1f} ms",
          flush=True)
    print_counters(res.counters)
    server.close()
    targets = H.Targets(ctx, o.width, o.height)
    targets.write(color=pixels)
    rgba = targets.tonemap(1.0, False, H.DRIFT_BUDGET_STILL)
    targets.close()
    if o.sequence:
        _sequence(ctx, ps, vol, cam, o)
    H.write_png(o.still_path, rgba)
    print(f"still {os.path.abspath(o.still_path)}", flush=True)
    ctx.close()


def counters_line(c) -> str | None:
    """The HUD's validation line (Renderer.swift:133-137) for a frame's
    MarchCounters; None when no ray was marched."""
    if c.rays == 0:
        return None
    return (f"drift over budget {100.0 * c.overDriftBudget / c.rays:.2f} percent, {c.exhausted} exhausted, "
            f"{c.captured} captured")


def print_counters(c) -> None:
    line = counters_line(c)
    if line:
        print(line, flush=True)


def _sequence(ctx, ps, vol, cam, o: Options) -> None:
    """Still.swift:67-90: interactive frames with the simulation advancing
    and the stochastic deposit, written beside the still."""
    from . import host as H

    targets = H.Targets(ctx, 960, 540)
    folder = os.path.dirname(os.path.abspath(o.still_path))
    for frame in range(o.sequence):
        ps.step(1)
        vol.splat(ps, exact=False)
        u = H.uniforms(cam, 960, 540, H.Settings.interactive(), H.DRIFT_BUDGET_INTERACTIVE, True, o.seed, spin=o.spin)
        if o.spin == 0.0:
            ctx.enable_tables(u, float(cam.distance))
        print_counters(H.march(ctx, vol, u, targets))
        H.write_png(os.path.join(folder, f"seq-{frame:03d}.png"), targets.tonemap())
    targets.close()
    print(f"sequence of {o.sequence} frames beside the still", flush=True)


def _timing(fn, sync, warmup: int = 5, iterations: int = 30) -> dict:
    """Bench.time (Bench.swift:34-44): each call waited to completion."""
    samples = []
    for k in range(warmup + iterations):
        t0 = time.perf_counter()
        fn()
        sync()
        if k >= warmup:
            samples.append(time.perf_counter() - t0)
    s = sorted(samples)
    return {"mean_ms": 1e3 * sum(s) / len(s), "p50_ms": 1e3 * s[len(s) // 2], "max_ms": 1e3 * s[-1]}


def bench(o: Options) -> dict:
    """Bench.run (Bench.swift): every pass timed on the preset's scene."""
    from . import host as H
    from . import types as T

    ctx = H.Context()
    ps, vol = _settled_disk(ctx, o)
    particles, size, mw, mh = o.configuration
    cam = orbit_camera(o)
    sync = ctx.synchronize
    report = {"preset": o.preset, "particles": particles, "volume": size, "march": [mw, mh], "spin": o.spin}
    report["sim_step"] = _timing(lambda: ps.step(1), sync)
    report["splat_exact"] = _timing(lambda: vol.splat(ps, exact=True), sync)
    report["splat_stochastic"] = _timing(lambda: vol.splat(ps, exact=False), sync)
    targets = H.Targets(ctx, mw, mh)
    u = H.uniforms(cam, mw, mh, H.Settings.interactive(), H.DRIFT_BUDGET_INTERACTIVE, True, o.seed, spin=o.spin)
    if o.spin == 0.0:
        ctx.enable_tables(u, float(cam.distance))
    report["march_interactive"] = _timing(lambda: H.march(ctx, vol, u, targets), sync)
    report["march_interactive_as_written"] = _timing(
        lambda: H.march(ctx, vol, u, targets, T.PRECISION_PLAIN_AS_WRITTEN), sync)
    us = H.uniforms(cam, mw, mh, H.Settings.still(), H.DRIFT_BUDGET_STILL, True, o.seed, spin=o.spin)
    if o.spin == 0.0:
        ctx.enable_tables(us, float(cam.distance))
    report["march_still_compensated"] = _timing(lambda: H.march(ctx, vol, us, targets, T.PRECISION_COMPENSATED),
                                                sync, iterations=10)
    report["march_still_plain"] = _timing(lambda: H.march(ctx, vol, us, targets), sync, iterations=10)
    report["march_still_as_written"] = _timing(lambda: H.march(ctx, vol, us, targets, T.PRECISION_PLAIN_AS_WRITTEN),
                                               sync, iterations=10)
    report["present"] = _timing(lambda: targets.tonemap(), sync)
    if o.strategy == "bake":
        bake = H.Bake(ctx, mw, mh)
        ub = H.uniforms(cam, mw, mh, H.Settings.interactive(), H.DRIFT_BUDGET_INTERACTIVE, True, o.seed,
                        bake_spacing=H.Bake.spacing(size))
        if o.spin == 0.0:
            ctx.enable_tables(ub, float(cam.distance))
        report["bake_full"] = _timing(lambda: bake.bake_full(ub), sync, iterations=5)
        bake.overflow(reset=True)
        bake.bake_full(ub)
        sync()
        report["bake_truncated_rays"] = bake.overflow()  # rays whose samples overran BAKE_SAMPLES
        report["walk"] = _timing(lambda: bake.walk(vol, ub, targets), sync)
        bake.close()
    targets.close()
    ctx.close()
    print(json.dumps(report), flush=True)
    return report


def constants_header() -> str:
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "..", "include", "gargantua_constants.h")) as fh:
        return fh.read()


def validate(o: Options) -> int:
    """Validate.run (Validate.swift:19-55) through the C++ host, which links
    the same library: its table on stdout, its exit code returned."""
    import subprocess

    exe = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cli", "gargantua")
    if not os.path.exists(exe):
        raise OperationalError(f"validate runs the C++ host, which is not built: make -C {os.path.dirname(exe)}.")
    argv = [exe, "validate", "--preset", o.preset, "--seed", str(o.seed)]
    if o.particles:
        argv += ["--particles", str(o.particles)]
    if o.volume:
        argv += ["--volume", str(o.volume)]
    sys.stdout.flush()
    return subprocess.run(argv).returncode


def run(o: Options) -> int:
    if o.command == "version":
        print(f"gargantua-b200 {VERSION}")
    elif o.command == "constants":
        sys.stdout.write(constants_header())
    elif o.command == "still":
        still(o)
    elif o.command == "bench":
        bench(o)
    elif o.command == "validate":
        return validate(o)
    else:
        raise OperationalError("The interactive window needs a display; use --still or bench.")
    return 0


def main(argv: list[str] | None = None) -> int:
    """Exit codes as Exit.swift:5-18: 64 usage, 2 operational, 0 success."""
    try:
        o = parse(sys.argv[1:] if argv is None else argv)
    except UsageError as e:
        sys.stderr.write(f"{e}\n")
        return 64
    try:
        return run(o)
    except OperationalError as e:
        sys.stderr.write(f"{e}\n")
        return 2
    except Exception as e:  # GargantuaError and the like: one sentence, exit 2
        from ._lib import GargantuaError

        if isinstance(e, GargantuaError):
            sys.stderr.write(f"{e}\n")
            return 2
        raise
    return 0
