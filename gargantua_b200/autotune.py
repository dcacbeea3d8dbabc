"""Shape autotuning: the splat's brick shape and the server's wave shape,
chosen by timing candidates on the caller's own data.

* Splat: gg_splat_autotune times gg_splat_bin under every brick edge and
  chunk (and direct atomics) on the given particles and keeps the fastest in
  the volume, per deposit mode.
* March: the image kernels' thread block, timed on a frame of the caller's
  shape (tune_march_block).
* Server: each candidate (chunk_rays, wave_rays, max_waves_in_flight; the
  schedule and refill cadence when asked for) serves
  the same sample of requests closed-loop on a fresh server; the candidate
  with the smallest device span (first launch to last, CUDA events) wins.
  The sample should look like the traffic to come: sizes, step budgets and
  spins in the same proportions.

Results are plain dicts, so a host can store them and pass them back as
ServerConfig fields (gg_server_config) on later runs.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import host as H
from . import types as T

CHUNKS = (32, 64, 128)
WAVES = (2 << 20, 4 << 20, 8 << 20)
IN_FLIGHT = (3, 6, 8)
CADENCES = ((8, 8), (4, 4), (16, 8), (8, 16))  # (steps_per_round, refill_idle)
# The chunk schedule only, by default: on a 16-request sample the lane-refill
# schedule once timed fastest by a hair and then served the full stream at
# 60 G ray-steps/s against the chunk schedule's 80 (B200, 7 blocks per SM).
# A caller may still tune it in by passing `schedules`.
SCHEDULES = (T.SCHEDULE_CHUNKS,)


@dataclass
class ServerShape:
    chunk_rays: int
    wave_rays: int
    max_waves_in_flight: int
    steps_per_round: int
    refill_idle: int
    schedule: int
    span_seconds: float
    ray_steps: int

    @property
    def rate(self) -> float:
        return self.ray_steps / self.span_seconds if self.span_seconds > 0 else 0.0

    def config(self) -> dict:
        return {"chunk_rays": self.chunk_rays, "wave_rays": self.wave_rays,
                "max_waves_in_flight": self.max_waves_in_flight, "steps_per_round": self.steps_per_round,
                "refill_idle": self.refill_idle, "schedule": self.schedule}


def tune_splat(ps: H.Particles, vol: H.Volume) -> dict:
    """Both deposit modes; the volume keeps the winners (its sums are left
    zeroed)."""
    out = {}
    for exact in (True, False):
        edge, chunk, ms = vol.autotune(ps, exact)
        out["exact" if exact else "stochastic"] = {"brick_edge": edge, "chunk": chunk, "ms": ms}
    return out


def _serve(ctx: H.Context, vol, specs, shape: dict, memory_bytes: int) -> ServerShape:
    server = H.Server(ctx, vol, T.SERVE_BATCHED, memory_bytes=memory_bytes, **shape)
    try:
        server.totals(reset=True)
        tickets = [server.submit(s) for s in specs]
        steps = sum(int(server.wait(t)[2].ray_steps) for t in tickets)
        tot = server.totals(reset=True)
        return ServerShape(shape["chunk_rays"], shape["wave_rays"], shape["max_waves_in_flight"],
                           shape["steps_per_round"], shape["refill_idle"], shape["schedule"], tot["span_seconds"],
                           steps)
    finally:
        server.close()


def tune_server(ctx: H.Context, vol, specs: list[H.RequestSpec], memory_bytes: int = 0, chunks=CHUNKS, waves=WAVES,
                in_flight=IN_FLIGHT, cadences=CADENCES, schedules=SCHEDULES, repeats: int = 2) -> dict:
    """The fastest server shape for `specs`, found one group of settings at
    a time (the schedule, chunk size and waves in flight, then wave size,
    then, for the lane-refill schedule, its cadence), as ServerConfig
    keyword arguments, plus every trial's rate."""
    if not specs:
        raise ValueError("tune_server needs a sample of requests")
    best = {"chunk_rays": chunks[0], "wave_rays": waves[len(waves) // 2], "max_waves_in_flight": in_flight[0],
            "steps_per_round": cadences[0][0], "refill_idle": cadences[0][1], "schedule": schedules[0]}
    _serve(ctx, vol, specs[:2], best, memory_bytes)  # build kernels, graphs, pools
    trials = []

    def measure(shape):
        r = min((_serve(ctx, vol, specs, shape, memory_bytes) for _ in range(repeats)), key=lambda t: t.span_seconds)
        trials.append(r)
        return r

    groups = [
        [{"schedule": sch} for sch in schedules],
        [{"chunk_rays": c, "max_waves_in_flight": f} for c in chunks for f in in_flight],
        [{"wave_rays": w} for w in waves],
        [{"steps_per_round": spr, "refill_idle": idle} for spr, idle in cadences],
    ]
    for group in groups:
        if "steps_per_round" in group[0] and best["schedule"] != T.SCHEDULE_LANE_REFILL:
            continue  # the cadence only matters to the lane-refill schedule
        if len(group) == 1:
            best = dict(best, **group[0])
            continue
        results = []
        for change in group:
            shape = dict(best, **change)
            results.append(measure(shape))
        best = max(results, key=lambda t: t.rate).config()
    win = max((t for t in trials if t.config() == best), key=lambda t: t.rate)
    return dict(best, rate=win.rate, trials=[dict(t.config(), rate=t.rate) for t in trials])


MARCH_BLOCKS = ((8, 8), (16, 4), (32, 2), (8, 4), (16, 8), (32, 4), (8, 16), (16, 16), (32, 8))


def tune_march_block(ctx: H.Context, vol, u: T.MarchUniforms, precision: int = T.PRECISION_PLAIN,
                     blocks=MARCH_BLOCKS, repeats: int = 3) -> dict:
    """The image kernels' thread block for this frame shape: gg_march timed
    (CUDA events on the context's stream) under each block shape; the
    context keeps the fastest."""
    import torch

    w, h = u.resolution.x, u.resolution.y
    ext = torch.cuda.ExternalStream(H.lib().gg_context_stream(ctx.handle))
    targets = H.Targets(ctx, w, h)
    times = {}
    try:
        for bw, bh in blocks:
            ctx.set_march_block(bw, bh)
            H.march(ctx, vol, u, targets, precision)  # warm
            best = float("inf")
            for _ in range(repeats):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(ext)
                H.march(ctx, vol, u, targets, precision)
                e1.record(ext)
                ext.synchronize()
                best = min(best, e0.elapsed_time(e1))
            times[(bw, bh)] = best
    finally:
        targets.close()
    win = min(times, key=times.get)
    ctx.set_march_block(*win)
    return {"block": list(win), "ms": times[win], "trials": [{"block": list(k), "ms": v} for k, v in times.items()]}

