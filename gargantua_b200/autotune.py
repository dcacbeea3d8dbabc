"""Shape autotuning: the splat's brick shape and the server's wave shape,
chosen by timing candidates on the caller's own data.

* Splat: gg_splat_autotune times gg_splat_bin under every brick edge and
  chunk (and direct atomics) on the given particles and keeps the fastest in
  the volume, per deposit mode.
* Server: each candidate (chunk_rays, wave_rays, max_waves_in_flight) serves
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
IN_FLIGHT = (2, 3)


@dataclass
class ServerShape:
    chunk_rays: int
    wave_rays: int
    max_waves_in_flight: int
    span_seconds: float
    ray_steps: int

    @property
    def rate(self) -> float:
        return self.ray_steps / self.span_seconds if self.span_seconds > 0 else 0.0


def tune_splat(ps: H.Particles, vol: H.Volume) -> dict:
    """Both deposit modes; the volume keeps the winners (its sums are left
    zeroed)."""
    out = {}
    for exact in (True, False):
        edge, chunk, ms = vol.autotune(ps, exact)
        out["exact" if exact else "stochastic"] = {"brick_edge": edge, "chunk": chunk, "ms": ms}
    return out


def _serve(ctx: H.Context, vol, specs, chunk: int, wave: int, flight: int, memory_bytes: int) -> ServerShape:
    server = H.Server(ctx, vol, T.SERVE_BATCHED, memory_bytes=memory_bytes, wave_rays=wave, chunk_rays=chunk,
                      max_waves_in_flight=flight)
    try:
        server.totals(reset=True)
        tickets = [server.submit(s) for s in specs]
        steps = sum(int(server.wait(t)[2].ray_steps) for t in tickets)
        tot = server.totals(reset=True)
        return ServerShape(chunk, wave, flight, tot["span_seconds"], steps)
    finally:
        server.close()


def tune_server(ctx: H.Context, vol, specs: list[H.RequestSpec], memory_bytes: int = 0, chunks=CHUNKS, waves=WAVES,
                in_flight=IN_FLIGHT, repeats: int = 2) -> dict:
    """The fastest (chunk_rays, wave_rays, max_waves_in_flight) for `specs`,
    as ServerConfig keyword arguments, plus every candidate's rate."""
    if not specs:
        raise ValueError("tune_server needs a sample of requests")
    _serve(ctx, vol, specs[:2], CHUNKS[0], WAVES[0], IN_FLIGHT[0], memory_bytes)  # build kernels, graphs, pools
    trials = []
    for chunk in chunks:
        for wave in waves:
            for flight in in_flight:
                best = None
                for _ in range(repeats):
                    r = _serve(ctx, vol, specs, chunk, wave, flight, memory_bytes)
                    if best is None or r.span_seconds < best.span_seconds:
                        best = r
                trials.append(best)
    win = max(trials, key=lambda t: t.rate)
    return {"chunk_rays": win.chunk_rays, "wave_rays": win.wave_rays, "max_waves_in_flight": win.max_waves_in_flight,
            "rate": win.rate,
            "trials": [{"chunk_rays": t.chunk_rays, "wave_rays": t.wave_rays,
                        "max_waves_in_flight": t.max_waves_in_flight, "rate": t.rate} for t in trials]}
