"""Host-side mirror of gargantua's pass interface over the C ABI.

Names and argument meanings follow the Swift host: OrbitCamera
(Sources/Gargantua/Camera.swift), Schwarzschild.Settings .interactive/.still
(Sources/Oracle/Schwarzschild.swift:138-185), MarchPass.uniforms
(Passes/MarchPass.swift:61-98), Probes.aimed/cameraGrid
(Validation/Probes.swift:46-66), and thin owners for the context, particle
system, volume, targets and bake (GpuContext, ParticleSystem, Volume,
MarchPass.Targets, BakePass). Every call goes through libgargantua_b200.so;
errors raise GargantuaError, as the Swift host exits with code 2.
"""
from __future__ import annotations

import ctypes as C
import math
import weakref
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import types as T
from ._lib import check, lib, ptr

# Constants the host uses (include/gargantua_constants.h).
VOLUME_HALF_EXTENT = 30.0
VOLUME_OPACITY = 5e-4
STAR_BRIGHTNESS = 1.5
BAKE_SAMPLES = 96
BAKE_SPACING_VOXELS = 0.5
DRIFT_BUDGET_INTERACTIVE = 1e-4
DRIFT_BUDGET_STILL = 1e-5
R_CAPTURE = 2.02
R_ESCAPE = 60.0
T_PEAK = 8000.0
EMISSION_SCALE = 5e-4
STILL_SETTLE_STEPS = 600
SIM_SUBSTEPS = 2


@dataclass
class Settings:
    """Schwarzschild.Settings (Schwarzschild.swift:138-185)."""

    step_cap: int
    step_factor: float = 0.02
    step_min: float = 0.02
    step_max: float = 0.5
    capture_radius: float = R_CAPTURE
    escape_radius: float = R_ESCAPE
    empty_step_factor: float | None = None
    empty_step_max: float | None = None

    def __post_init__(self):
        if self.empty_step_factor is None:
            self.empty_step_factor = self.step_factor
        if self.empty_step_max is None:
            self.empty_step_max = self.step_max

    @staticmethod
    def interactive() -> "Settings":
        return Settings(step_cap=256, empty_step_factor=0.1, empty_step_max=3.0)

    @staticmethod
    def still() -> "Settings":
        return Settings(step_cap=4096, empty_step_factor=0.06, empty_step_max=1.5)

    def geodesic(self) -> T.GeodesicSettings:
        """MarchPass.settings (MarchPass.swift:61-65): infinities clamp to 1e9."""
        return T.GeodesicSettings(
            self.step_factor, self.step_min, min(self.step_max, 1e9), self.capture_radius, self.escape_radius,
            self.step_cap, self.empty_step_factor, min(self.empty_step_max, 1e9))


def f32(x: float) -> float:
    return float(np.float32(x))


@dataclass
class OrbitCamera:
    """Camera.swift:4-33: an orbit camera looking at the hole, disk in xy.

    The basis is computed in float32 like the Swift host's SIMD3<Float>."""

    azimuth: float = 0.6
    elevation: float = 0.32
    distance: float = 52.0
    fov_y: float = 50.0 * math.pi / 180.0

    def _f(self):
        az, el, d = np.float32(self.azimuth), np.float32(self.elevation), np.float32(self.distance)
        c = np.float32(np.cos(el))
        pos = d * np.array([c * np.float32(np.cos(az)), c * np.float32(np.sin(az)), np.float32(np.sin(el))],
                           np.float32)
        fwd = -pos / np.float32(np.sqrt(np.float32(pos @ pos)))
        right = np.cross(fwd, np.array([0, 0, 1], np.float32)).astype(np.float32)
        right = right / np.float32(np.sqrt(np.float32(right @ right)))
        up = np.cross(right, fwd).astype(np.float32)
        return pos.astype(np.float32), right, up, fwd.astype(np.float32)

    @property
    def position(self) -> np.ndarray:
        return self._f()[0]

    @property
    def right(self) -> np.ndarray:
        return self._f()[1]

    @property
    def up(self) -> np.ndarray:
        return self._f()[2]

    @property
    def forward(self) -> np.ndarray:
        return self._f()[3]


def _f3(v) -> T.Float3:
    return T.Float3(float(v[0]), float(v[1]), float(v[2]), 0.0)


def uniforms(camera: OrbitCamera, width: int, height: int, settings: Settings, drift_budget: float,
             redshift: bool, star_seed: int, stars: bool = True, tile_origin=(0, 0), jitter=(0.0, 0.0),
             bake_spacing: float = 0.0, spin: float = 0.0) -> T.MarchUniforms:
    """MarchPass.uniforms (MarchPass.swift:67-98) without the table step: call
    Context.enable_tables to turn on the sphere jump (DeflectionTables.apply)."""
    tan_half = np.float32(np.tan(np.float32(camera.fov_y) * np.float32(0.5)))
    pos, right, up, fwd = camera._f()
    u = T.MarchUniforms()
    u.cameraPosition = _f3(pos)
    u.cameraRight = _f3(right)
    u.cameraUp = _f3(up)
    u.cameraForward = _f3(fwd)
    u.tanHalfFov = T.Float2(float(tan_half * np.float32(width) / np.float32(height)), float(tan_half))
    u.resolution = T.UInt2(width, height)
    u.tileOrigin = T.UInt2(*tile_origin)
    u.volumeHalfExtent = VOLUME_HALF_EXTENT
    u.opacityScale = VOLUME_OPACITY
    u.starBrightness = STAR_BRIGHTNESS if stars else 0.0
    u.driftBudget = drift_budget
    u.starSeed = star_seed & 0xFFFFFFFF
    u.redshift = 1 if redshift else 0
    u.bakeSpacing = bake_spacing
    u.bakeCapacity = BAKE_SAMPLES
    u.spin = spin
    u.jitter = T.Float2(*jitter)
    u.geodesic = settings.geodesic()
    return u


@dataclass
class Launch:
    origin: np.ndarray
    direction: np.ndarray


def aimed(radius: float, b: float) -> Launch:
    """Probes.aimed (Probes.swift:46-49): from `radius` on the x axis toward
    the hole with impact parameter b, via the FP64 launch's position and
    direction (Schwarzschild.launch(radius:impactParameter:))."""
    f = 1.0 - 2.0 / radius
    dphi = b * math.sqrt(f) / radius
    dr = -math.sqrt(max(0.0, 1.0 - dphi * dphi))
    # The launch reproduces its origin and direction exactly (GeodesicTests.swift:6-16).
    return Launch(np.array([radius, 0.0, 0.0]), np.array([dr, dphi, 0.0]))


def camera_grid(camera: OrbitCamera, columns: int, rows: int, aspect: float) -> list[Launch]:
    """Probes.cameraGrid (Probes.swift:52-66)."""
    tan_half = float(np.float32(np.tan(np.float32(camera.fov_y) * np.float32(0.5))))
    origin = camera.position.astype(np.float64)
    right, up, fwd = camera.right.astype(np.float64), camera.up.astype(np.float64), camera.forward.astype(np.float64)
    out = []
    for row in range(rows):
        for col in range(columns):
            x = (2.0 * (col + 0.5) / columns - 1.0) * tan_half * aspect
            y = (1.0 - 2.0 * (row + 0.5) / rows) * tan_half
            d = fwd + x * right + y * up
            out.append(Launch(origin.copy(), d / np.linalg.norm(d)))
    return out


def as_float32_launch(l: Launch) -> Launch:
    """Round a launch to the single precision values the GPU receives."""
    return Launch(l.origin.astype(np.float32).astype(np.float64), l.direction.astype(np.float32).astype(np.float64))


class Context:
    """GpuContext (Gpu/GpuContext.swift): one device, one stream, a budget."""

    def __init__(self, device: int = 0, budget_bytes: int = 0):
        self.handle = C.c_void_p()
        self.device = device
        self._children = weakref.WeakSet()
        self._pinned_cache: dict[int, list[int]] = {}  # released page-locked blocks by size (pinned_array)
        check(lib().gg_context_create(device, budget_bytes, C.byref(self.handle)))

    def adopt(self, child) -> None:
        """Every handle dies before its context: close() closes them first."""
        self._children.add(child)

    def close(self):
        if self.handle:
            for child in list(self._children):
                child.close()
            for blocks in self._pinned_cache.values():
                for address in blocks:
                    lib().gg_host_free(address)
            self._pinned_cache.clear()
            lib().gg_context_destroy(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(lib().gg_context_synchronize(self.handle))

    def memory(self):
        b, u = C.c_uint64(), C.c_uint64()
        check(lib().gg_context_memory(self.handle, C.byref(b), C.byref(u)))
        return b.value, u.value

    def enable_tables(self, u: T.MarchUniforms, camera_radius: float) -> T.MarchUniforms:
        """DeflectionTables.update + apply (DeflectionTables.swift:57-76)."""
        check(lib().gg_tables_update(self.handle, camera_radius, C.byref(u)))
        return u

    def tables(self):
        n = 1024
        s, c, k = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32)
        check(lib().gg_tables_read(self.handle, ptr(s), ptr(c), ptr(k)))
        return s, c, k

    def atomic_peak_gadds(self, records: int = 128 ** 3) -> float:
        """Scattered 32-bit global atomic adds per second (G/s) into a grid
        of six-word records, the splat's ceiling."""
        r = C.c_double()
        check(lib().gg_measure_atomic_peak(self.handle, records, C.byref(r)))
        return r.value

    def shared_atomic_peak_gadds(self) -> float:
        """Scattered 32-bit shared-memory atomic adds per second (G/s) into a
        9^3 tile of six-word records, the brick splat's ceiling."""
        r = C.c_double()
        check(lib().gg_measure_shared_atomic_peak(self.handle, C.byref(r)))
        return r.value

    def capture_boundary(self, u: T.MarchUniforms, origin, base, axis, lo: float, hi: float, rays: int = 1024,
                         rounds: int = 3) -> float:
        """gg_capture_boundary: t of the capture boundary of the rays
        origin -> base + t axis, bisected in FP64 on the device."""
        o, b, a = (np.ascontiguousarray(v, np.float64) for v in (origin, base, axis))
        for v, what in ((o, "origin"), (b, "base"), (a, "axis")):
            expect_size(v, 3, what)
        t = C.c_double()
        check(lib().gg_capture_boundary(self.handle, C.byref(u), ptr(o), ptr(b), ptr(a), lo, hi, rays, rounds,
                                        C.byref(t)))
        return t.value

    def set_march_block(self, width: int, height: int):
        """gg_context_set_march_block: the image kernels' thread block."""
        check(lib().gg_context_set_march_block(self.handle, width, height))

    def set_fp64_policy(self, policy: int):
        """gg_context_set_fp64_policy for gg_march and gg_probe."""
        check(lib().gg_context_set_fp64_policy(self.handle, policy))

    def fp32_peak_tflops(self) -> float:
        t = C.c_double()
        check(lib().gg_measure_fp32_peak(self.handle, C.byref(t)))
        return t.value

    def blackbody(self) -> np.ndarray:
        out = np.zeros((256, 4), np.float32)
        check(lib().gg_context_blackbody(self.handle, out.ctypes.data_as(L.f32p), 256))
        return out

    def probe(self, launches: list[Launch], u: T.MarchUniforms, precision: int = T.PRECISION_PLAIN):
        """Probes.run (Probes.swift:26-43): float launches in, results out as a
        structured numpy array."""
        n = len(launches)
        arr = (T.RayProbe * n)()
        for k, l in enumerate(launches):
            arr[k].origin = T.Packed3(*[float(np.float32(x)) for x in l.origin])
            arr[k].direction = T.Packed3(*[float(np.float32(x)) for x in l.direction])
        res = (T.RayProbeResult * n)()
        check(lib().gg_probe(self.handle, C.byref(u), C.cast(arr, C.c_void_p), C.cast(res, C.c_void_p), n, precision))
        return probe_results_to_numpy(res)


def probe_results_to_numpy(res) -> dict:
    n = len(res)
    buf = np.frombuffer(bytes(res), dtype=np.dtype([
        ("position", "<f4", 3), ("direction", "<f4", 3), ("drift", "<f4"), ("outcome", "<u4"),
        ("steps", "<u4"), ("energy", "<f4"), ("angularMomentum", "<f4")]), count=n)
    return buf


class Particles:
    """ParticleSystem (Sim/ParticleSystem.swift) + SimPass (Passes/SimPass.swift)."""

    def __init__(self, ctx: Context, count: int, seed: int = 1, potential: int = T.POTENTIAL_PACZYNSKI_WIITA,
                 first_index: int = 0):
        self.ctx = ctx
        self.count = count
        self.seed = seed
        self.first_index = first_index
        self.handle = C.c_void_p()
        check(lib().gg_particles_create_shard(ctx.handle, count, first_index, seed, potential, C.byref(self.handle)))
        ctx.adopt(self)

    def close(self):
        if self.handle:
            lib().gg_particles_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def uniforms(self) -> T.SimUniforms:
        u = T.SimUniforms()
        check(lib().gg_particles_uniforms(self.handle, C.byref(u)))
        return u

    def seed_particles(self):
        check(lib().gg_particles_seed(self.handle))

    def step(self, dispatches: int = 1):
        check(lib().gg_particles_step(self.handle, dispatches))

    def advance(self, dispatches: int, seed_first: bool):
        """Validate.advance (Validate.swift:70-85)."""
        if seed_first:
            self.seed_particles()
        if dispatches:
            self.step(dispatches)

    def read(self) -> np.ndarray:
        """Particle records as an (n, 8) float32 array (respawns as bits in column 7)."""
        out = np.zeros((self.count, 8), np.float32)
        check(lib().gg_particles_read(self.handle, ptr(out), self.count))
        return out

    def write(self, parts: np.ndarray):
        parts = np.ascontiguousarray(parts, np.float32)
        expect_size(parts, self.count * 8, "particle records (count x 8 float32)")
        check(lib().gg_particles_write(self.handle, ptr(parts), self.count))

    def checksum(self) -> int:
        h = C.c_uint64()
        check(lib().gg_particles_checksum(self.handle, C.byref(h)))
        return h.value

    def seed_profile(self, fraction: float = 0.7, exponent: float = 3.0):
        """gg_particles_seed_profile: seed `fraction` of the particles from a
        power-law surface density ~ r^-exponent (the max preset's contention
        workload); call before seed_particles."""
        check(lib().gg_particles_seed_profile(self.handle, fraction, exponent))

    def profile_table(self) -> np.ndarray:
        out = np.zeros(1024, np.float32)
        check(lib().gg_particles_profile_table(self.handle, out.ctypes.data_as(L.f32p), 1024))
        return out

    def inverse_cdf(self) -> np.ndarray:
        out = np.zeros(1024, np.float32)
        check(lib().gg_particles_inverse_cdf(self.handle, out.ctypes.data_as(L.f32p), 1024))
        return out


def splat_uniforms(size: int, particles: int, seed: int, frame: int = 0, exact: bool = True) -> T.SplatUniforms:
    """SplatPass.uniforms (SplatPass.swift:21-31)."""
    u = T.SplatUniforms()
    u.volumeSize = size
    u.particleCount = particles
    u.halfExtent = VOLUME_HALF_EXTENT
    u.peakTemperature = T_PEAK
    u.emissionScale = EMISSION_SCALE
    u.frame = frame & 0xFFFFFFFF
    u.exactDeposit = 1 if exact else 0
    u.seed = T.UInt2(seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    return u


class Volume:
    """Volume (Gpu/Volume.swift) + SplatPass (Passes/SplatPass.swift)."""

    def __init__(self, ctx: Context, size: int):
        self.ctx = ctx
        self.size = size
        self.handle = C.c_void_p()
        self.frame = 0
        check(lib().gg_volume_create(ctx.handle, size, C.byref(self.handle)))
        ctx.adopt(self)

    def close(self):
        if self.handle:
            lib().gg_volume_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def splat(self, ps: Particles, exact: bool = True):
        """SplatPass.encode: bin, resolve, clear; the frame counter advances."""
        u = splat_uniforms(self.size, ps.count, ps.seed, self.frame, exact)
        check(lib().gg_splat(ps.handle, self.handle, C.byref(u)))
        self.frame += 1

    def bin(self, ps: Particles, exact: bool = True, frame: int | None = None):
        u = splat_uniforms(self.size, ps.count, ps.seed, self.frame if frame is None else frame, exact)
        check(lib().gg_splat_bin(ps.handle, self.handle, C.byref(u)))

    def set_shape(self, exact: bool, brick_edge: int, chunk: int = 0):
        """gg_volume_splat_shape: 0 = direct global atomics, else 4/8/16."""
        check(lib().gg_volume_splat_shape(self.handle, 1 if exact else 0, brick_edge, chunk))

    def autotune(self, ps: "Particles", exact: bool = True) -> tuple[int, int, float]:
        """gg_splat_autotune: (brick edge, chunk, ms) of the fastest shape."""
        u = splat_uniforms(self.size, ps.count, ps.seed, self.frame, exact)
        e, c, ms = C.c_uint32(), C.c_uint32(), C.c_float()
        check(lib().gg_splat_autotune(ps.handle, self.handle, C.byref(u), C.byref(e), C.byref(c), C.byref(ms)))
        return e.value, c.value, ms.value

    def resolve(self):
        u = splat_uniforms(self.size, 0, 0)
        check(lib().gg_splat_resolve(self.handle, C.byref(u), None))

    def clear(self):
        check(lib().gg_volume_clear(self.handle))

    def read_sums(self):
        n3 = self.size ** 3
        em = np.zeros(2 * n3, np.uint32)
        mo = np.zeros(3 * n3, np.int32)
        ma = np.zeros(n3, np.uint32)
        check(lib().gg_volume_read_sums(self.handle, ptr(em), ptr(mo), ptr(ma)))
        return em, mo, ma

    def write_sums(self, em: np.ndarray, mo: np.ndarray, ma: np.ndarray):
        em = np.ascontiguousarray(em, np.uint32)
        mo = np.ascontiguousarray(mo, np.int32)
        ma = np.ascontiguousarray(ma, np.uint32)
        n3 = self.size ** 3
        expect_size(em, 2 * n3, "emission sums")
        expect_size(mo, 3 * n3, "momentum sums")
        expect_size(ma, n3, "mass sums")
        check(lib().gg_volume_write_sums(self.handle, ptr(em), ptr(mo), ptr(ma)))

    def read(self):
        n3 = self.size ** 3
        e = np.zeros((n3, 4), np.float16)
        v = np.zeros((n3, 4), np.float16)
        check(lib().gg_volume_read(self.handle, ptr(e), ptr(v)))
        return e, v

    def write(self, emission: np.ndarray, velocity: np.ndarray):
        e = np.ascontiguousarray(emission, np.float16)
        v = np.ascontiguousarray(velocity, np.float16)
        expect_size(e, 4 * self.size ** 3, "emission texels (half4)")
        expect_size(v, 4 * self.size ** 3, "velocity texels (half4)")
        check(lib().gg_volume_write(self.handle, ptr(e), ptr(v)))


class Targets:
    """MarchPass.Targets (MarchPass.swift:35-50)."""

    def __init__(self, ctx: Context, width: int, height: int):
        self.ctx = ctx
        self.width, self.height = width, height
        self.handle = C.c_void_p()
        check(lib().gg_targets_create(ctx.handle, width, height, C.byref(self.handle)))
        ctx.adopt(self)

    def close(self):
        if self.handle:
            lib().gg_targets_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def read(self):
        n = self.width * self.height
        color = np.zeros((n, 4), np.float16)
        debug = np.zeros((n, 4), np.float16)
        depth = np.zeros(n, np.float32)
        check(lib().gg_targets_read(self.handle, ptr(color), ptr(debug), ptr(depth), None))
        return color, debug, depth

    def write(self, color: np.ndarray | None = None, debug: np.ndarray | None = None):
        """Load width*height half4 pixels (e.g. a served request's output)."""
        c = None if color is None else np.ascontiguousarray(color, np.float16)
        d = None if debug is None else np.ascontiguousarray(debug, np.float16)
        for a in (c, d):
            if a is not None and a.size != self.width * self.height * 4:
                raise ValueError(f"{a.size} values for a {self.width}x{self.height} half4 target")
        check(lib().gg_targets_write(self.handle, None if c is None else ptr(c), None if d is None else ptr(d)))

    def tonemap(self, exposure: float = 1.0, debug_view: bool = False, drift_budget: float = DRIFT_BUDGET_INTERACTIVE):
        u = T.PresentUniforms()
        u.exposure = exposure
        u.debugView = 1 if debug_view else 0
        u.driftBudget = drift_budget
        out = np.zeros((self.height, self.width, 4), np.uint8)
        check(lib().gg_tonemap(self.handle, C.byref(u), ptr(out)))
        return out


def march(ctx: Context, vol: Volume | None, u: T.MarchUniforms, targets: Targets,
          precision: int = T.PRECISION_PLAIN) -> T.MarchCounters:
    """MarchPass.encodeImage (MarchPass.swift:103-124)."""
    counters = T.MarchCounters()
    check(lib().gg_march(ctx.handle, vol.handle if vol else None, C.byref(u), targets.handle, precision,
                         C.byref(counters)))
    return counters


def march_stats(ctx: Context) -> tuple[int, int, int]:
    """Ray steps, gather samples and FP64-re-integrated rays of the last march."""
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
    check(lib().gg_march_stats(ctx.handle, C.byref(a), C.byref(b), C.byref(c)))
    return a.value, b.value, c.value


class Bake:
    """BakePass (Passes/BakePass.swift)."""

    def __init__(self, ctx: Context, width: int, height: int):
        self.ctx = ctx
        self.width, self.height = width, height
        self.handle = C.c_void_p()
        check(lib().gg_bake_create(ctx.handle, width, height, C.byref(self.handle)))
        ctx.adopt(self)

    def close(self):
        if self.handle:
            lib().gg_bake_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def spacing(volume_size: int) -> float:
        """BakePass.spacing (BakePass.swift:50-52)."""
        return float(np.float32(2.0 * VOLUME_HALF_EXTENT / volume_size * BAKE_SPACING_VOXELS))

    def bake_rows(self, u: T.MarchUniforms, row_begin: int, row_end: int):
        check(lib().gg_bake_rows(self.handle, C.byref(u), row_begin, row_end))

    def bake_full(self, u: T.MarchUniforms, frames: int = 4):
        """encodeFullBake: BAKE_FRAMES chunks of rows (BakePass.swift:55-84)."""
        rows = max(self.height // frames, 1)
        r = 0
        while r < self.height:
            n = min(rows, self.height - r)
            self.bake_rows(u, r, r + n)
            r += n

    def overflow(self, reset: bool = False) -> int:
        c = C.c_uint32()
        check(lib().gg_bake_overflow(self.handle, C.byref(c), 1 if reset else 0))
        return c.value

    def walk(self, vol: Volume | None, u: T.MarchUniforms, targets: Targets):
        check(lib().gg_walk(self.handle, vol.handle if vol else None, C.byref(u), targets.handle))

    def read(self):
        n = self.width * self.height
        samples = np.zeros((n, BAKE_SAMPLES, 4), np.float16)
        headers = np.zeros((n, 4), np.uint32)
        check(lib().gg_bake_read(self.handle, ptr(samples), ptr(headers)))
        return samples, headers


def write_png(path: str, rgba8: np.ndarray):
    rgba8 = np.ascontiguousarray(rgba8, np.uint8)
    if rgba8.ndim != 3 or rgba8.shape[2] != 4:
        raise ValueError(f"a PNG needs height x width x 4 bytes, not shape {rgba8.shape}")
    h, w = rgba8.shape[:2]
    check(lib().gg_write_png(path.encode(), ptr(rgba8), w, h))


@dataclass
class RequestSpec:
    """One still request (gg_request): orbit camera, size, step budget, spin."""

    width: int
    height: int
    step_cap: int = 4096
    spin: float = 0.0
    azimuth: float = 0.6
    elevation: float = 0.32
    distance: float = 52.0
    fov_y: float = 50.0 * math.pi / 180.0
    star_seed: int = 1
    flags: int = 0
    volume: "Volume | None" = None  # None: the server's volume


PINNED_CACHE_PER_SIZE = 4  # released blocks a context keeps for reuse, per size


def pinned_array(ctx: Context, shape, dtype=np.float16) -> np.ndarray:
    """A numpy array in page-locked host memory (gg_host_alloc): the
    library's copies into or out of it run at the link's rate. Page-locking
    costs time of its own, so once the array and every view of it are gone
    the block goes back to the context, which hands it to the next array of
    the same size (up to PINNED_CACHE_PER_SIZE kept per size) and releases
    it (gg_host_free) when it closes. The contents start undefined."""
    dtype = np.dtype(dtype)
    shape = tuple(int(x) for x in (shape if isinstance(shape, (tuple, list)) else (shape,)))
    nbytes = int(np.prod(shape)) * dtype.itemsize
    size = max(nbytes, 1)
    cached = ctx._pinned_cache.get(size)
    if cached:
        address = cached.pop()
    else:
        p = C.c_void_p()
        check(lib().gg_host_alloc(ctx.handle, size, C.byref(p)))
        address = p.value
    owner = weakref.ref(ctx)
    free = lib().gg_host_free

    def release(_block):
        try:
            c = owner()
            if c is not None and c.handle:
                kept = c._pinned_cache.setdefault(size, [])
                if len(kept) < PINNED_CACHE_PER_SIZE:
                    kept.append(address)
                    return
            free(address)
        except Exception:
            pass

    # A ctypes array over the block whose finaliser hands it back; numpy
    # arrays made from it keep it alive through their base.
    block_type = type("PinnedBlock", (C.c_char * size,), {"__del__": release})
    block = block_type.from_address(address)
    return np.frombuffer(block, dtype=np.uint8, count=nbytes).view(dtype).reshape(shape)


def expect_size(a: np.ndarray, values: int, what: str) -> None:
    """The library reads or writes exactly `values` elements at an array's
    address: refuse any other size before it does."""
    if a.size != values:
        raise ValueError(f"{what}: {a.size} values given, {values} expected")


def check_pixel_buffer(output: np.ndarray, pixels: int) -> None:
    """A request's output array: the library writes pixels x 4 half floats
    to its address, so anything smaller, strided or of another type is
    refused here rather than overrun."""
    if not isinstance(output, np.ndarray) or output.dtype != np.float16:
        raise TypeError("the output must be a numpy float16 array")
    if not output.flags["C_CONTIGUOUS"] or not output.flags["WRITEABLE"]:
        raise ValueError("the output must be a writeable C-contiguous array")
    if output.size != pixels * 4:
        raise ValueError(f"the output holds {output.size} half floats; the request writes {pixels * 4}")


class Server:
    """gg_server: continuous batching (SERVE_BATCHED) or the serial plain
    per-request baseline (SERVE_SERIAL_PLAIN) over one resident volume."""

    def __init__(self, ctx: Context, vol: Volume | None, mode: int = T.SERVE_BATCHED, memory_bytes: int = 0,
                 wave_rays: int = 0, chunk_rays: int = 0, max_waves_in_flight: int = 0,
                 fp64_policy: int = T.FP64_ESCAPING, steps_per_round: int = 0, refill_idle: int = 0,
                 schedule: int = T.SCHEDULE_CHUNKS):
        self.ctx = ctx
        self.handle = C.c_void_p()
        cfg = T.ServerConfig(mode, memory_bytes, wave_rays, chunk_rays, max_waves_in_flight, fp64_policy,
                             steps_per_round, refill_idle, schedule)
        check(lib().gg_server_create(ctx.handle, vol.handle if vol else None, C.byref(cfg), C.byref(self.handle)))
        ctx.adopt(self)
        self._buffers = {}

    def close(self):
        if self.handle:
            lib().gg_server_destroy(self.handle)
            self.handle = C.c_void_p()
            self._buffers.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, spec: RequestSpec, output: np.ndarray | None = None, debug: bool = False) -> int:
        """Queue a request; `output` (height*width*4 float16, kept alive here)
        receives the pixels. Without one, the request gets page-locked
        arrays (pinned_array), into which the result copies at the link's
        rate."""
        n = spec.width * spec.height
        if output is None:
            output = pinned_array(self.ctx, (n, 4), np.float16)
        check_pixel_buffer(output, n)
        dbg = pinned_array(self.ctx, (n, 4), np.float16) if debug else None
        q = T.Request(spec.azimuth, spec.elevation, spec.distance, spec.fov_y, spec.width, spec.height,
                      spec.step_cap, spec.spin, spec.star_seed & 0xFFFFFFFF, spec.flags,
                      output.ctypes.data, dbg.ctypes.data if dbg is not None else None,
                      spec.volume.handle if spec.volume is not None else None)
        t = C.c_uint64()
        check(lib().gg_server_submit(self.handle, C.byref(q), C.byref(t)))
        self._buffers[t.value] = (output, dbg)
        return t.value

    def poll(self, ticket: int) -> bool:
        d = C.c_int()
        check(lib().gg_server_poll(self.handle, ticket, C.byref(d)))
        return bool(d.value)

    def wait(self, ticket: int, timeout_s: float = 600.0):
        """(pixels, debug-or-None, RequestResult). A cancelled request raises
        GargantuaError with status GG_ERR_CANCELLED (9)."""
        res = T.RequestResult()
        status = lib().gg_server_wait(self.handle, ticket, timeout_s, C.byref(res))
        if status == 9:  # the library forgot the ticket: so do its buffers
            self._buffers.pop(ticket, None)
        check(status)
        out, dbg = self._buffers.pop(ticket)
        return out, dbg, res

    def cancel(self, ticket: int) -> None:
        """gg_server_cancel: withdraw a request still waiting for admission
        (GargantuaError with GG_ERR_NOT_READY once it is admitted)."""
        check(lib().gg_server_cancel(self.handle, ticket))

    def totals(self, reset: bool = False):
        a, b, c, d, e = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_double(), C.c_double()
        check(lib().gg_server_totals(self.handle, 1 if reset else 0, C.byref(a), C.byref(b), C.byref(c), C.byref(d),
                                     C.byref(e)))
        return {"requests": a.value, "ray_steps": b.value, "launches": c.value, "busy_seconds": d.value,
                "span_seconds": e.value}


class Sequence:
    """A sequence render request (the still's --sequence frames,
    Still.swift:67-90) served alongside other requests: its own particle
    system advances one dispatch and splats stochastically into its own
    volume before each frame, and each frame is an interactive 256-step
    request on `server` marching that volume. Frames run in order: frame
    k + 1's splat waits until frame k's rays are done with the volume."""

    def __init__(self, server: "Server", ctx: Context, particles: int, size: int, frames: int, width: int = 960,
                 height: int = 540, spin: float = 0.0, seed: int = 1, camera: OrbitCamera | None = None,
                 settle_dispatches: int = 300):
        self.server = server
        self.frames = frames
        self.camera = camera or OrbitCamera()
        self.width, self.height, self.spin, self.seed = width, height, spin, seed
        self.particles = Particles(ctx, particles, seed)
        self.particles.advance(settle_dispatches, seed_first=True)
        self.volume = Volume(ctx, size)

    def spec(self) -> RequestSpec:
        c = self.camera
        return RequestSpec(self.width, self.height, 256, self.spin, c.azimuth, c.elevation, c.distance, c.fov_y,
                           star_seed=self.seed & 0xFFFFFFFF, volume=self.volume)

    def frame(self, timeout_s: float = 600.0):
        """Advance, splat, serve one frame: (pixels, RequestResult)."""
        self.particles.step(1)
        self.volume.splat(self.particles, exact=False)
        pixels, _, res = self.server.wait(self.server.submit(self.spec()), timeout_s)
        return pixels, res

    def run(self):
        return [self.frame() for _ in range(self.frames)]

    def snapshot(self) -> dict:
        """The sequence's state between frames: the particle records (the AoS
        Particle layout), their FNV-1a checksum (Validate.swift:378-387) and
        the splat's frame counter. Every later random draw is pcg4d(index,
        event, seed), so this is all a resume needs."""
        return {"particles": self.particles.read(), "checksum": self.particles.checksum(),
                "splat_frame": self.volume.frame}

    def restore(self, snap: dict) -> None:
        """Resume from snapshot(): the particle records are written back and
        checked against the snapshot's checksum, and the splat's frame
        counter is restored, so the following frames are the ones the
        snapshotted sequence would have rendered, bit for bit."""
        self.particles.write(snap["particles"])
        got = self.particles.checksum()
        if got != snap["checksum"]:
            raise ValueError(f"particle checksum {got:016x} does not match the snapshot's {snap['checksum']:016x}")
        self.volume.frame = int(snap["splat_frame"])

    def close(self):
        self.volume.close()
        self.particles.close()

