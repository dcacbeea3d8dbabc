"""ctypes access to the oracle (oracle/liboracle.so) for the tests.

The oracle is the checker: a C restatement of gargantua's FP64 oracle and
FP32 replicas of its particle and deposit kernels. Nothing in the product
imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle.so")

CAPTURED, ESCAPED, EXHAUSTED = 0, 1, 2

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_ip = _i32p
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class Settings(C.Structure):
    """o_settings, the oracle's Schwarzschild.Settings (Schwarzschild.swift:138-185)."""

    _fields_ = [
        ("step_factor", C.c_double),
        ("step_min", C.c_double),
        ("step_max", C.c_double),
        ("capture_radius", C.c_double),
        ("escape_radius", C.c_double),
        ("step_cap", C.c_int64),
        ("empty_step_factor", C.c_double),
        ("empty_step_max", C.c_double),
    ]


class KerrSettings(C.Structure):
    """o_kerr_settings (KerrGeodesic.swift:176-197)."""

    _fields_ = [
        ("step_factor", C.c_double),
        ("step_min", C.c_double),
        ("step_max", C.c_double),
        ("capture_margin", C.c_double),
        ("escape_radius", C.c_double),
        ("step_cap", C.c_int64),
    ]


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class Ray(C.Structure):
    _fields_ = [
        ("s", C.c_double * 6),
        ("e1", Vec3),
        ("e2", Vec3),
        ("energy", C.c_double),
        ("angular_momentum", C.c_double),
    ]


def _build() -> None:
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    _build()
    L = C.CDLL(LIB_PATH)
    d, i, u32, u64, i64 = C.c_double, C.c_int, C.c_uint32, C.c_uint64, C.c_int64
    P = C.POINTER
    sig = {
        "o_pcg4d": (None, [P(u32), P(u32)]),
        "o_hash_draw": (None, [u64, u32, u32, u32, P(u32)]),
        "o_hash_unit": (d, [u32]),
        "o_gaussian_pair": (None, [d, d, P(d), P(d)]),
        "o_potential_energy": (d, [i, d]),
        "o_potential_gradient": (d, [i, d]),
        "o_circular_speed": (d, [i, d]),
        "o_angular_frequency": (d, [i, d]),
        "o_circular_energy": (d, [i, d]),
        "o_circular_angular_momentum": (d, [i, d]),
        "o_disk_shape": (d, [d, d]),
        "o_disk_temperature": (d, [d, d]),
        "o_disk_peak_radius": (d, []),
        "o_steady_surface_density": (d, [d]),
        "o_radial_number_density": (d, [d]),
        "o_radial_inverse_cdf": (None, [i, i, _dp]),
        "o_disk_spawn": (None, [u32, u32, u64, _dp, i, i, _dp]),
        "o_circular_orbit": (None, [d, d, i, _dp]),
        "o_dynamics_step": (None, [i, d, d, _dp]),
        "o_dynamics_removed": (i, [_dp, _dp]),
        "o_specific_energy": (d, [i, _dp]),
        "o_angular_momentum_z": (d, [_dp]),
        "o_disk_settle": (None, [u32, u64, u32, i, d, d, _dp, P(u32)]),
        "o_disk_inner_edge": (d, [_dp, i, d, d, d]),
        "o_settings_interactive": (None, [P(Settings)]),
        "o_settings_still": (None, [P(Settings)]),
        "o_f": (d, [d]),
        "o_launch": (None, [_dp, _dp, P(Ray)]),
        "o_launch_b": (None, [d, d, P(Ray)]),
        "o_energy": (d, [P(d)]),
        "o_angular_momentum": (d, [P(d)]),
        "o_null_residual": (d, [P(d)]),
        "o_ray_position": (None, [P(Ray), _dp]),
        "o_ray_direction": (None, [P(Ray), _dp]),
        "o_integrate": (i, [P(Ray), P(Settings), P(i64), P(d)]),
        "o_redshift_factor": (d, [d, _dp, _dp]),
        "o_deflection": (d, [P(Ray), P(Ray)]),
        "o_critical_impact_parameter": (d, [d, P(Settings), i]),
        "o_integrate_batch": (None, [_dp, i, P(Settings), _dp, i]),
        "o_kerr_settings_default": (None, [P(KerrSettings), i64]),
        "o_kerr_outer_horizon": (d, [d]),
        "o_kerr_null_residual": (d, [d, _dp]),
        "o_kerr_carter": (d, [d, _dp]),
        "o_kerr_radius": (d, [d, _dp]),
        "o_kerr_launch": (None, [d, _dp, _dp, _dp]),
        "o_kerr_position": (None, [d, _dp, _dp]),
        "o_kerr_direction": (None, [d, _dp, _dp]),
        "o_kerr_integrate": (i, [d, _dp, P(KerrSettings), P(i64), P(d)]),
        "o_kerr_bisect_critical_xi": (d, [d, d, d, P(KerrSettings), i]),
        "o_kerr_critical_xi": (d, [d, d]),
        "o_kerr_critical_eta": (d, [d, d]),
        "o_kerr_photon_orbits": (None, [d, P(d), P(d)]),
        "o_kerr_integrate_batch": (None, [d, _dp, i, P(KerrSettings), _dp, i]),
        "o_max_impact_parameter": (d, [d]),
        "o_sweep": (d, [d, d, i]),
        "o_table_impact_parameter": (d, [d, d, d]),
        "o_table_coordinate": (d, [d, d, d]),
        "o_periapsis": (d, [d]),
        "o_turning_sweep": (d, [d, d, i]),
        "o_escape_sweep": (d, [d, d, i]),
        "o_sweep_table": (None, [d, i, i, _dp]),
        "o_sky_table": (None, [d, d, i, i, _dp]),
        "o_blackbody_color": (None, [d, _dp]),
        "o_blackbody_chromaticity": (None, [d, P(d), P(d)]),
        "o_blackbody_table": (None, [i, d, d, _dp]),
        "o_blackbody_coordinate": (d, [d, d, d]),
        "o_volume_sample": (None, [i, d, _dp, _dp, _dp, _dp, _dp]),
        "o_lensed_image": (None, [i, i, _dp, i, d, _dp, _dp, P(Settings), d, d, i, _dp, i]),
        "o_luminance": (d, [_dp]),
        "o_side_ratio": (d, [_dp, i, i]),
        "o32_seed": (None, [_fp, u32, u32, u32, u32, _fp, u32, C.c_float, u32]),
        "o32_step": (None, [_fp, u32, u32, u32, u32, _fp, u32, C.c_float, C.c_float, C.c_float, u32, i, u32]),
        "o32_seed_profile": (None, [_fp, u32, u32, u32, u32, _fp, u32, C.c_float, u32, _fp, C.c_float]),
        "o_fnv1a": (u64, [C.c_void_p, u64]),
        "o32_deposit": (None, [_fp, u32, u32, C.c_float, C.c_float, C.c_float, u32, u32, u32, u32, _u32p, _i32p, _u32p,
                                u32, i]),
        "o32_resolve": (None, [_u32p, _i32p, _u32p, u32, C.c_float, C.c_float, _fp, i, _fp, _fp, i]),
        "o_pbr_neutral": (None, [_dp, _dp]),
        "o32_present": (None, [_fp, u32, C.c_float, u32, C.c_float, _fp]),
        "o32_srgb8": (None, [_fp, C.c_uint64, _u8p]),
        "o_bake_batch": (None, [_dp, i, C.POINTER(Settings), C.c_double, C.c_double, i, _dp, _ip, _ip, _ip, _dp, i]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def still() -> Settings:
    s = Settings()
    lib().o_settings_still(C.byref(s))
    return s


def interactive() -> Settings:
    s = Settings()
    lib().o_settings_interactive(C.byref(s))
    return s


def kerr_settings(step_cap: int) -> KerrSettings:
    s = KerrSettings()
    lib().o_kerr_settings_default(C.byref(s), step_cap)
    return s


def launch(origin, direction) -> Ray:
    r = Ray()
    lib().o_launch(np.asarray(origin, np.float64), np.asarray(direction, np.float64), C.byref(r))
    return r


def launch_b(radius: float, b: float) -> Ray:
    r = Ray()
    lib().o_launch_b(radius, b, C.byref(r))
    return r


def integrate(ray: Ray, settings: Settings):
    steps = C.c_int64()
    drift = C.c_double()
    outcome = lib().o_integrate(C.byref(ray), C.byref(settings), C.byref(steps), C.byref(drift))
    return outcome, steps.value, drift.value


def position(ray: Ray) -> np.ndarray:
    out = np.zeros(3)
    lib().o_ray_position(C.byref(ray), out)
    return out


def direction(ray: Ray) -> np.ndarray:
    out = np.zeros(3)
    lib().o_ray_direction(C.byref(ray), out)
    return out


def integrate_batch(probes: np.ndarray, settings: Settings, threads: int = 0) -> np.ndarray:
    """probes: (n, 6) origin+direction -> (n, 11) position, direction, drift,
    outcome, steps, E, L."""
    probes = np.ascontiguousarray(probes, np.float64)
    out = np.zeros((len(probes), 11))
    lib().o_integrate_batch(probes, len(probes), C.byref(settings), out, threads)
    return out


def kerr_integrate_batch(spin: float, probes: np.ndarray, settings: KerrSettings, threads: int = 0) -> np.ndarray:
    probes = np.ascontiguousarray(probes, np.float64)
    out = np.zeros((len(probes), 11))
    lib().o_kerr_integrate_batch(spin, probes, len(probes), C.byref(settings), out, threads)
    return out


def inverse_cdf(count: int = 1024, resolution: int = 8192) -> np.ndarray:
    out = np.zeros(count)
    lib().o_radial_inverse_cdf(count, resolution, out)
    return out


def hash_draw(seed: int, index: int, event: int, lane: int = 0):
    out = (C.c_uint32 * 4)()
    lib().o_hash_draw(seed, index, event, lane, out)
    return tuple(out)


def blackbody_table(count: int = 256, tmin: float = 1000.0, tmax: float = 40000.0) -> np.ndarray:
    out = np.zeros((count, 3))
    lib().o_blackbody_table(count, tmin, tmax, out)
    return out


def sweep_table(radius: float, count: int, intervals: int) -> np.ndarray:
    out = np.zeros(count)
    lib().o_sweep_table(radius, count, intervals, out)
    return out


def sky_table(camera_radius: float, sphere_radius: float, count: int, intervals: int) -> np.ndarray:
    out = np.zeros(count)
    lib().o_sky_table(camera_radius, sphere_radius, count, intervals, out)
    return out


def seed32(n: int, seed: int, potential: int, cdf: np.ndarray, temperature_scale: float,
           first_index: int = 0) -> np.ndarray:
    parts = np.zeros((n, 8), np.float32)
    cdf = np.ascontiguousarray(cdf, np.float32)
    lib().o32_seed(parts, n, seed & 0xFFFFFFFF, seed >> 32, potential, cdf, len(cdf), temperature_scale, first_index)
    return parts


def seed32_profile(n: int, seed: int, potential: int, cdf: np.ndarray, temperature_scale: float,
                   profile: np.ndarray, fraction: float, first_index: int = 0) -> np.ndarray:
    parts = np.zeros((n, 8), np.float32)
    cdf = np.ascontiguousarray(cdf, np.float32)
    profile = np.ascontiguousarray(profile, np.float32)
    lib().o32_seed_profile(parts, n, seed & 0xFFFFFFFF, seed >> 32, potential, cdf, len(cdf), temperature_scale,
                           first_index, profile, fraction)
    return parts


def step32(parts: np.ndarray, seed: int, potential: int, cdf: np.ndarray, dt: float, alpha: float,
           temperature_scale: float, dispatches: int, threads: int = 0, first_index: int = 0) -> None:
    cdf = np.ascontiguousarray(cdf, np.float32)
    lib().o32_step(parts, len(parts), seed & 0xFFFFFFFF, seed >> 32, potential, cdf, len(cdf), dt, alpha,
                   temperature_scale, dispatches, threads, first_index)


def fnv1a(buf: np.ndarray) -> int:
    buf = np.ascontiguousarray(buf)
    return lib().o_fnv1a(buf.ctypes.data, buf.nbytes)


def deposit32(parts: np.ndarray, size: int, frame: int, exact: bool, seed: int, half_extent: float = 30.0,
              peak_temperature: float = 8000.0, emission_scale: float = 5e-4, first_index: int = 0,
              threads: int = 1):
    n3 = size ** 3
    em = np.zeros(2 * n3, np.uint32)
    mo = np.zeros(3 * n3, np.int32)
    ma = np.zeros(n3, np.uint32)
    lib().o32_deposit(np.ascontiguousarray(parts, np.float32), len(parts), size, half_extent, peak_temperature,
                      emission_scale, frame, 1 if exact else 0, seed & 0xFFFFFFFF, seed >> 32, em, mo, ma,
                      first_index, threads)
    return em, mo, ma


def resolve32(em, mo, ma, size: int, bb_rgb: np.ndarray, half_extent: float = 30.0, peak_temperature: float = 8000.0,
              threads: int = 1):
    n3 = size ** 3
    eo = np.zeros((n3, 4), np.float32)
    vo = np.zeros((n3, 4), np.float32)
    bb = np.ascontiguousarray(bb_rgb, np.float32)
    lib().o32_resolve(em, mo, ma, size, half_extent, peak_temperature, bb, len(bb), eo, vo, threads)
    return eo, vo


def lensed_image(width: int, height: int, camera: np.ndarray, size: int, half_extent: float,
                 emission: np.ndarray, velocity: np.ndarray, settings: Settings, opacity: float = 5e-4,
                 slab: float = 6.0, redshift: bool = True, threads: int = 0) -> np.ndarray:
    out = np.zeros((height * width, 3))
    lib().o_lensed_image(width, height, np.ascontiguousarray(camera, np.float64), size, half_extent,
                         np.ascontiguousarray(emission, np.float64), np.ascontiguousarray(velocity, np.float64),
                         C.byref(settings), opacity, slab, 1 if redshift else 0, out, threads)
    return out


def luminance(rgb: np.ndarray) -> np.ndarray:
    return 0.2126 * rgb[..., 0] + 0.7152 * rgb[..., 1] + 0.0722 * rgb[..., 2]


def side_ratio(lum: np.ndarray, width: int, height: int) -> float:
    lum = np.ascontiguousarray(lum, np.float64)
    return lib().o_side_ratio(lum, width, height)


def present32(rgba_half: np.ndarray, exposure: float = 1.0, debug_view: bool = False,
              drift_budget: float = 1e-4) -> np.ndarray:
    """The tone-map kernel's output for half4 pixels (n x 4 float16): the
    FP32 replica of PBR Neutral or the drift heat map, rounded to half as the
    fragment returns it, then encoded to 8-bit sRGB; alpha 255."""
    n = len(rgba_half)
    src = np.ascontiguousarray(rgba_half.astype(np.float32))
    rgb = np.zeros((n, 3), np.float32)
    lib().o32_present(src, n, exposure, 1 if debug_view else 0, drift_budget, rgb)
    halved = np.ascontiguousarray(rgb.astype(np.float16).astype(np.float32))
    out = np.full((n, 4), 255, np.uint8)
    codes = np.zeros((n, 3), np.uint8)
    lib().o32_srgb8(halved, halved.size, codes)
    out[:, :3] = codes
    return out


def bake_batch(probes: np.ndarray, settings: Settings, spacing: float, half_extent: float = 30.0,
               capacity: int = 96, threads: int = 0):
    """FP64 bake of rays launched at the camera: samples (n x capacity x 4),
    counts, overflowed, falls_in, direction_depth (n x 4)."""
    probes = np.ascontiguousarray(probes, np.float64)
    n = len(probes)
    samples = np.zeros((n, capacity, 4))
    counts = np.zeros(n, np.int32)
    over = np.zeros(n, np.int32)
    falls = np.zeros(n, np.int32)
    dd = np.zeros((n, 4))
    lib().o_bake_batch(probes, n, C.byref(settings), spacing, half_extent, capacity, samples, counts, over, falls, dd,
                       threads)
    return samples, counts, over, falls, dd
