"""ctypes mirrors of the ShaderTypes.h structs (include/gargantua_types.h).

Field names, order, sizes and offsets follow gargantua's
Sources/ShaderTypes/include/ShaderTypes.h:14-162 under Apple's simd layout
rules (simd_float3 = 16 bytes, simd_float2 / simd_uint2 = 8 bytes); explicit
padding fields stand in for the alignment ctypes cannot express.
"""
import ctypes as C

f32, u32 = C.c_float, C.c_uint32


class Packed3(C.Structure):
    _fields_ = [("x", f32), ("y", f32), ("z", f32)]


class Float2(C.Structure):
    _fields_ = [("x", f32), ("y", f32)]


class Float3(C.Structure):
    """simd_float3: three floats padded to 16 bytes."""

    _fields_ = [("x", f32), ("y", f32), ("z", f32), ("pad_w", f32)]


class Float4(C.Structure):
    _fields_ = [("x", f32), ("y", f32), ("z", f32), ("w", f32)]


class UInt2(C.Structure):
    _fields_ = [("x", u32), ("y", u32)]


class Particle(C.Structure):
    _fields_ = [("position", Packed3), ("velocity", Packed3), ("temperature", f32), ("respawns", u32)]


class SimUniforms(C.Structure):
    _fields_ = [
        ("seed", UInt2),
        ("particleCount", u32),
        ("potential", u32),
        ("inverseCdfCount", u32),
        ("dt", f32),
        ("alpha", f32),
        ("temperatureScale", f32),
    ]


class PresentUniforms(C.Structure):
    _fields_ = [("hudRect", Float4), ("exposure", f32), ("hudVisible", u32), ("debugView", u32), ("driftBudget", f32)]


class GeodesicSettings(C.Structure):
    _fields_ = [
        ("stepFactor", f32),
        ("stepMin", f32),
        ("stepMax", f32),
        ("captureRadius", f32),
        ("escapeRadius", f32),
        ("stepCap", u32),
        ("emptyStepFactor", f32),
        ("emptyStepMax", f32),
    ]


class RayProbe(C.Structure):
    _fields_ = [("origin", Packed3), ("direction", Packed3)]


class RayProbeResult(C.Structure):
    _fields_ = [
        ("position", Packed3),
        ("direction", Packed3),
        ("drift", f32),
        ("outcome", u32),
        ("steps", u32),
        ("energy", f32),
        ("angularMomentum", f32),
    ]


class SplatUniforms(C.Structure):
    _fields_ = [
        ("volumeSize", u32),
        ("particleCount", u32),
        ("halfExtent", f32),
        ("peakTemperature", f32),
        ("emissionScale", f32),
        ("frame", u32),
        ("exactDeposit", u32),
        ("pad_", u32),
        ("seed", UInt2),
    ]


class MarchUniforms(C.Structure):
    _fields_ = [
        ("cameraPosition", Float3),
        ("cameraRight", Float3),
        ("cameraUp", Float3),
        ("cameraForward", Float3),
        ("tanHalfFov", Float2),
        ("resolution", UInt2),
        ("tileOrigin", UInt2),
        ("volumeHalfExtent", f32),
        ("opacityScale", f32),
        ("starBrightness", f32),
        ("driftBudget", f32),
        ("starSeed", u32),
        ("redshift", u32),
        ("bakeSpacing", f32),
        ("bakeCapacity", u32),
        ("sphereRadius", f32),
        ("cameraRadius", f32),
        ("sphereMaxB", f32),
        ("sphereTableMaxB", f32),
        ("cameraMaxB", f32),
        ("skyMinB", f32),
        ("skyMaxB", f32),
        ("spin", f32),
        ("jitter", Float2),
        ("geodesic", GeodesicSettings),
    ]


class BakedRay(C.Structure):
    _fields_ = [("count", u32), ("fallsIn", u32), ("directionXY", u32), ("directionZDepth", u32)]


class MarchCounters(C.Structure):
    _fields_ = [("rays", u32), ("overDriftBudget", u32), ("exhausted", u32), ("captured", u32)]


class Request(C.Structure):
    """gg_request (include/gargantua.h)."""

    _fields_ = [
        ("azimuth", f32), ("elevation", f32), ("distance", f32), ("fov_y", f32),
        ("width", u32), ("height", u32), ("step_cap", u32), ("spin", f32), ("star_seed", u32), ("flags", u32),
        ("output", C.c_void_p), ("debug_output", C.c_void_p), ("volume", C.c_void_p),
    ]


class RequestResult(C.Structure):
    _fields_ = [
        ("submitted", C.c_double), ("admitted", C.c_double), ("finished", C.c_double),
        ("ray_steps", C.c_uint64), ("samples", C.c_uint64), ("fp64_rays", C.c_uint64),
        ("counters", MarchCounters), ("status", C.c_int),
    ]


class ServerConfig(C.Structure):
    _fields_ = [("mode", C.c_int), ("memory_bytes", C.c_uint64), ("wave_rays", u32), ("chunk_rays", u32),
                ("max_waves_in_flight", u32), ("fp64_policy", u32), ("steps_per_round", u32), ("refill_idle", u32),
                ("schedule", u32)]


SCHEDULE_CHUNKS, SCHEDULE_LANE_REFILL = 0, 1


FP64_ESCAPING, FP64_ALL_FLAGGED = 0, 1
IPC_HANDLE_BYTES, MAX_PEERS = 64, 7  # GG_IPC_HANDLE_BYTES, GG_MAX_PEERS
SERVE_BATCHED, SERVE_SERIAL_PLAIN, SERVE_SERIAL_PLAIN_AS_WRITTEN = 0, 1, 2
REQUEST_NO_STARS, REQUEST_NO_REDSHIFT, REQUEST_BAKE = 1, 2, 4


# Sizes the C header pins with static assertions (gargantua_types.h).
LAYOUT = {
    Particle: 32,
    SimUniforms: 32,
    PresentUniforms: 32,
    GeodesicSettings: 32,
    RayProbe: 24,
    RayProbeResult: 44,
    SplatUniforms: 40,
    MarchUniforms: 192,
    BakedRay: 16,
    MarchCounters: 16,
}

RAY_CAPTURED, RAY_ESCAPED, RAY_EXHAUSTED = 0, 1, 2
POTENTIAL_NEWTONIAN, POTENTIAL_PACZYNSKI_WIITA = 0, 1
PRECISION_PLAIN, PRECISION_COMPENSATED, PRECISION_PLAIN_AS_WRITTEN, PRECISION_RENORMALISED = 0, 1, 2, 3
