"""Loader for the in-tree sm_100a library (libgargantua_b200.so) and the
argument types of every C entry point in include/gargantua.h.

There is no fallback: if the library is missing, importing this module's
`lib()` raises, and every call that fails on the device raises GargantuaError
with the library's own sentence (gg_last_error).
"""
import ctypes as C
import os

from . import types as T

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgargantua_b200.so")

STATUS = {
    0: "ok",
    1: "invalid argument",
    2: "out of memory",
    3: "over budget",
    4: "device error",
    5: "timeout",
    6: "not ready",
    7: "no device",
    8: "unsupported",
    9: "cancelled",
}


class GargantuaError(RuntimeError):
    """A failed library call: `status` is the gg_status code."""

    def __init__(self, status: int, sentence: str):
        super().__init__(f"{STATUS.get(status, status)}: {sentence}")
        self.status = status
        self.sentence = sentence


_lib = None

P = C.POINTER
vp = C.c_void_p
u8p = P(C.c_uint8)
u16p = P(C.c_uint16)
u32p = P(C.c_uint32)
i32p = P(C.c_int32)
f32p = P(C.c_float)
i, u32, u64 = C.c_int, C.c_uint32, C.c_uint64

SIGNATURES = {
    "gg_version": (C.c_char_p, []),
    "gg_last_error": (C.c_char_p, []),
    "gg_status_name": (C.c_char_p, [i]),
    "gg_context_create": (i, [i, u64, P(vp)]),
    "gg_context_destroy": (None, [vp]),
    "gg_context_synchronize": (i, [vp]),
    "gg_context_memory": (i, [vp, P(u64), P(u64)]),
    "gg_context_stream": (vp, [vp]),
    "gg_host_alloc": (i, [vp, u64, P(vp)]),
    "gg_host_free": (None, [vp]),
    "gg_context_blackbody": (i, [vp, f32p, u32]),
    "gg_particles_create": (i, [vp, u32, u64, u32, P(vp)]),
    "gg_particles_destroy": (None, [vp]),
    "gg_particles_create_shard": (i, [vp, u32, u32, u64, u32, P(vp)]),
    "gg_particles_seed_profile": (i, [vp, C.c_float, C.c_float]),
    "gg_particles_profile_table": (i, [vp, f32p, u32]),
    "gg_particles_uniforms": (i, [vp, P(T.SimUniforms)]),
    "gg_particles_seed": (i, [vp]),
    "gg_particles_step": (i, [vp, u32]),
    "gg_particles_read": (i, [vp, vp, u32]),
    "gg_particles_write": (i, [vp, vp, u32]),
    "gg_particles_checksum": (i, [vp, P(u64)]),
    "gg_particles_inverse_cdf": (i, [vp, f32p, u32]),
    "gg_volume_create": (i, [vp, u32, P(vp)]),
    "gg_volume_destroy": (None, [vp]),
    "gg_splat": (i, [vp, vp, P(T.SplatUniforms)]),
    "gg_splat_bin": (i, [vp, vp, P(T.SplatUniforms)]),
    "gg_splat_resolve": (i, [vp, P(T.SplatUniforms), vp]),
    "gg_volume_clear": (i, [vp]),
    "gg_volume_read_sums": (i, [vp, vp, vp, vp]),
    "gg_volume_write_sums": (i, [vp, vp, vp, vp]),
    "gg_volume_sums": (i, [vp, P(vp), P(u64)]),
    "gg_volume_ipc_handle": (i, [vp, vp]),
    "gg_volume_attach_peers": (i, [vp, vp, u32]),
    "gg_volume_splat_shape": (i, [vp, i, u32, u32]),
    "gg_splat_autotune": (i, [vp, vp, P(T.SplatUniforms), P(u32), P(u32), P(C.c_float)]),
    "gg_volume_read": (i, [vp, vp, vp]),
    "gg_volume_write": (i, [vp, vp, vp]),
    "gg_tables_update": (i, [vp, C.c_float, P(T.MarchUniforms)]),
    "gg_tables_read": (i, [vp, vp, vp, vp]),
    "gg_context_set_march_block": (i, [vp, u32, u32]),
    "gg_context_set_fp64_policy": (i, [vp, i]),
    "gg_targets_create": (i, [vp, u32, u32, P(vp)]),
    "gg_targets_destroy": (None, [vp]),
    "gg_targets_read": (i, [vp, vp, vp, vp, vp]),
    "gg_targets_write": (i, [vp, vp, vp]),
    "gg_march": (i, [vp, vp, P(T.MarchUniforms), vp, i, P(T.MarchCounters)]),
    "gg_probe": (i, [vp, P(T.MarchUniforms), vp, vp, u32, i]),
    "gg_capture_boundary": (i, [vp, P(T.MarchUniforms), vp, vp, vp, C.c_double, C.c_double, u32, u32,
                                P(C.c_double)]),
    "gg_march_stats": (i, [vp, P(u64), P(u64), P(u64)]),
    "gg_march_compensated_noalloc": (i, [vp, vp, P(T.MarchUniforms), vp, P(T.MarchCounters)]),
    "gg_bake_create": (i, [vp, u32, u32, P(vp)]),
    "gg_bake_destroy": (None, [vp]),
    "gg_bake_rows": (i, [vp, P(T.MarchUniforms), u32, u32]),
    "gg_bake_overflow": (i, [vp, P(u32), i]),
    "gg_walk": (i, [vp, vp, P(T.MarchUniforms), vp]),
    "gg_bake_read": (i, [vp, vp, vp]),
    "gg_tonemap": (i, [vp, P(T.PresentUniforms), vp]),
    "gg_write_png": (i, [C.c_char_p, vp, u32, u32]),
    "gg_server_create": (i, [vp, vp, P(T.ServerConfig), P(vp)]),
    "gg_server_destroy": (None, [vp]),
    "gg_server_submit": (i, [vp, P(T.Request), P(u64)]),
    "gg_server_inject_fault": (i, [vp, i]),
    "gg_server_poll": (i, [vp, u64, P(i)]),
    "gg_server_cancel": (i, [vp, u64]),
    "gg_server_wait": (i, [vp, u64, C.c_double, P(T.RequestResult)]),
    "gg_server_totals": (i, [vp, i, P(u64), P(u64), P(u64), P(C.c_double), P(C.c_double)]),
    "gg_measure_fp32_peak": (i, [vp, P(C.c_double)]),
    "gg_measure_atomic_peak": (i, [vp, u32, P(C.c_double)]),
    "gg_measure_shared_atomic_peak": (i, [vp, P(C.c_double)]),
}


def lib() -> C.CDLL:
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(there is no CPU fallback)."
        )
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def extra_signature(name: str, res, args) -> None:
    """Register the argument types of an entry point defined elsewhere."""
    fn = getattr(lib(), name)
    fn.restype = res
    fn.argtypes = args
    SIGNATURES[name] = (res, args)


def check(status: int) -> None:
    if status != 0:
        sentence = lib().gg_last_error().decode("utf-8", "replace")
        raise GargantuaError(status, sentence)


def ptr(array) -> int:
    """Raw data pointer of a numpy array (None passes NULL)."""
    if array is None:
        return None
    return array.ctypes.data
