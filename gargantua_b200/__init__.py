"""gargantua-b200: gargantua's per-frame compute (particle sim, cloud-in-cell
splat and resolve, null-geodesic march, probes, bake/walk, tone curve) as
sm_100a kernels behind the C ABI in include/gargantua.h.

The kernels live in libgargantua_b200.so, built in-tree by
__graft_entry__.build(); this package is the Python view of that ABI.
"""
from . import types
from ._lib import GargantuaError, lib
from .host import (Bake, Context, Launch, OrbitCamera, Particles, RequestSpec, Sequence, Server, Settings, Targets, Volume,
                   aimed, as_float32_launch, camera_grid, march, march_stats, pinned_array, splat_uniforms, uniforms,
                   write_png)

__all__ = [
    "types", "GargantuaError", "lib", "Bake", "Context", "Launch", "OrbitCamera", "Particles", "Settings",
    "Targets", "Volume", "RequestSpec", "Sequence", "Server", "march_stats", "aimed", "as_float32_launch", "camera_grid", "march", "pinned_array", "splat_uniforms",
    "uniforms", "write_png",
]
