"""gg_march_compensated_noalloc: the compensated march for callers that must
not allocate device memory while they render (hosts that hand the device's
memory to their own pool up front, frame loops that cannot absorb a
cudaMalloc/cudaFree stall or failure mid-frame, plugins inside a program that
owns the memory budget).

Called through the C ABI, its pixels must match the regular compensated
march (gg_march with GG_PRECISION_COMPENSATED) on two calls in a row, it must
leave the context's device memory untouched, and it must refuse targets
larger than its fixed scratch. This file is collected last so a run that
stops at the first failure has run every other test first; it also passes
alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOALLOC_MAX_PIXELS = 2097152


@pytest.fixture(scope="module")
def scene():
    import gargantua_b200 as g

    ctx = g.Context()
    ps = g.Particles(ctx, 200_000, seed=3)
    ps.advance(100, seed_first=True)
    vol = g.Volume(ctx, 64)
    vol.splat(ps, exact=True)
    yield ctx, vol
    ctx.close()


def noalloc(ctx, vol, u, targets):
    from gargantua_b200 import _lib, types as T

    counters = T.MarchCounters()
    status = _lib.lib().gg_march_compensated_noalloc(ctx.handle, vol.handle, C.byref(u), targets.handle,
                                                      C.byref(counters))
    return status, counters


@pytest.mark.parametrize("spin,step_cap", [(0.0, 4096), (0.9, 4096), (0.0, 256)])
def test_noalloc_matches_gg_march_on_two_calls(scene, spin, step_cap):
    import gargantua_b200 as g

    ctx, vol = scene
    cam = g.OrbitCamera(0.9, 0.25, 48.0)
    settings = g.Settings.still() if step_cap == 4096 else g.Settings.interactive()
    u = g.uniforms(cam, 320, 180, settings, 1e-5 if step_cap == 4096 else 1e-4, True, 7, spin=spin)
    if spin == 0.0:
        ctx.enable_tables(u, float(np.float32(cam.distance)))
    ref_t = g.Targets(ctx, 320, 180)
    ref_counters = g.march(ctx, vol, u, ref_t, g.types.PRECISION_COMPENSATED)
    ref_color, ref_debug, ref_depth = ref_t.read()
    t = g.Targets(ctx, 320, 180)
    used_before = ctx.memory()[1]
    for call in range(2):
        status, counters = noalloc(ctx, vol, u, t)
        assert status == 0, g.lib().gg_last_error()
        color, debug, depth = t.read()
        # Same kernels, same inputs: identical pixels (the tests' image
        # tolerance, 1e-2 relative luminance, is met with room to spare).
        assert np.array_equal(color.view(np.uint16), ref_color.view(np.uint16)), call
        assert np.array_equal(debug.view(np.uint16), ref_debug.view(np.uint16)), call
        assert np.array_equal(depth.view(np.uint32), ref_depth.view(np.uint32)), call
        assert counters.rays == ref_counters.rays == 320 * 180
        assert counters.captured == ref_counters.captured
        assert counters.exhausted == ref_counters.exhausted
    assert ctx.memory()[1] == used_before  # nothing allocated against the budget
    t.close()
    ref_t.close()


def test_noalloc_reintegrates_the_same_rays_and_allocates_nothing(scene):
    """A Kerr still close to the hole (a = 0.9, camera at r = 9, 4096 steps,
    every flagged ray re-integrated) puts rays on the FP64 list, so the fixed
    array is written and read: the FP64 ray count and the pixels must equal
    gg_march's on two calls in a row, and the device's free memory must not
    move across the calls after the first (which loads the array)."""
    import torch

    import gargantua_b200 as g

    ctx, vol = scene
    cam = g.OrbitCamera(0.4, 0.3, 9.0)
    st = g.Settings.still()
    u = g.uniforms(cam, 256, 144, st, 1e-5, True, 5, spin=0.9)
    ctx.set_fp64_policy(g.types.FP64_ALL_FLAGGED)
    try:
        ref_t = g.Targets(ctx, 256, 144)
        g.march(ctx, vol, u, ref_t, g.types.PRECISION_COMPENSATED)
        ref_fp64 = g.march_stats(ctx)[2]
        ref_color, _, _ = ref_t.read()
        assert ref_fp64 > 0
        t = g.Targets(ctx, 256, 144)
        free = []
        for call in range(3):
            status, _ = noalloc(ctx, vol, u, t)
            assert status == 0, g.lib().gg_last_error()
            ctx.synchronize()
            free.append(torch.cuda.mem_get_info(0)[0])
            assert g.march_stats(ctx)[2] == ref_fp64, call
            color, _, _ = t.read()
            assert np.array_equal(color.view(np.uint16), ref_color.view(np.uint16)), call
        assert free[1] == free[0] and free[2] == free[0], free
        t.close()
        ref_t.close()
    finally:
        ctx.set_fp64_policy(g.types.FP64_ESCAPING)


def test_noalloc_refuses_targets_beyond_its_scratch(scene):
    import gargantua_b200 as g

    ctx, vol = scene
    cam = g.OrbitCamera()
    w, h = 2048, NOALLOC_MAX_PIXELS // 2048 + 1
    u = g.uniforms(cam, w, h, g.Settings.interactive(), 1e-4, True, 1, spin=0.9)
    big = g.Targets(ctx, w, h)
    status, _ = noalloc(ctx, vol, u, big)
    assert status == 1  # GG_ERR_INVALID_ARGUMENT
    assert str(NOALLOC_MAX_PIXELS) in g.lib().gg_last_error().decode()
    big.close()
