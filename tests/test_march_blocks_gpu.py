"""The image kernels' block shape (gg_context_set_march_block) changes how
pixels are grouped into blocks, never a pixel's value; the autotuner keeps a
measured shape. Refusals for shapes that are not whole warps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    import gargantua_b200 as g

    ctx = g.Context()
    ps = g.Particles(ctx, 100_000, seed=6)
    ps.advance(50, seed_first=True)
    vol = g.Volume(ctx, 64)
    vol.splat(ps, exact=True)
    yield ctx, vol
    ctx.close()


@pytest.mark.parametrize("spin", [0.0, 0.9])
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_block_shape_does_not_change_pixels(scene, spin, precision):
    import gargantua_b200 as g

    ctx, vol = scene
    cam = g.OrbitCamera(0.7, 0.3, 50.0)
    u = g.uniforms(cam, 250, 130, g.Settings.still(), 1e-5, True, 3, spin=spin)  # ragged edges for every shape
    if spin == 0.0:
        ctx.enable_tables(u, float(np.float32(cam.distance)))
    t = g.Targets(ctx, 250, 130)
    ref = None
    for bw, bh in ((8, 8), (32, 1), (16, 16), (32, 8), (8, 4)):
        ctx.set_march_block(bw, bh)
        counters = g.march(ctx, vol, u, t, precision)
        color, debug, depth = t.read()
        got = (color.view(np.uint16).copy(), debug.view(np.uint16).copy(), depth.view(np.uint32).copy(),
               counters.rays, counters.captured, counters.exhausted)
        if ref is None:
            ref = got
        else:
            for a, b in zip(got[:3], ref[:3]):
                assert np.array_equal(a, b), (bw, bh)
            assert got[3:] == ref[3:]
    ctx.set_march_block(8, 8)
    t.close()


def test_block_shape_refusals_and_autotune(scene):
    import gargantua_b200 as g
    from gargantua_b200 import autotune

    ctx, vol = scene
    for bad in ((0, 8), (5, 5), (16, 32), (512, 1)):
        with pytest.raises(g.GargantuaError):
            ctx.set_march_block(*bad)
    cam = g.OrbitCamera()
    u = g.uniforms(cam, 320, 180, g.Settings.interactive(), 1e-4, True, 1, spin=0.9)
    tuned = autotune.tune_march_block(ctx, vol, u, blocks=((8, 8), (32, 4)), repeats=1)
    assert tuned["block"] in ([8, 8], [32, 4]) and tuned["ms"] > 0.0 and len(tuned["trials"]) == 2
    ctx.set_march_block(8, 8)
