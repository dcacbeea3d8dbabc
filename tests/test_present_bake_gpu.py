"""Parity of the present and bake passes and of the device sweep tables.

Tone curve (present.metal:22-35) and drift heat map (present.metal:40-46):
gg_tonemap against the FP32 replica (oracle/replica.c, every operation
rounded on its own like the kernel's --fmad=false build); the only
difference allowed is powf's last bit in the sRGB encode, so every channel
is within one code value and nearly all are equal.

Bake (bake.metal:17-92) and walk (:94-144): rays launched at the camera
(no sphere jump) against the FP64 bake of the oracle, sample by sample; the
full 960x540 bake with the jump keeps the layout's invariants and truncates
as many rays as the reference's own bench reports; the walk of a bake
renders the image the march renders.

Sweep tables (Deflection.swift:95-106): the FP64 device build against the
oracle's tables, entry by entry.
"""
import numpy as np
import pytest

import oracle_ffi as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import gargantua_b200 as g

    c = g.Context()
    yield c
    c.close()


@pytest.fixture(scope="module")
def disk(ctx):
    """The default preset's disk (1M particles, 128^3) settled 600 substeps."""
    import gargantua_b200 as g

    ps = g.Particles(ctx, 1_000_000, seed=1)
    ps.advance(300, seed_first=True)
    vol = g.Volume(ctx, 128)
    vol.splat(ps, exact=True)
    yield vol
    vol.close()
    ps.close()


def _random_half4(rng, n, low, high):
    return rng.uniform(low, high, (n, 4)).astype(np.float16)


@pytest.mark.parametrize("exposure", [0.35, 1.0, 2.7])
def test_tonemap_matches_the_fp32_replica(ctx, exposure):
    import gargantua_b200 as g

    rng = np.random.default_rng(int(exposure * 100))
    w, h = 257, 129  # not a multiple of the kernel's 256-thread block
    color = _random_half4(rng, w * h, -0.2, 6.0)
    color[::7] = _random_half4(rng, len(color[::7]), 0.0, 0.09)  # the toe (x < 0.08)
    color[::11] = 0.0
    color[::13] = _random_half4(rng, len(color[::13]), 20.0, 6e4)  # far over the shoulder
    t = g.Targets(ctx, w, h)
    t.write(color=color, debug=np.zeros_like(color))
    got = t.tonemap(exposure=exposure).reshape(-1, 4)
    want = O.present32(color, exposure)
    diff = np.abs(got.astype(np.int32) - want.astype(np.int32))
    assert diff.max() <= 1, diff.max()
    assert (diff == 0).mean() > 0.999
    assert (got[:, 3] == 255).all()
    t.close()


def test_drift_heat_map_matches_the_fp32_replica(ctx):
    import gargantua_b200 as g

    rng = np.random.default_rng(5)
    w, h = 200, 90
    n = w * h
    debug = np.zeros((n, 4), np.float16)
    debug[:, 0] = rng.uniform(0.0, 3e-4, n)      # drift, up to 3x the budget
    debug[::5, 0] = 0.0
    debug[:, 1] = rng.integers(0, 600, n)          # steps
    debug[:, 2] = rng.integers(0, 2, n)            # escaped (1) / captured (0)
    debug[:, 3] = 1.0
    t = g.Targets(ctx, w, h)
    t.write(color=np.zeros_like(debug), debug=debug)
    for budget in (1e-4, 1e-5):
        got = t.tonemap(debug_view=True, drift_budget=budget).reshape(-1, 4)
        want = O.present32(debug, debug_view=True, drift_budget=budget)
        diff = np.abs(got.astype(np.int32) - want.astype(np.int32))
        assert diff.max() <= 1
        assert (diff == 0).mean() > 0.999
    t.close()


def test_tonemap_of_a_marched_image(ctx, disk):
    """A real frame: the march's half4 colour through gg_tonemap and the
    replica, and the march's own debug target through the heat map."""
    import gargantua_b200 as g

    cam = g.OrbitCamera()
    u = g.uniforms(cam, 320, 180, g.Settings.interactive(), 1e-4, True, 1)
    ctx.enable_tables(u, float(np.float32(cam.distance)))
    t = g.Targets(ctx, 320, 180)
    g.march(ctx, disk, u, t)
    color, debug, _ = t.read()
    for view, src in ((False, color), (True, debug)):
        got = t.tonemap(exposure=1.4, debug_view=view).reshape(-1, 4)
        want = O.present32(src, 1.4, debug_view=view)
        diff = np.abs(got.astype(np.int32) - want.astype(np.int32))
        assert diff.max() <= 1
        assert (diff == 0).mean() > 0.999
    t.close()


def _bake_launches(u, width, height):
    """The bake kernel's rays (bake.metal:30-33): pixel centres, no jitter,
    direction formed in FP32 from the uniforms' camera basis."""
    f32 = np.float32
    pos = np.array([u.cameraPosition.x, u.cameraPosition.y, u.cameraPosition.z], f32)
    right = np.array([u.cameraRight.x, u.cameraRight.y, u.cameraRight.z], f32)
    up = np.array([u.cameraUp.x, u.cameraUp.y, u.cameraUp.z], f32)
    fwd = np.array([u.cameraForward.x, u.cameraForward.y, u.cameraForward.z], f32)
    px, py = np.meshgrid(np.arange(width, dtype=f32), np.arange(height, dtype=f32))
    sx, sy = px.ravel() + f32(0.5), py.ravel() + f32(0.5)
    nx = (f32(2.0) * sx / f32(width) - f32(1.0)) * f32(u.tanHalfFov.x)
    ny = (f32(1.0) - f32(2.0) * sy / f32(height)) * f32(u.tanHalfFov.y)
    d = fwd[None, :] + nx[:, None] * right[None, :] + ny[:, None] * up[None, :]
    d = d.astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([np.broadcast_to(pos.astype(np.float64), d.shape), d], axis=1)


def _half2(words):
    return words.astype(np.uint32).view(np.float16).reshape(-1, 2).astype(np.float64)


def test_bake_follows_the_fp64_bake(ctx):
    """Rays launched at the camera (sphere jump off), still step policy:
    sample counts, stored points and paths, the falls-in flag, the final
    direction and depth against the FP64 bake."""
    import gargantua_b200 as g

    w, h = 96, 54
    cam = g.OrbitCamera()
    spacing = g.Bake.spacing(128)
    u = g.uniforms(cam, w, h, g.Settings.still(), 1e-5, True, 1, bake_spacing=spacing)
    assert u.sphereRadius == 0.0
    b = g.Bake(ctx, w, h)
    b.bake_full(u)
    samples, headers = b.read()
    overflow = b.overflow()
    probes = _bake_launches(u, w, h)
    o_samples, o_counts, o_over, o_falls, o_dd = O.bake_batch(probes, O.still(), float(spacing))
    counts = headers[:, 0].astype(np.int64)
    # Counts: the FP32 path crosses the slab and spacing thresholds where the
    # FP64 path does, up to a point now and then.
    assert (counts == o_counts).mean() > 0.97
    assert np.abs(counts - o_counts).max() <= 3
    assert overflow == int(o_over.sum()) or abs(overflow - int(o_over.sum())) <= max(2, 0.02 * o_over.sum())
    assert (headers[:, 1] == o_falls).mean() > 0.995
    # Stored points of rays whose counts agree: position within the half
    # precision of the store plus FP32 path error, path within 1 %.
    same = counts == o_counts
    k = np.arange(96)[None, :] < counts[:, None]
    mask = same[:, None] & k
    dev = samples.astype(np.float64)[mask]
    ref = o_samples[mask]
    pos_err = np.linalg.norm(dev[:, :3] - ref[:, :3], axis=1)
    assert (pos_err < 0.02 + 2e-3 * np.linalg.norm(ref[:, :3], axis=1)).mean() > 0.99
    path_err = np.abs(dev[:, 3] - ref[:, 3]) / ref[:, 3]
    assert (path_err < 1e-2).mean() > 0.99
    assert (dev[:, 3] >= np.float16(spacing) * (1 - 2 ** -10)).all()  # at least the spacing, after half rounding
    assert (np.abs(dev[:, 2]) < 6.0 + 1e-2).all() and (np.abs(dev[:, :2]) < 30.0 + 2e-2).all()
    # Final direction and depth (half precision) of rays that do not fall in.
    xy, zd = _half2(headers[:, 2]), _half2(headers[:, 3])
    d = np.concatenate([xy, zd[:, :1]], axis=1)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out = (headers[:, 1] == 0) & (o_falls == 0)
    cosang = np.clip((d[out] * o_dd[out, :3]).sum(axis=1), -1, 1)
    assert (np.arccos(cosang) < 5e-3).mean() > 0.99
    assert (np.abs(zd[:, 1] - o_dd[:, 3]) < 2e-3 + 1e-2 * o_dd[:, 3]).mean() > 0.99
    b.close()


def test_bake_with_the_jump_keeps_its_layout_and_truncates_like_the_reference(ctx):
    """The reference's bench bake (Bench.swift:156-171, 193-206): the default
    camera at 960x540, the still geodesic settings, spacing for 128^3, sweep
    tables on. Every stored point is in the slab, every path at least the
    spacing, counts within the capacity, sky-only rays empty; the truncated
    rays agree with the reference's bench report, 35,975
    (bench/results/2026-08-23-192754.json:2-4), within 3 %."""
    import gargantua_b200 as g

    w, h = 960, 540
    cam = g.OrbitCamera()
    spacing = g.Bake.spacing(128)
    u = g.uniforms(cam, w, h, g.Settings.interactive(), 1e-4, True, 1, bake_spacing=spacing)
    ctx.enable_tables(u, float(np.float32(cam.distance)))
    u.geodesic = g.Settings.still().geodesic()
    b = g.Bake(ctx, w, h)
    b.bake_full(u)
    overflow = b.overflow()
    samples, headers = b.read()
    counts = headers[:, 0].astype(np.int64)
    assert counts.max() <= 96
    assert abs(overflow - 35975) / 35975 < 0.03, overflow
    assert (counts == 96).sum() >= overflow  # a truncated ray filled its budget
    live = np.arange(96)[None, :] < counts[:, None]
    pts = samples.astype(np.float64)[live]
    assert (np.abs(pts[:, 2]) < 6.0 + 1e-2).all() and (np.abs(pts[:, :2]) < 30.0 + 2e-2).all()
    assert (pts[:, 3] >= np.float16(spacing) * (1 - 2 ** -10)).all()
    zd = _half2(headers[:, 3])
    assert ((zd[:, 1] >= 0.0) & (zd[:, 1] <= 1.0)).all()
    assert (counts == 0).any() and (counts > 0).mean() > 0.1
    b.close()


def test_walk_renders_the_march_image(ctx, disk):
    """The bake strategy's frame renders the march's: the same camera, the
    still step policy, the same volume. The walk is a coarser quadrature of
    the same emission integral -- stored points at least half a voxel apart,
    each weighted by the path since the previous one, the redshift taken
    along the chord between points (from the camera for the first) -- where
    the march gathers at every RK4 step with the photon's own direction. So
    the image's light agrees to 1 % (the jump golden's bar for two
    quadratures of one image, goldens/jump.json) and most pixels closely,
    while pixels on sharp emission edges differ more (measured on a B200:
    median 0, 95th percentile 17.5 %, 99th 45 % relative)."""
    import gargantua_b200 as g

    w, h = 480, 270
    cam = g.OrbitCamera()
    spacing = g.Bake.spacing(128)
    u = g.uniforms(cam, w, h, g.Settings.still(), 1e-5, True, 1, bake_spacing=spacing)
    ctx.enable_tables(u, float(np.float32(cam.distance)))
    b = g.Bake(ctx, w, h)
    b.bake_full(u)
    walked = g.Targets(ctx, w, h)
    b.walk(disk, u, walked)
    marched = g.Targets(ctx, w, h)
    g.march(ctx, disk, u, marched)
    wc = walked.read()[0].astype(np.float64)[:, :3]
    mc = marched.read()[0].astype(np.float64)[:, :3]
    lw, lm = O.luminance(wc), O.luminance(mc)
    total = abs(lw.sum() - lm.sum()) / lm.sum()
    assert total < 0.01, total
    rel = np.abs(lw - lm) / np.maximum(lm, 1e-3 * lm.max())
    q50, q95, q99 = np.quantile(rel, [0.5, 0.95, 0.99])
    assert q50 < 0.01 and q95 < 0.25 and q99 < 0.6, (q50, q95, q99)
    walked.close()
    marched.close()
    b.close()


@pytest.mark.parametrize("camera_radius", [52.0, 88.5])
def test_device_sweep_tables_match_the_oracle(ctx, camera_radius):
    """Sphere, camera and sky tables built in FP64 on the device (one CTA per
    entry, tree-ordered sums) against the oracle's serial FP64 tables
    (Deflection.swift:95-106), each rounded to FP32: at most one ulp apart."""
    import gargantua_b200 as g

    u = g.uniforms(g.OrbitCamera(distance=camera_radius), 8, 8, g.Settings.interactive(), 1e-4, True, 1)
    ctx.enable_tables(u, camera_radius)
    sphere, camera, sky = ctx.tables()
    want = {
        "sphere": O.sweep_table(30.0, 1024, 2048),
        "camera": O.sweep_table(camera_radius, 1024, 256),
        "sky": O.sky_table(camera_radius, 29.0, 1024, 256),
    }
    for name, got in (("sphere", sphere), ("camera", camera), ("sky", sky)):
        ref = want[name].astype(np.float32)
        ulps = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
        assert ulps.max() <= 1, (name, ulps.max())
