"""The served path (gg_server_*): continuous batching of still requests
against the plain per-request baseline, result identity alone vs in a mix,
admission by device footprint, and drift budgets."""
import math

import numpy as np
import pytest

import oracle_ffi as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def world():
    import gargantua_b200 as g

    ctx = g.Context()
    ps = g.Particles(ctx, 1_000_000, seed=1)
    ps.advance(300, seed_first=True)
    vol = g.Volume(ctx, 128)
    vol.splat(ps, exact=True)
    yield {"ctx": ctx, "vol": vol, "ps": ps}
    ctx.close()


def luminance(pix):
    return O.luminance(pix[:, :3].astype(np.float64))


def mix_specs():
    import gargantua_b200 as g

    return [
        g.RequestSpec(320, 180, 4096, 0.0, azimuth=0.6, elevation=0.32, distance=52.0),
        g.RequestSpec(640, 360, 256, 0.9, azimuth=1.1, elevation=0.5, distance=70.0),
        g.RequestSpec(480, 270, 4096, 0.5, azimuth=2.0, elevation=1.2, distance=45.0),
        g.RequestSpec(320, 180, 256, 0.0, azimuth=-0.4, elevation=0.2, distance=110.0),
        g.RequestSpec(160, 90, 4096, 0.9, azimuth=0.2, elevation=0.1, distance=40.0),
        # The ends of the spin range (Options.swift:119-124): near-extremal,
        # and barely spinning (the Kerr path, not the Schwarzschild one).
        g.RequestSpec(240, 135, 4096, 0.998, azimuth=0.9, elevation=0.3, distance=50.0),
        g.RequestSpec(240, 135, 256, 0.02, azimuth=3.0, elevation=0.7, distance=60.0),
    ]


def run(server, specs, debug=False):
    tickets = [server.submit(s, debug=debug) for s in specs]
    return [server.wait(t) for t in tickets]


@pytest.mark.parametrize("mode", ["SERVE_SERIAL_PLAIN", "SERVE_SERIAL_PLAIN_AS_WRITTEN"])
def test_served_matches_plain_per_request(world, mode):
    import gargantua_b200 as g

    specs = mix_specs()
    batched = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED)
    plain = g.Server(world["ctx"], world["vol"], getattr(g.types, mode))
    a = run(batched, specs, debug=True)
    b = run(plain, specs, debug=True)
    for spec, (pa, da, ra), (pb, db, rb) in zip(specs, a, b):
        n = spec.width * spec.height
        assert ra.counters.rays == n and rb.counters.rays == n
        la, lb = luminance(pa), luminance(pb)
        diff = np.abs(la - lb).sum() / max(lb.sum(), 1e-30)
        assert diff < 1e-2, (spec, diff)
        # Pixel by pixel: 99 % within 1e-2 relative (luminance floor at 1e-3
        # of the image's brightest pixel, below which pixels are sky black).
        rel = np.abs(la - lb) / np.maximum(lb, 1e-3 * lb.max())
        assert np.mean(rel < 1e-2) > 0.99, (spec, np.mean(rel < 1e-2))
        # Same algorithm, same step counts up to rays whose fate flips at a
        # boundary (compensated vs plain rounding).
        assert abs(int(ra.ray_steps) - int(rb.ray_steps)) <= 0.01 * rb.ray_steps + 64, (ra.ray_steps, rb.ray_steps)
        # Rounding differences can move a step across a step-policy switch
        # (coarse vs fine near the slab) or an exit test, shifting a ray's
        # count; the bulk of rays agree closely.
        dsteps = np.abs(da[:, 1].astype(np.float32) - db[:, 1].astype(np.float32))
        assert np.median(dsteps) <= 1.0, np.median(dsteps)
        assert np.mean(dsteps <= 4.0) > 0.95, np.mean(dsteps <= 4.0)
    batched.close()
    plain.close()


def test_each_result_is_the_same_alone_and_in_the_mix(world):
    """A request's pixels do not depend on what else shares its waves."""
    import gargantua_b200 as g

    specs = mix_specs()
    server = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED, chunk_rays=128)
    mixed = run(server, specs, debug=True)
    for k, spec in enumerate(specs):
        alone = run(server, [spec], debug=True)[0]
        assert np.array_equal(alone[0].view(np.uint16), mixed[k][0].view(np.uint16)), spec
        assert np.array_equal(alone[1].view(np.uint16), mixed[k][1].view(np.uint16)), spec
        assert alone[2].ray_steps == mixed[k][2].ray_steps
    server.close()


def test_page_locked_outputs_match_pageable_ones(world):
    """gg_host_alloc / gg_host_free: a request served into page-locked memory
    (Server.submit's default) gives the pixels a pageable array gets, a view
    outlives its array, and blocks go back to the context for reuse as
    their arrays go."""
    import gc

    import gargantua_b200 as g

    spec = g.RequestSpec(320, 180, 256, 0.5, azimuth=0.7, elevation=0.3, distance=55.0)
    server = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED)
    pageable = np.zeros((320 * 180, 4), np.float16)
    a = server.wait(server.submit(spec, pageable))[0]
    b = server.wait(server.submit(spec))[0]
    assert np.array_equal(a.view(np.uint16), b.view(np.uint16))
    copy = b[1000:1010].copy()
    view = b[1000:1010]
    del b
    gc.collect()
    assert np.array_equal(copy.view(np.uint16), view.view(np.uint16))  # the view still reads the block
    server.close()
    addresses = set()
    for _ in range(64):  # one 1 MB block, handed back and reused
        block = g.pinned_array(world["ctx"], (1 << 20,), np.uint8)
        block[:] = 7
        assert int(block.sum()) == 7 << 20
        addresses.add(block.__array_interface__["data"][0])
        del block
    assert len(addresses) == 1
    import ctypes as C

    from gargantua_b200._lib import check

    with pytest.raises(g.GargantuaError):  # a zero size is refused with a sentence
        check(g.lib().gg_host_alloc(world["ctx"].handle, 0, C.byref(C.c_void_p())))


def test_overlapping_arrivals_are_admitted_as_memory_frees(world):
    """A server whose memory holds about two requests still completes a
    stream of eight, admitting each as an earlier one releases its targets."""
    import gargantua_b200 as g

    spec = g.RequestSpec(320, 180, 4096, 0.0)
    one = 320 * 180 * 8 + 128 + 8192
    server = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED, memory_bytes=2 * one + 1000)
    results = run(server, [spec] * 8)
    first = results[0][0]
    for pix, _, res in results:
        assert res.counters.rays == 320 * 180
        assert np.array_equal(pix.view(np.uint16), first.view(np.uint16))
    admitted = sorted(r[2].admitted for r in results)
    submitted = max(r[2].submitted for r in results)
    assert admitted[-1] > submitted  # later requests waited for memory
    with pytest.raises(g.GargantuaError) as e:
        server.submit(g.RequestSpec(1920, 1080, 256, 0.0))
    assert e.value.status == 3
    server.close()


def test_still_drift_budget_and_fp64_reintegration(world):
    """4096-step Schwarzschild rays stay under the 1e-5 still budget; Kerr
    rays over budget after entering r < 4 come back from FP64."""
    import gargantua_b200 as g

    server = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED)
    (pix, dbg, res), = run(server, [g.RequestSpec(640, 360, 4096, 0.0)], debug=True)
    drift = dbg[:, 0].astype(np.float32)
    assert res.counters.rays == 640 * 360
    assert float(drift.max()) < 1e-5, float(drift.max())
    (kp, kd, kres), = run(server, [g.RequestSpec(320, 180, 4096, 0.9)], debug=True)
    assert kres.counters.rays == 320 * 180
    assert np.isfinite(kp.astype(np.float32)).all()
    # Kerr drift (Carter constant and null residual, the maximum over the
    # ray's steps, march.metal:160-163) at the FP64 integrator's floor: the
    # share of rays over the 1e-5 still budget is within 3 points of the
    # FP64 oracle's for rays of the same camera (a 32x18 grid), and the
    # median ray drifts far less than the budget.
    kdrift = kd[:, 0].astype(np.float64)
    cam = g.OrbitCamera()
    launches = [g.as_float32_launch(l) for l in g.camera_grid(cam, 32, 18, 320 / 180)]
    probes = np.array([np.concatenate([l.origin, l.direction]) for l in launches])
    ref = O.kerr_integrate_batch(0.9, probes, O.KerrSettings(0.02, 0.005, 0.5, 0.05, 62.0, 4096))
    served_over, oracle_over = float(np.mean(kdrift > 1e-5)), float(np.mean(ref[:, 6] > 1e-5))
    assert served_over <= oracle_over + 0.03, (served_over, oracle_over)
    assert float(np.median(kdrift)) < 1e-6, float(np.median(kdrift))
    server.close()


def test_invalid_requests_are_refused(world):
    import gargantua_b200 as g

    server = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED)
    for bad in (g.RequestSpec(0, 10), g.RequestSpec(10, 10, step_cap=5000), g.RequestSpec(10, 10, spin=1.0),
                g.RequestSpec(10, 10, distance=20.0)):
        with pytest.raises(g.GargantuaError) as e:
            server.submit(bad)
        assert e.value.status == 1
    totals = server.totals()
    assert totals["requests"] == 0
    server.close()


def test_server_autotune_picks_a_measured_candidate(world):
    import gargantua_b200 as g
    from gargantua_b200 import autotune

    specs = mix_specs()[:4]
    tuned = autotune.tune_server(world["ctx"], world["vol"], specs, chunks=(32, 64), waves=(1 << 20,),
                                 in_flight=(2,), cadences=((8, 8), (4, 4)),
                                 schedules=(g.types.SCHEDULE_LANE_REFILL,), repeats=1)
    assert tuned["chunk_rays"] in (32, 64) and tuned["rate"] > 0.0
    assert (tuned["steps_per_round"], tuned["refill_idle"]) in ((8, 8), (4, 4))
    assert len(tuned["trials"]) == 4  # two chunk sizes, then two cadences
    shape = {k: tuned[k] for k in ("chunk_rays", "wave_rays", "max_waves_in_flight", "steps_per_round", "refill_idle",
                                   "schedule")}
    server = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED, **shape)
    pixels, _, res = server.wait(server.submit(specs[0]))
    assert res.status == 0 and res.counters.rays == specs[0].width * specs[0].height
    server.close()


def test_sequence_frames_march_their_own_advancing_volume(world):
    """Sequence frames served in a mix with a still: each frame equals the
    plain march of the same sim state within the served-vs-plain bar, and
    the frames change as the disk advances."""
    import gargantua_b200 as g

    ctx = world["ctx"]
    server = g.Server(ctx, world["vol"], g.types.SERVE_BATCHED)
    seq = g.Sequence(server, ctx, 50_000, 48, frames=3, width=320, height=180, spin=0.0, seed=4,
                     settle_dispatches=50)
    # A replica of the sequence's state, marched per frame with gg_march.
    ps = g.Particles(ctx, 50_000, seed=4)
    ps.advance(50, seed_first=True)
    vol = g.Volume(ctx, 48)
    t = g.Targets(ctx, 320, 180)
    other = server.submit(g.RequestSpec(640, 360, 4096, 0.9))
    lums = []
    for k in range(3):
        pixels, res = seq.frame()
        assert res.status == 0 and res.counters.rays == 320 * 180
        ps.step(1)
        vol.splat(ps, exact=False)
        u = g.uniforms(seq.camera, 320, 180, g.Settings.interactive(), 1e-4, True, 4)
        ctx.enable_tables(u, float(np.float32(seq.camera.distance)))
        g.march(ctx, vol, u, t)
        ref, _, _ = t.read()
        la, lb = luminance(pixels), luminance(ref)
        assert np.abs(la - lb).sum() / max(lb.sum(), 1e-30) < 1e-2, k
        lums.append(la)
    assert not np.array_equal(lums[0], lums[2])  # the disk moved
    server.wait(other)
    t.close()
    vol.close()
    ps.close()
    seq.close()
    server.close()


def test_fp64_policy_skips_captured_rays_by_default(world):
    """GG_FP64_ESCAPING re-integrates fewer rays than GG_FP64_ALL_FLAGGED on
    a Kerr still whose flagged rays are mostly captured; the images agree."""
    import gargantua_b200 as g

    spec = g.RequestSpec(480, 270, 4096, 0.9, azimuth=1.0, elevation=0.4, distance=52.0)
    counts, lum = {}, {}
    for policy in (g.types.FP64_ESCAPING, g.types.FP64_ALL_FLAGGED):
        server = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED, fp64_policy=policy)
        (pix, _, res), = run(server, [spec])
        counts[policy] = int(res.fp64_rays)
        lum[policy] = luminance(pix)
        server.close()
    assert counts[g.types.FP64_ALL_FLAGGED] > counts[g.types.FP64_ESCAPING]
    a, b = lum[g.types.FP64_ESCAPING], lum[g.types.FP64_ALL_FLAGGED]
    assert np.abs(a - b).sum() / max(b.sum(), 1e-30) < 1e-3


def test_schedules_give_the_same_pixels(world):
    """The chunk and lane-refill schedules march the same rays with the same
    step arithmetic: equal ray-step and FP64 counts for every request of a
    mix, and the same pixels up to the rounding of the compiler's own
    contraction choices in each kernel's Kerr gather (measured: at most 33
    pixels of a request, by at most 2.5e-4, luminance within 3e-7)."""
    import gargantua_b200 as g

    specs = mix_specs()
    out = {}
    for sch in (g.types.SCHEDULE_CHUNKS, g.types.SCHEDULE_LANE_REFILL):
        server = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED, schedule=sch)
        out[sch] = run(server, specs)
        server.close()
    for spec, (pa, _, ra), (pb, _, rb) in zip(specs, out[g.types.SCHEDULE_CHUNKS], out[g.types.SCHEDULE_LANE_REFILL]):
        assert ra.ray_steps == rb.ray_steps and ra.counters.rays == rb.counters.rays
        assert ra.fp64_rays == rb.fp64_rays
        differ = np.any(pa.view(np.uint16) != pb.view(np.uint16), axis=1)
        if spec.spin == 0.0:
            assert not differ.any()
        assert differ.mean() < 5e-3
        assert np.abs(pa.astype(np.float64) - pb.astype(np.float64)).max() < 1e-3
        la, lb = luminance(pa), luminance(pb)
        assert np.abs(la - lb).sum() / max(lb.sum(), 1e-30) < 1e-5


def test_a_sequence_resumes_from_its_snapshot(world):
    """Checkpoint and resume of a served sequence: a second sequence
    restored from the first one's snapshot after two frames renders the
    first one's frames three and four bit for bit (the particle records are
    checked against their FNV-1a checksum on restore; every later random
    draw is keyed on index, event and seed)."""
    import gargantua_b200 as g

    ctx = world["ctx"]
    server = g.Server(ctx, world["vol"], g.types.SERVE_BATCHED)
    first = g.Sequence(server, ctx, 40_000, 48, frames=4, width=320, height=180, seed=6, settle_dispatches=20)
    frames = [first.frame()[0] for _ in range(2)]
    snap = first.snapshot()
    frames += [first.frame()[0] for _ in range(2)]
    second = g.Sequence(server, ctx, 40_000, 48, frames=2, width=320, height=180, seed=6, settle_dispatches=1)
    second.restore(snap)
    for k in (2, 3):
        pixels, res = second.frame()
        assert res.status == 0
        assert np.array_equal(pixels.view(np.uint16), frames[k].view(np.uint16)), k
    assert first.particles.checksum() == second.particles.checksum()
    bad = dict(snap, checksum=snap["checksum"] ^ 1)
    with pytest.raises(ValueError):
        second.restore(bad)
    first.close()
    second.close()
    server.close()


def test_bake_requests_are_served_beside_marches(world):
    """GG_REQUEST_BAKE (the bake strategy as a served request): the walk of
    its bake renders the march's image of the same camera (image light
    within 1 %, the jump golden's bar for two quadratures of one image), it
    reports its ray steps, and its pixels are the same alone, in a mix with
    marches, and through the one-at-a-time baseline server."""
    import gargantua_b200 as g

    bake = g.RequestSpec(480, 270, 4096, 0.0, azimuth=0.9, elevation=0.3, distance=58.0, flags=g.types.REQUEST_BAKE)
    march = g.RequestSpec(480, 270, 4096, 0.0, azimuth=0.9, elevation=0.3, distance=58.0)
    server = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED)
    mixed = run(server, [bake, march, g.RequestSpec(320, 180, 256, 0.9)], debug=True)
    (bp, bd, br), (mp, _, mr) = mixed[0], mixed[1]
    assert br.counters.rays == 480 * 270 and br.ray_steps > 0
    assert not bd.any()  # the walk writes colour only
    lb, lm = luminance(bp), luminance(mp)
    assert abs(lb.sum() - lm.sum()) / lm.sum() < 0.01, abs(lb.sum() - lm.sum()) / lm.sum()
    alone = run(server, [bake])[0]
    assert np.array_equal(alone[0].view(np.uint16), bp.view(np.uint16))
    assert alone[2].ray_steps == br.ray_steps
    server.close()
    serial = g.Server(world["ctx"], world["vol"], g.types.SERVE_SERIAL_PLAIN)
    one = run(serial, [bake])[0]
    assert np.array_equal(one[0].view(np.uint16), bp.view(np.uint16)) and one[2].ray_steps == br.ray_steps
    serial.close()


def test_bake_storage_counts_in_admission(world):
    """A bake request's footprint holds its stored samples (96 half4 and a
    16-byte header per pixel): with memory for one such request at a time,
    three are served one after another, each admitted once the previous one
    released its storage, all with the same pixels. A Kerr bake is
    refused."""
    import gargantua_b200 as g

    spec = g.RequestSpec(480, 270, 256, 0.0, flags=g.types.REQUEST_BAKE)
    one = 480 * 270 * (8 + 96 * 8 + 16) + 128 + 8192 + 4
    server = g.Server(world["ctx"], world["vol"], g.types.SERVE_BATCHED, memory_bytes=int(one * 1.5))
    results = run(server, [spec] * 3)
    for pix, _, res in results:
        assert res.counters.rays == 480 * 270
        assert np.array_equal(pix.view(np.uint16), results[0][0].view(np.uint16))
    order = sorted(results, key=lambda r: r[2].admitted)
    for before, after in zip(order, order[1:]):
        assert after[2].admitted >= before[2].finished  # admitted only once storage frees (server clock)
    with pytest.raises(g.GargantuaError) as e:
        server.submit(g.RequestSpec(320, 180, 256, 0.5, flags=g.types.REQUEST_BAKE))
    assert e.value.status == 8
    server.close()
