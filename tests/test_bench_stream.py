"""The served-stream workload bench.py measures: 512 still requests from a
fixed seed, Poisson arrivals at 40 per second, resolutions 320x180 to
3840x2160, 256 or 4096 steps, spin 0, 0.5 or 0.9, camera radius in [40, 120],
inclination in [10, 90] degrees, any azimuth; the same seed gives the same
stream."""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_stream_is_reproducible_and_seeded():
    a, b = bench.make_stream(1), bench.make_stream(1)
    assert a == b
    assert bench.make_stream(2) != a
    assert len(a) == bench.STREAM_LENGTH == 512


def test_stream_parameters_stay_in_their_sets_and_ranges():
    s = bench.make_stream(1)
    assert {(q["width"], q["height"]) for q in s} == set(bench.RESOLUTIONS)
    assert {q["step_cap"] for q in s} == {256, 4096}
    assert {q["spin"] for q in s} == {0.0, 0.5, 0.9}
    r = np.array([q["distance"] for q in s])
    assert r.min() >= 40.0 and r.max() <= 120.0
    inc = np.degrees(math.pi / 2.0 - np.array([q["elevation"] for q in s]))
    assert inc.min() >= 10.0 - 1e-9 and inc.max() <= 90.0 + 1e-9
    az = np.array([q["azimuth"] for q in s])
    assert az.min() >= 0.0 and az.max() < 2.0 * math.pi
    assert len({q["seed"] for q in s}) == len(s)


def test_arrivals_are_poisson_at_forty_per_second():
    t = np.array([q["t"] for q in bench.make_stream(1)])
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert (gaps > 0).all()
    rate = len(t) / t[-1]
    assert 34.0 < rate < 46.0  # 512 exponential gaps: the sample rate is within ~12 %
    # exponential gaps: the coefficient of variation is near 1
    assert 0.8 < gaps.std() / gaps.mean() < 1.2


def test_every_slice_and_the_latency_replay_are_full_at_any_step_count():
    """bench.py --steps 20 --warmup 5 at 32 requests per step needs 800 timed
    and warm-up requests plus 48 for the open-loop latency replay; the stream
    grows to cover them, and its first 512 requests do not change."""
    for warmup, steps, per_step, latency in [(5, 20, 32, 48), (3, 8, 32, 48), (1, 1, 2, 0)]:
        count = bench.stream_length(warmup, steps, per_step, latency)
        s = bench.make_stream(1, count)
        slices = [s[i * per_step:(i + 1) * per_step] for i in range(warmup + steps)]
        assert all(len(sl) == per_step for sl in slices)
        assert len(s[(warmup + steps) * per_step:(warmup + steps) * per_step + latency]) == latency
    assert bench.make_stream(1, 900)[:512] == bench.make_stream(1)


def test_class_requests_cover_one_class_each():
    for (w, h) in bench.RESOLUTIONS:
        for cap in bench.STEP_CAPS:
            for kerr in (False, True):
                reqs = bench.class_requests(w, h, cap, kerr, 7)
                assert 2 <= len(reqs) <= 32
                assert {(q["width"], q["height"], q["step_cap"]) for q in reqs} == {(w, h, cap)}
                spins = {q["spin"] for q in reqs}
                assert spins <= ({0.5, 0.9} if kerr else {0.0})
