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
