"""The particle step tests |v| > PLUNGE_SPEED_LIMIT and the swept chord's
closest approach < R_CAPTURE on squared lengths (sim.metal:66-72 takes the
square roots). The rewrite is exact only for the bounds in sim.cu; this
repeats the search that found them: every float near the square, through a
correctly rounded float32 square root."""
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _sim_constants():
    with open(os.path.join(ROOT, "gargantua_b200", "csrc", "sim.cu")) as fh:
        src = fh.read()
    speed = float(re.search(r"kPlungeSpeedSquared = ([0-9.]+)f;", src).group(1))
    capture_bits = int(re.search(r"kCaptureClosestSquaredBits = (0x[0-9a-f]+)u;", src).group(1), 16)
    return np.float32(speed), np.uint32(capture_bits).view(np.float32)


def _floats_around(x, span=1 << 14):
    base = int(np.float32(x).view(np.uint32))
    return np.arange(base - span, base + span, dtype=np.int64).astype(np.uint32).view(np.float32)


def test_speed_bound_is_exact():
    speed_sq, _ = _sim_constants()
    s = _floats_around(np.float32(12.0) * np.float32(12.0))
    assert np.array_equal(np.sqrt(s) > np.float32(12.0), s > speed_sq)


def test_capture_bound_is_exact():
    _, capture_sq = _sim_constants()
    c = np.float32(2.02)
    s = _floats_around(c * c)
    assert np.array_equal(np.sqrt(s) < c, s < capture_sq)


def test_bounds_hold_far_from_the_squares():
    # sqrt is monotone, so one agreement on each side of the window covers
    # every other float; check the extremes and the specials anyway.
    speed_sq, capture_sq = _sim_constants()
    s = np.array([0.0, 1e-30, 1.0, 4.0, 100.0, 1e10, 3.4e38, np.inf, np.nan], np.float32)
    assert np.array_equal(np.sqrt(s) > np.float32(12.0), s > speed_sq)
    assert np.array_equal(np.sqrt(s) < np.float32(2.02), s < capture_sq)


def test_chord_test_skip_never_changes_the_capture_decision():
    """The step kernel skips the chord's closest-approach test when the
    substep starts at |x| > 4 and moves less than 1 (squared length < 1):
    then the squared closest approach, computed in float32 in the kernel's
    order, is far above the capture bound, so the test could not fire.
    Checked on random and adversarial chords (aimed at the centre, starting
    just outside 4, moving just under 1)."""
    rng = np.random.default_rng(3)
    f = np.float32
    n = 200_000
    b = rng.normal(size=(n, 3)).astype(f)
    b /= np.linalg.norm(b, axis=1, keepdims=True).astype(f)
    rb = rng.uniform(4.0, 6.0, n).astype(f)
    rb[: n // 2] = np.nextafter(f(4.0), f(5.0))
    b *= rb[:, None]
    t = -b / np.linalg.norm(b, axis=1, keepdims=True).astype(f)  # straight at the centre
    t[n // 2:] = rng.normal(size=(n - n // 2, 3)).astype(f)
    t /= np.linalg.norm(t, axis=1, keepdims=True).astype(f)
    t *= rng.uniform(0.9, 0.99999, n).astype(f)[:, None]
    r = np.sqrt((b * b).sum(axis=1, dtype=f)).astype(f)
    tt = (t[:, 0] * t[:, 0] + t[:, 1] * t[:, 1] + t[:, 2] * t[:, 2]).astype(f)
    skip = (r > f(4.0)) & (tt < f(1.0))
    assert skip.sum() > n // 2
    bt = (b[:, 0] * t[:, 0] + b[:, 1] * t[:, 1] + b[:, 2] * t[:, 2]).astype(f)
    along = np.clip(-bt / np.maximum(tt, f(1e-12)), f(0), f(1)).astype(f)
    c = (b + along[:, None] * t).astype(f)
    closest_squared = (c[:, 0] * c[:, 0] + c[:, 1] * c[:, 1] + c[:, 2] * c[:, 2]).astype(f)
    bound = np.array([0x408292A2], np.uint32).view(f)[0]
    assert (closest_squared[skip] > f(8.9)).all()
    assert (closest_squared[skip] >= bound).all()
