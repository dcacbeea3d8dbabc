"""The oracle pinned to the reference's own known-answer tests.

Each test restates one of gargantua's oracle tests (Tests/OracleTests/*.swift,
file:line in each docstring) against the C restatement in oracle/, so the
checker every GPU parity test relies on is itself anchored to the analytic
values and tolerances the reference holds its oracle to. CPU only.
"""
import math

import numpy as np
import pytest

import oracle_ffi as O
from conftest import golden_passes, load_golden

PW, NEWTON = 1, 0


# ---------------------------------------------------------------- potentials

def test_pw_angular_momentum_minimal_at_isco():
    """OracleTests.swift:6-17"""
    L = O.lib()
    rs = np.arange(3.0, 20.0, 1e-4)
    ls = np.array([L.o_circular_angular_momentum(PW, r) for r in rs[::10]])
    best = rs[::10][np.argmin(ls)]
    # refine around the coarse minimum at the original 1e-4 spacing
    fine = np.arange(best - 2e-3, best + 2e-3, 1e-4)
    best = fine[np.argmin([L.o_circular_angular_momentum(PW, r) for r in fine])]
    assert abs(best - 6.0) < 1e-3


def test_pw_marginally_bound_orbit_zero_energy():
    """OracleTests.swift:19-22"""
    assert abs(O.lib().o_circular_energy(PW, 4.0)) < 1e-12


def test_circular_speeds_closed_forms():
    """OracleTests.swift:24-28"""
    L = O.lib()
    assert abs(L.o_circular_speed(PW, 6.0) - math.sqrt(6.0) / 4.0) < 1e-12
    assert abs(L.o_circular_speed(NEWTON, 4.0) - 0.5) < 1e-12
    assert abs(L.o_angular_frequency(PW, 6.0) - 1.0 / math.sqrt(96.0)) < 1e-12


# ------------------------------------------------------------------ dynamics

def test_circular_orbit_stays_circular_without_drag():
    """OracleTests.swift:38-55"""
    L = O.lib()
    st = np.zeros(6)
    L.o_circular_orbit(8.0, 0.3, PW, st)
    period = 2 * math.pi / L.o_angular_frequency(PW, 8.0)
    steps = int(100.0 * period / 0.1)
    e0 = L.o_specific_energy(PW, st)
    lz0 = L.o_angular_momentum_z(st)
    low = high = 8.0
    for _ in range(steps):
        L.o_dynamics_step(PW, 0.1, 0.0, st)
        r = math.sqrt(st[0] ** 2 + st[1] ** 2 + st[2] ** 2)
        low, high = min(low, r), max(high, r)
    assert high - low < 0.1
    assert abs(L.o_specific_energy(PW, st) - e0) / abs(e0) < 1e-4
    assert abs(L.o_angular_momentum_z(st) - lz0) / abs(lz0) < 1e-9


def test_drag_spirals_inward():
    """OracleTests.swift:57-65"""
    L = O.lib()
    st = np.zeros(6)
    L.o_circular_orbit(12.0, 0.0, PW, st)
    period = 2 * math.pi / L.o_angular_frequency(PW, 12.0)
    for _ in range(int(2.0 * period / 0.1)):
        L.o_dynamics_step(PW, 0.1, 0.003, st)
    r = math.sqrt(st[0] ** 2 + st[1] ** 2 + st[2] ** 2)
    assert 9.5 < r < 11.5


def test_orbit_inside_isco_plunges_and_outside_survives():
    """OracleTests.swift:67-78, 92-103"""
    L = O.lib()
    st = np.zeros(6)
    L.o_circular_orbit(5.0, 0.0, PW, st)
    st[3:] *= 0.99
    captured = False
    for _ in range(20000):
        L.o_dynamics_step(PW, 0.1, 0.0, st)
        if math.sqrt(st[0] ** 2 + st[1] ** 2 + st[2] ** 2) < 2.02:
            captured = True
            break
    assert captured
    L.o_circular_orbit(8.0, 0.0, PW, st)
    st[3:] *= 0.99
    low = 8.0
    for _ in range(20000):
        L.o_dynamics_step(PW, 0.1, 0.0, st)
        low = min(low, math.sqrt(st[0] ** 2 + st[1] ** 2 + st[2] ** 2))
    assert low > 5.0


def test_tunnelling_through_the_capture_sphere_counts():
    """OracleTests.swift:80-90"""
    L = O.lib()
    assert L.o_dynamics_removed(np.array([3.0, 0.1, 0.0]), np.array([-3.0, 0.1, 0.0, -60.0, 0.0, 0.0]))
    assert not L.o_dynamics_removed(np.array([2.6, 2.4, 0.0]), np.array([2.5, 2.5, 0.0, 0.5, 0.0, 0.0]))
    assert L.o_dynamics_removed(np.array([9.0, 0.0, 0.0]), np.array([10.0, 0.0, 0.0, 40.0, 0.0, 0.0]))


# ---------------------------------------------------------------- disk model

def test_temperature_peaks_at_49_over_36_isco():
    """OracleTests.swift:107-120"""
    L = O.lib()
    peak_r = L.o_disk_peak_radius()
    peak = L.o_disk_temperature(peak_r, 8000.0)
    assert abs(peak - 8000.0) < 1e-9
    assert L.o_disk_temperature(7.5, 8000.0) < peak
    assert L.o_disk_temperature(9.0, 8000.0) < peak
    assert L.o_disk_temperature(24.0, 8000.0) < 0.7 * peak
    edge = L.o_disk_temperature(6.0, 8000.0)
    assert 0.0 < edge < 0.8 * 8000.0
    assert L.o_disk_temperature(3.0, 8000.0) > edge


def test_steady_profile_vanishes_at_edges():
    """OracleTests.swift:122-128"""
    L = O.lib()
    assert L.o_steady_surface_density(6.0) == 0.0
    assert L.o_steady_surface_density(24.0) == 0.0
    assert L.o_steady_surface_density(10.0) > 0.0
    ratio = L.o_steady_surface_density(6.2) / L.o_steady_surface_density(6.1)
    assert abs(ratio - 2.0 * (6.1 / 6.2) ** 1.5) < 1e-9


def test_inverse_cdf_monotone_and_spans_disk():
    """OracleTests.swift:130-136"""
    t = O.inverse_cdf(1024)
    assert t[0] == 6.0 and t[-1] == 24.0
    assert np.all(np.diff(t) >= 0)
    assert 10.0 < t[512] < 20.0


def test_inverse_cdf_reproduces_profile():
    """OracleTests.swift:138-156"""
    L = O.lib()
    table = O.inverse_cdf(4096)
    bins = 36
    counts = np.zeros(bins)
    draws = 200_000
    for i in range(draws):
        u = O.lib().o_hash_unit(O.hash_draw(7, i, 0)[0])
        pos = u * (len(table) - 1)
        k = min(int(pos), len(table) - 2)
        r = table[k] + (pos - k) * (table[k + 1] - table[k])
        counts[min(int((r - 6.0) / 0.5), bins - 1)] += 1
    expected = np.array([L.o_radial_number_density(6.0 + (b + 0.5) * 0.5) for b in range(bins)])
    expected *= draws / expected.sum()
    for b in range(1, bins - 1):
        if expected[b] > 2000:
            assert abs(counts[b] - expected[b]) / expected[b] < 0.05


# ----------------------------------------------------------------- blackbody

def test_blackbody_locus_and_table():
    """OracleTests.swift:160-180"""
    L = O.lib()
    import ctypes as C

    x, y = C.c_double(), C.c_double()
    L.o_blackbody_chromaticity(6500.0, C.byref(x), C.byref(y))
    assert abs(x.value - 0.3135) < 0.01 and abs(y.value - 0.3237) < 0.01
    cool, hot = np.zeros(3), np.zeros(3)
    L.o_blackbody_color(2000.0, cool)
    L.o_blackbody_color(20000.0, hot)
    assert cool[0] == 1.0 and cool[1] < cool[0] and cool[2] < cool[1]
    assert hot[2] == 1.0 and hot[0] < hot[2]
    table = O.blackbody_table()
    assert table.shape == (256, 3)
    assert np.all(table.max(axis=1) == 1.0) and table.min() >= 0.0
    assert L.o_blackbody_coordinate(1000.0, 1000.0, 40000.0) == 0.0
    assert L.o_blackbody_coordinate(40000.0, 1000.0, 40000.0) == 1.0


# ---------------------------------------------------------------------- hash

def test_pcg4d_deterministic_and_lanes_differ():
    """OracleTests.swift:184-192"""
    a = O.hash_draw(42, 7, 3)
    assert a == O.hash_draw(42, 7, 3)
    assert O.hash_draw(43, 7, 3) != a
    assert O.hash_draw(42, 8, 3) != a
    assert O.hash_draw(42, 7, 4) != a
    assert O.hash_draw(42, 7, 3, lane=1) != a


def test_pcg4d_known_answer():
    """The pcg4d arithmetic (Hash.swift:9-21) restated in numpy agrees with
    the oracle bit for bit over many inputs."""
    rng = np.random.default_rng(0)
    v = rng.integers(0, 2**32, size=(1000, 4), dtype=np.uint64).astype(np.uint32)
    w = (v * np.uint32(1664525) + np.uint32(1013904223)).astype(np.uint32)
    for _ in range(2):
        w[:, 0] += w[:, 1] * w[:, 3]
        w[:, 1] += w[:, 2] * w[:, 0]
        w[:, 2] += w[:, 0] * w[:, 1]
        w[:, 3] += w[:, 1] * w[:, 2]
        if _ == 0:
            w ^= w >> np.uint32(16)
    import ctypes as C

    for row, expect in zip(v[:50], w[:50]):
        out = (C.c_uint32 * 4)()
        O.lib().o_pcg4d((C.c_uint32 * 4)(*[int(x) for x in row]), out)
        assert tuple(out) == tuple(int(x) for x in expect)


def test_unit_deviates_uniform_and_gaussian_variance():
    """OracleTests.swift:194-221"""
    L = O.lib()
    n = 100_000
    us = np.array([L.o_hash_unit(O.hash_draw(1, i, 0)[1]) for i in range(n)])
    assert abs(us.mean() - 0.5) < 0.005 and us.min() >= 0.0 and us.max() < 1.0
    import ctypes as C

    g0, g1 = C.c_double(), C.c_double()
    s = ss = 0.0
    for i in range(n):
        h = O.hash_draw(3, i, 1)
        L.o_gaussian_pair(L.o_hash_unit(h[0]), L.o_hash_unit(h[1]), C.byref(g0), C.byref(g1))
        s += g0.value + g1.value
        ss += g0.value ** 2 + g1.value ** 2
    mean = s / (2 * n)
    assert abs(mean) < 0.01 and abs(ss / (2 * n) - mean * mean - 1.0) < 0.02


# ------------------------------------------------------------------ geodesic

def test_launch_reproduces_origin_direction_and_null_condition():
    """GeodesicTests.swift:6-16"""
    origin = np.array([30.0, -10.0, 12.0])
    d = np.array([-0.8, 0.3, -0.1])
    ray = O.launch(origin, d)
    unit = d / np.linalg.norm(d)
    assert np.max(np.abs(O.position(ray) - origin)) < 1e-12
    assert abs(O.direction(ray) @ unit - 1.0) < 1e-12
    assert abs(O.lib().o_null_residual(ray.s)) < 1e-12
    assert abs(ray.energy - math.sqrt(1 - 2 / np.linalg.norm(origin))) < 1e-12


def test_impact_parameter_launch():
    """GeodesicTests.swift:18-22"""
    ray = O.launch_b(50.0, 5.0)
    assert abs(ray.angular_momentum / ray.energy - 5.0) < 1e-12
    assert ray.s[4] < 0


def test_conserved_quantities_hold_in_double_precision():
    """GeodesicTests.swift:24-41: drift < 1e-6 and fourth-order refinement."""
    st = O.Settings(0.02, 0.02, 0.5, 2.02, 60.0, 4096, 0.02, 0.5)
    ray = O.launch([40.0, 5.0, 15.0], [-0.95, -0.2, -0.3])
    outcome, steps, drift = O.integrate(ray, st)
    assert outcome != O.EXHAUSTED
    assert drift < 1e-6
    assert abs(O.lib().o_null_residual(ray.s)) < 1e-6
    fine = O.Settings(0.01, 0.01, 0.25, 2.02, 60.0, 4096, 0.01, 0.25)
    ray2 = O.launch([40.0, 5.0, 15.0], [-0.95, -0.2, -0.3])
    _, _, drift2 = O.integrate(ray2, fine)
    assert drift2 < drift / 8.0


def test_critical_impact_parameter_is_three_root_three():
    """GeodesicTests.swift:43-46"""
    bc = O.lib().o_critical_impact_parameter(50.0, O.still(), 60)
    assert abs(bc - 3 * math.sqrt(3)) / (3 * math.sqrt(3)) < 1e-4


def test_capture_inside_and_escape_outside():
    """GeodesicTests.swift:48-53"""
    assert O.integrate(O.launch_b(50.0, 4.0), O.still())[0] == O.CAPTURED
    assert O.integrate(O.launch_b(50.0, 7.0), O.still())[0] == O.ESCAPED


def test_weak_field_deflection_is_four_over_b():
    """GeodesicTests.swift:55-65"""
    b, radius = 1000.0, 50000.0
    st = O.Settings(0.02, 0.02, math.inf, 2.02, radius, 4096, 0.02, math.inf)
    launch = O.launch_b(radius, b)
    ray = O.launch_b(radius, b)
    outcome, _, _ = O.integrate(ray, st)
    assert outcome == O.ESCAPED
    import ctypes as C

    defl = O.lib().o_deflection(C.byref(launch), C.byref(ray))
    assert abs(defl - 4.0 / b) / (4.0 / b) < 0.005


def test_radial_ray_falls_straight_in():
    """GeodesicTests.swift:67-73"""
    ray = O.launch([20.0, 0.0, 0.0], [-1.0, 0.0, 0.0])
    outcome, _, _ = O.integrate(ray, O.interactive())
    assert outcome == O.CAPTURED
    assert abs(ray.s[2]) < 1e-12 and abs(ray.angular_momentum) < 1e-12


# ---------------------------------------------------------------- deflection

def test_sweep_tables():
    """DeflectionTests.swift:6-54"""
    L = O.lib()
    assert abs(L.o_sweep(100.0, 0.01, 2048) - 0.01 / 100.0) < 1e-9
    for b in (6.0, 10.0, 30.0, 1000.0):
        peri = L.o_periapsis(b)
        assert abs(1.0 - b * b / (peri * peri) * (1.0 - 2.0 / peri)) < 1e-12
        assert 3.0 < peri < b
    b = 1000.0
    peri = L.o_periapsis(b)
    defl = 2.0 * L.o_sweep(peri, b, 2048) - math.pi
    assert abs(defl - 4.0 / b) / (4.0 / b) < 0.005
    assert abs(L.o_escape_sweep(1e7, b, 2048) - (defl + math.pi - b / 1e7)) < 1e-7
    for t in (0.0, 0.1, 0.5, 0.9, 1.0):
        bb = L.o_table_impact_parameter(2.0, 30.0, t)
        assert abs(L.o_table_coordinate(2.0, 30.0, bb) - t) < 1e-12
    sphere = O.sweep_table(30.0, 256, 2048)
    assert sphere[0] == 0.0 and np.all(np.diff(sphere) >= 0) and sphere[-1] < math.pi
    sky = O.sky_table(52.0, 30.0, 256, 2048)
    assert np.all((sky > 0.0) & (sky < 2 * math.pi))


def test_sweep_agrees_with_the_integrator():
    """DeflectionTests.swift:36-45"""
    b = 10.0
    ray = O.launch_b(50000.0, b)
    st = O.Settings(0.01, 0.02, 2.0, 2.02, 50000.0, 200000, 0.01, 2.0)
    outcome, _, _ = O.integrate(ray, st)
    assert outcome == O.ESCAPED
    expected = O.lib().o_turning_sweep(50000.0, b, 2048)
    assert abs(ray.s[2] - expected) < 1e-5


# ---------------------------------------------------------------------- kerr

def test_kerr_photon_orbits_bracket_schwarzschild():
    """KerrTests.swift:6-15"""
    import ctypes as C

    L = O.lib()
    pro, retro = C.c_double(), C.c_double()
    L.o_kerr_photon_orbits(0.9, C.byref(pro), C.byref(retro))
    assert abs(pro.value - 2.0 * (1.0 + math.cos(2.0 / 3.0 * math.acos(-0.9)))) < 1e-12
    assert pro.value < 3.0 < retro.value
    for rc in (pro.value, retro.value):
        assert abs(L.o_kerr_critical_eta(0.9, rc)) < 1e-9
    L.o_kerr_photon_orbits(1e-9, C.byref(pro), C.byref(retro))
    assert abs(pro.value - 3.0) < 1e-3 and abs(retro.value - 3.0) < 1e-3


def test_kerr_zero_spin_reduces_to_schwarzschild():
    """KerrTests.swift:17-32"""
    for aim in (0.15, 0.3):
        s = np.zeros(7)
        O.lib().o_kerr_launch(0.0, np.array([50.0, 0, 0]), np.array([-1.0, aim, 0.0]), s)
        import ctypes as C

        steps, drift = C.c_int64(), C.c_double()
        ko = O.lib().o_kerr_integrate(0.0, s, C.byref(O.kerr_settings(100_000)), C.byref(steps), C.byref(drift))
        ray = O.launch([50.0, 0, 0], [-1.0, aim, 0.0])
        so, _, _ = O.integrate(ray, O.Settings(0.02, 0.02, 0.5, 2.02, 60.0, 100_000, 0.02, 0.5))
        assert ko == O.ESCAPED and so == O.ESCAPED
        assert abs(s[2] - ray.s[2]) < 2e-4


def test_kerr_carter_and_null_residual_hold():
    """KerrTests.swift:34-43"""
    import ctypes as C

    for d in ([-1.0, 0.12, 0.0], [-1.0, -0.09, 0.05], [-0.9, 0.05, -0.2]):
        s = np.zeros(7)
        O.lib().o_kerr_launch(0.9, np.array([45.0, 12.0, 9.0]), np.array(d), s)
        assert abs(O.lib().o_kerr_null_residual(0.9, s)) < 1e-10
        steps, drift = C.c_int64(), C.c_double()
        out = O.lib().o_kerr_integrate(0.9, s, C.byref(O.kerr_settings(100_000)), C.byref(steps), C.byref(drift))
        assert out != O.EXHAUSTED
        assert drift.value < 1e-7


def test_kerr_shadow_edges_match_bardeen():
    """KerrTests.swift:45-77"""
    import ctypes as C

    a, radius = 0.9, 5000.0
    st = O.KerrSettings(0.02, 0.005, 1e9, 0.05, radius, 40_000)
    L = O.lib()
    pro, retro = C.c_double(), C.c_double()
    L.o_kerr_photon_orbits(a, C.byref(pro), C.byref(retro))
    xi_pro = L.o_kerr_critical_xi(a, pro.value)
    xi_retro = L.o_kerr_critical_xi(a, retro.value)
    m_pro = L.o_kerr_bisect_critical_xi(a, radius, 1.0, C.byref(st), 48)
    m_retro = L.o_kerr_bisect_critical_xi(a, radius, -1.0, C.byref(st), 48)
    assert abs(m_pro - xi_pro) / abs(xi_pro) < 1e-3
    assert abs(m_retro - xi_retro) / abs(xi_retro) < 1e-3
    assert abs(m_retro / m_pro) > 2.0


def test_kerr_zero_angular_momentum_rays_are_dragged():
    """KerrTests.swift:79-87"""
    import ctypes as C

    s = np.zeros(7)
    O.lib().o_kerr_launch(0.9, np.array([20.0, 0, 0]), np.array([-1.0, 0.0, 0.0]), s)
    s[6] = 0.0
    steps, drift = C.c_int64(), C.c_double()
    out = O.lib().o_kerr_integrate(0.9, s, C.byref(O.kerr_settings(100_000)), C.byref(steps), C.byref(drift))
    assert out == O.CAPTURED and s[2] > 0.05


# ------------------------------------------------------- volume and rendering

def test_volume_field_texel_centres_exact_and_zero_outside():
    """LensedRenderTests.swift:55-71"""
    size = 4
    em = np.zeros((64, 4))
    vel = np.tile([1.0, 2.0, 3.0], (64, 1))
    em[(1 * 4 + 2) * 4 + 3] = [5, 6, 7, 8]
    centre = np.array([3.5, 2.5, 1.5]) - 2.0
    e4, v3 = np.zeros(4), np.zeros(3)
    O.lib().o_volume_sample(size, 2.0, em, vel, centre, e4, v3)
    assert list(e4) == [5, 6, 7, 8] and list(v3) == [1, 2, 3]
    O.lib().o_volume_sample(size, 2.0, em, vel, centre - np.array([0.5, 0, 0]), e4, v3)
    assert abs(e4[3] - 4.0) < 1e-12
    O.lib().o_volume_sample(size, 2.0, em, vel, np.array([3.0, 0, 0]), e4, v3)
    assert e4[3] == 0.0 and list(v3) == [0, 0, 0]


def synthetic_disk(size: int, moving: bool):
    """The SyntheticDisk fixture (LensedRenderTests.swift:7-53)."""
    L = O.lib()
    half = 30.0
    voxel = 2 * half / size
    em = np.zeros((size ** 3, 4))
    vel = np.zeros((size ** 3, 3))
    c = (np.arange(size) + 0.5) * voxel - half
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    r = np.sqrt(x * x + y * y)
    mask = (r > 6.0) & (r < 24.0) & (np.abs(z) < 0.75)
    idx = np.flatnonzero(mask.ravel())
    rr = r.ravel()[idx]
    for i, rv in zip(idx, rr):
        t = L.o_disk_temperature(rv, 8000.0)
        col = np.zeros(3)
        L.o_blackbody_color(t, col)
        em[i, :3] = col * (t / 8000.0) ** 4
        em[i, 3] = 100.0
        if moving:
            v = L.o_circular_speed(PW, rv)
            vel[i] = [-v * y.ravel()[i] / rv, v * x.ravel()[i] / rv, 0.0]
    return em, vel


def synthetic_camera(width: int, height: int):
    """SyntheticDisk.camera (LensedRenderTests.swift:55-66): elevation 0.32,
    azimuth 0.6, distance 52, fov 50 degrees."""
    el, az, dist = 0.32, 0.6, 52.0
    pos = dist * np.array([math.cos(el) * math.cos(az), math.cos(el) * math.sin(az), math.sin(el)])
    fwd = -pos / dist
    right = np.array([fwd[1], -fwd[0], 0.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    t = math.tan(50.0 * math.pi / 360.0)
    return np.concatenate([pos, right, up, fwd, [t * width / height, t]])


def test_static_disk_symmetric_moving_disk_beamed():
    """LensedRenderTests.swift:75-87"""
    w, h = 64, 36
    cam = synthetic_camera(w, h)
    em, vel = synthetic_disk(60, moving=False)
    img = O.lensed_image(w, h, cam, 60, 30.0, em, vel, O.still())
    ratio = O.side_ratio(O.luminance(img), w, h)
    assert abs(ratio - 1.0) < 0.05
    assert O.luminance(img).sum() > 0
    em, vel = synthetic_disk(60, moving=True)
    img = O.lensed_image(w, h, cam, 60, 30.0, em, vel, O.still())
    assert O.side_ratio(O.luminance(img), w, h) > 1.3


def test_redshift_factor_limits():
    """LensedRenderTests.swift:89-104"""
    L = O.lib()
    x = np.array([1.0, 0, 0])
    zero = np.zeros(3)
    assert abs(L.o_redshift_factor(1e6, x, zero) - 1.0) < 1e-5
    assert abs(L.o_redshift_factor(2.5, x, zero) - math.sqrt(1 - 2 / 2.5)) < 1e-12
    assert L.o_redshift_factor(1e6, x, np.array([-0.3, 0, 0])) > 1.0
    assert L.o_redshift_factor(1e6, x, np.array([0.3, 0, 0])) < 1.0
    fast = L.o_redshift_factor(1e6, x, np.array([-5.0, 0, 0]))
    assert math.isfinite(fast) and fast < (1 + 0.85) / math.sqrt(1 - 0.85) * 1.0001
    plunge = L.o_redshift_factor(2.05, np.array([0, 1.0, 0]), np.array([0, -89.0, 0]))
    assert math.isfinite(plunge) and plunge > 0


# ------------------------------------------------------------------- goldens

def test_every_golden_parses_and_tolerance_semantics():
    """GoldenTests.swift:18-33"""
    import os

    from conftest import GOLDEN_DIR

    names = sorted(f[:-5] for f in os.listdir(GOLDEN_DIR) if f.endswith(".json"))
    assert len(names) == 11
    for n in names:
        g = load_golden(n)
        assert g["name"] == n and g["claim"] and g["method"]
    iso = load_golden("isco")
    assert golden_passes(iso, 6.29) and not golden_passes(iso, 6.31) and golden_passes(iso, 5.71)


def test_oracle_disk_settles_to_an_inner_edge_at_isco():
    """GoldenTests.swift:39-64: 24 000 particles, seed 11, 1500 substeps."""
    import ctypes as C

    g = load_golden("isco")
    count = 24000
    radii = np.zeros(count)
    respawns = C.c_uint32()
    O.lib().o_disk_settle(count, 11, int(g["parameters"]["settlingSteps"]), PW, 0.1, 0.003, radii, C.byref(respawns))
    p = g["parameters"]
    edge = O.lib().o_disk_inner_edge(radii, count, p["binWidth"], p["fitInner"], p["fitOuter"])
    assert golden_passes(g, edge), edge
    assert respawns.value > 0


def test_edge_measurement_recovers_analytic_profile():
    """GoldenTests.swift:66-77"""
    table = O.inverse_cdf(4096)
    L = O.lib()
    n = 400_000
    u = np.array([L.o_hash_unit(O.hash_draw(5, i, 0)[0]) for i in range(n)])
    pos = u * (len(table) - 1)
    k = np.minimum(pos.astype(np.int64), len(table) - 2)
    radii = table[k] + (pos - k) * (table[k + 1] - table[k])
    edge = L.o_disk_inner_edge(np.ascontiguousarray(radii), n, 0.25, 6.5, 9.0)
    assert abs(edge - 6.0) < 0.1


def test_bake_oracle_follows_the_integrator():
    """The FP64 bake (o_bake_batch, bake.metal:46-91 in the oracle's
    integrator) steps exactly as o_integrate does: a ray's final direction
    is the integrator's, every stored point lies in the slab at least the
    spacing of path after the previous one, and the stored paths add up to
    at most the path walked (the rest is after the last stored point)."""
    rng = np.random.default_rng(4)
    cam = np.array([40.0, 20.0, 16.0])
    fwd = -cam / np.linalg.norm(cam)
    dirs = fwd + rng.normal(scale=0.12, size=(48, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    probes = np.concatenate([np.broadcast_to(cam, dirs.shape), dirs], axis=1)
    spacing = 0.234375
    samples, counts, over, falls, dd = O.bake_batch(probes, O.still(), spacing, threads=1)
    ref = O.integrate_batch(probes, O.still(), 1)
    assert counts.max() > 0 and (counts <= 96).all()
    for i in range(len(probes)):
        n = counts[i]
        if ref[i, 7] != O.CAPTURED:
            assert np.allclose(dd[i, :3], ref[i, 3:6], rtol=0, atol=1e-12), i
        pts = samples[i, :n]
        assert (np.abs(pts[:, 2]) < 6.0).all() and (np.abs(pts[:, :2]) < 30.0).all()
        assert (pts[:, 3] >= spacing).all()
        assert 0.0 <= dd[i, 3] <= 1.0
    assert set(np.unique(falls)) <= {0, 1}
    assert (falls[ref[:, 7] == O.CAPTURED] == 1).all()


def test_present_replica_matches_the_fp64_tone_curve():
    """The FP32 tone-curve replica (o32_present + o32_srgb8, the kernel's
    arithmetic) against PBR Neutral in FP64 (o_pbr_neutral, present.metal:
    22-35) encoded to sRGB in FP64: within one code value everywhere."""
    rng = np.random.default_rng(8)
    rgba = rng.uniform(0.0, 4.0, (4000, 4)).astype(np.float16)
    rgba[::5] = rng.uniform(0.0, 0.09, (len(rgba[::5]), 4)).astype(np.float16)
    got = O.present32(rgba, 1.3)
    want = np.zeros((len(rgba), 3))
    for k, row in enumerate(rgba.astype(np.float64)):
        out = np.zeros(3)
        O.lib().o_pbr_neutral(np.ascontiguousarray(np.maximum(row[:3] * float(np.float32(1.3)), 0.0)), out)
        v = np.clip(out, 0.0, 1.0)
        want[k] = np.round(np.where(v <= 0.0031308, 12.92 * v, 1.055 * v ** (1 / 2.4) - 0.055) * 255.0)
    assert np.abs(got[:, :3].astype(np.float64) - want).max() <= 1.0
    assert (got[:, 3] == 255).all()


def test_threaded_replicas_equal_the_serial_ones():
    """The CPU baseline's all-core deposit (atomic adds of the same integer
    words) and resolve (independent voxels) give the serial replica's
    outputs bit for bit."""
    rng = np.random.default_rng(1)
    n = 100_000
    p = np.zeros((n, 8), np.float32)
    p[:, :3] = rng.uniform(-31, 31, (n, 3))
    p[:, 3:6] = rng.normal(0, 1, (n, 3))
    p[:, 6] = rng.uniform(1000, 12000, n)
    for exact in (True, False):
        a = O.deposit32(p, 40, 3, exact, 1)
        b = O.deposit32(p, 40, 3, exact, 1, threads=0)
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
    bb = np.random.default_rng(2).uniform(0, 1, (256, 3)).astype(np.float32)
    r1, r2 = O.resolve32(*a, 40, bb), O.resolve32(*a, 40, bb, threads=0)
    assert all(np.array_equal(x.view(np.uint32), y.view(np.uint32)) for x, y in zip(r1, r2))
