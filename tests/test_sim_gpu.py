"""Particle pass on the device against the FP32 replica (bit-exact) and the
FP64 oracle (statistics), through the C ABI."""
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


def replica_args(ps):
    u = ps.uniforms()
    return u, ps.inverse_cdf()


def test_inverse_cdf_equals_the_oracle_table(ctx):
    """ParticleSystem.swift:23-26: the FP64 table rounded to float."""
    import gargantua_b200 as g

    ps = g.Particles(ctx, 16, seed=1)
    dev = ps.inverse_cdf()
    ref = O.inverse_cdf(1024).astype(np.float32)
    assert np.array_equal(dev.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("seed", [1, 7, 0xDEADBEEF12345678])
def test_seed_is_bit_exact_against_the_replica(ctx, seed):
    import gargantua_b200 as g

    n = 20000
    ps = g.Particles(ctx, n, seed=seed)
    ps.seed_particles()
    dev = ps.read()
    u, cdf = replica_args(ps)
    ref = O.seed32(n, seed, 1, cdf, u.temperatureScale)
    assert np.array_equal(dev.view(np.uint32), ref.view(np.uint32))


def test_step_is_bit_exact_against_the_replica_over_1000_substeps(ctx):
    """The determinism golden's 1000 substeps, against the CPU replica."""
    import gargantua_b200 as g

    n = 30000
    ps = g.Particles(ctx, n, seed=1)
    ps.seed_particles()
    ps.step(500)
    dev = ps.read()
    u, cdf = replica_args(ps)
    ref = O.seed32(n, 1, 1, cdf, u.temperatureScale)
    O.step32(ref, 1, 1, cdf, u.dt, u.alpha, u.temperatureScale, 500)
    respawned = ref.view(np.uint32)[:, 7].sum()
    assert respawned > 0  # the respawn path ran
    mismatch = np.flatnonzero((dev.view(np.uint32) != ref.view(np.uint32)).any(axis=1))
    assert mismatch.size == 0, f"{mismatch.size} particles differ, first {mismatch[:5]}"
    assert ps.checksum() == O.fnv1a(ref)


def test_newtonian_potential_is_bit_exact_against_the_replica(ctx):
    """The second potential of Common.h:32-46 (g = 1/r^2): seed and 1000
    substeps bit-exact against the replica. (The weaker pull plunges few
    particles in that time; the respawn path is covered above.)"""
    import gargantua_b200 as g

    n = 20000
    ps = g.Particles(ctx, n, seed=9, potential=g.types.POTENTIAL_NEWTONIAN)
    ps.seed_particles()
    ps.step(500)
    dev = ps.read()
    u, cdf = replica_args(ps)
    ref = O.seed32(n, 9, g.types.POTENTIAL_NEWTONIAN, cdf, u.temperatureScale)
    O.step32(ref, 9, g.types.POTENTIAL_NEWTONIAN, cdf, u.dt, u.alpha, u.temperatureScale, 500)
    mismatch = np.flatnonzero((dev.view(np.uint32) != ref.view(np.uint32)).any(axis=1))
    assert mismatch.size == 0, f"{mismatch.size} particles differ, first {mismatch[:5]}"
    assert ps.checksum() == O.fnv1a(ref)


def test_step_from_arbitrary_state_matches_replica(ctx):
    """Edge cases: particles on the capture sphere, beyond the escape radius,
    over the speed limit and at the origin's neighbourhood, uploaded through
    gg_particles_write and stepped once."""
    import gargantua_b200 as g

    rng = np.random.default_rng(3)
    n = 4096
    parts = np.zeros((n, 8), np.float32)
    parts[:, :3] = rng.uniform(-70, 70, size=(n, 3))
    parts[:8, :3] = [[2.01, 0, 0], [0, 2.5, 0.1], [61, 0, 0], [0, 0, 59.99], [3.0, 0.1, 0], [1e-3, 0, 0],
                     [-2.03, 0, 0], [30, 30, 30]]
    parts[:, 3:6] = rng.normal(0, 1, size=(n, 3))
    parts[8, 3:6] = [13.0, 0, 0]
    parts[9, 3:6] = [-60.0, 0, 0]
    parts[:, 7] = np.arange(n, dtype=np.uint32).view(np.float32)
    ps = g.Particles(ctx, n, seed=5)
    ps.write(parts)
    ps.step(1)
    dev = ps.read()
    u, cdf = replica_args(ps)
    ref = parts.copy()
    O.step32(ref, 5, 1, cdf, u.dt, u.alpha, u.temperatureScale, 1)
    assert np.array_equal(dev.view(np.uint32), ref.view(np.uint32))


def test_tiny_and_ragged_counts(ctx):
    import gargantua_b200 as g

    for n in (1, 31, 257):
        ps = g.Particles(ctx, n, seed=2)
        ps.seed_particles()
        ps.step(3)
        u, cdf = replica_args(ps)
        ref = O.seed32(n, 2, 1, cdf, u.temperatureScale)
        O.step32(ref, 2, 1, cdf, u.dt, u.alpha, u.temperatureScale, 3)
        assert np.array_equal(ps.read().view(np.uint32), ref.view(np.uint32))


def test_invalid_arguments_are_reported_not_trapped(ctx):
    import gargantua_b200 as g

    with pytest.raises(g.GargantuaError) as e:
        g.Particles(ctx, 0)
    assert e.value.status == 1
    with pytest.raises(g.GargantuaError) as e:
        g.Particles(ctx, 10, potential=7)
    assert e.value.status == 1
    small = g.Context(budget_bytes=1 << 20)
    with pytest.raises(g.GargantuaError) as e:
        g.Particles(small, 1_000_000)
    assert e.value.status == 3  # over budget, refused before allocating
    small.close()


def test_concentrated_seed_profile_is_bit_exact_and_concentrated(ctx):
    """The max preset's contention workload: 70 % of seeds from a power-law
    surface density ~ r^-3, against the replica with the same table."""
    import gargantua_b200 as g

    n = 40000
    ps = g.Particles(ctx, n, seed=5)
    ps.seed_profile(0.7, 3.0)
    table = ps.profile_table()
    assert table[0] == np.float32(6.0) and table[-1] == np.float32(24.0) and np.all(np.diff(table) > 0)
    # The table is Sigma ~ r^-3's inverse CDF: r(u) = (6^-1 + u (24^-1 - 6^-1))^-1.
    u_k = np.arange(1024) / 1023.0
    assert np.allclose(table, 1.0 / (1 / 6 + u_k * (1 / 24 - 1 / 6)), rtol=1e-6)
    ps.seed_particles()
    dev = ps.read()
    u, cdf = replica_args(ps)
    ref = O.seed32_profile(n, 5, 1, cdf, u.temperatureScale, table, 0.7)
    assert np.array_equal(dev.view(np.uint32), ref.view(np.uint32))
    plain = O.seed32(n, 5, 1, cdf, u.temperatureScale)
    r_dev = np.hypot(dev[:, 0], dev[:, 1])
    r_plain = np.hypot(plain[:, 0], plain[:, 1])
    assert np.median(r_dev) < np.median(r_plain) - 1.0  # pulled toward the ISCO
    ps.step(20)  # respawns ignore the profile; the step runs as before
    ps.close()
