"""Failure paths of the server, with the failure made on the host: a fake
device error (gg_server_inject_fault), timeouts, over-budget requests. No
test here faults, traps or hangs the GPU; the context stays usable after
each."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GG_ERR_OVER_BUDGET, GG_ERR_DEVICE, GG_ERR_TIMEOUT, GG_ERR_NOT_READY, GG_ERR_CANCELLED = 3, 4, 5, 6, 9


@pytest.fixture(scope="module")
def world():
    import gargantua_b200 as g

    ctx = g.Context()
    ps = g.Particles(ctx, 100_000, seed=2)
    ps.advance(50, seed_first=True)
    vol = g.Volume(ctx, 64)
    vol.splat(ps, exact=True)
    yield ctx, vol
    ctx.close()


def test_injected_device_error_reaches_every_waiter(world):
    import gargantua_b200 as g

    ctx, vol = world
    server = g.Server(ctx, vol, g.types.SERVE_BATCHED)
    tickets = [server.submit(g.RequestSpec(1920, 1080, 4096, 0.9)) for _ in range(4)]
    g.lib().gg_server_inject_fault(server.handle, GG_ERR_DEVICE)
    for t in tickets:
        with pytest.raises(g.GargantuaError) as e:
            server.wait(t, timeout_s=60.0)
        assert e.value.status == GG_ERR_DEVICE
        assert "Injected fault" in str(e.value)
    with pytest.raises(g.GargantuaError) as e:
        server.submit(g.RequestSpec(64, 64))
    assert e.value.status == GG_ERR_DEVICE
    server.close()
    # The context and a new server still work.
    again = g.Server(ctx, vol, g.types.SERVE_BATCHED)
    _, _, res = again.wait(again.submit(g.RequestSpec(64, 36, 256, 0.0)))
    assert res.status == 0 and res.counters.rays == 64 * 36
    again.close()


def test_wait_times_out_then_completes(world):
    import gargantua_b200 as g

    ctx, vol = world
    server = g.Server(ctx, vol, g.types.SERVE_BATCHED)
    ticket = server.submit(g.RequestSpec(3840, 2160, 4096, 0.9))
    with pytest.raises(g.GargantuaError) as e:
        server.wait(ticket, timeout_s=0.0)
    assert e.value.status == GG_ERR_TIMEOUT
    pixels, _, res = server.wait(ticket, timeout_s=120.0)
    assert res.status == 0 and np.isfinite(pixels.astype(np.float32)).all()
    server.close()


def test_request_larger_than_the_server_is_refused(world):
    import gargantua_b200 as g

    ctx, vol = world
    server = g.Server(ctx, vol, g.types.SERVE_BATCHED, memory_bytes=8 << 20)
    with pytest.raises(g.GargantuaError) as e:
        server.submit(g.RequestSpec(3840, 2160, 256))
    assert e.value.status == GG_ERR_OVER_BUDGET
    _, _, res = server.wait(server.submit(g.RequestSpec(320, 180, 256)))
    assert res.status == 0
    server.close()


def test_pending_requests_can_be_cancelled(world):
    """Request cancellation (host side): with memory for one request at a
    time, the requests queued behind it are withdrawn before admission --
    their waits report GG_ERR_CANCELLED, they never run -- while the one
    already admitted cannot be (GG_ERR_NOT_READY) and completes; the server
    then serves new work."""
    import gargantua_b200 as g

    ctx, vol = world
    spec = g.RequestSpec(1920, 1080, 4096, 0.9)
    one = 1920 * 1080 * 8 + 128 + 8192
    server = g.Server(ctx, vol, g.types.SERVE_BATCHED, memory_bytes=int(one * 1.5))
    tickets = [server.submit(spec) for _ in range(4)]
    cancelled = []
    for t in tickets[1:]:
        try:
            server.cancel(t)
            cancelled.append(t)
        except g.GargantuaError as e:
            assert e.status == GG_ERR_NOT_READY  # admitted before the cancel reached it
    assert cancelled, "at least the last request was still waiting"
    with pytest.raises(g.GargantuaError) as e:
        server.cancel(tickets[0])
    assert e.value.status == GG_ERR_NOT_READY
    for t in tickets:
        if t in cancelled:
            with pytest.raises(g.GargantuaError) as e:
                server.wait(t, timeout_s=60.0)
            assert e.value.status == GG_ERR_CANCELLED
        else:
            _, _, res = server.wait(t, timeout_s=120.0)
            assert res.status == 0 and res.counters.rays == 1920 * 1080
    assert server.totals()["requests"] == len(tickets) - len(cancelled)
    with pytest.raises(g.GargantuaError):
        server.cancel(tickets[0])  # forgotten after its wait
    _, _, res = server.wait(server.submit(g.RequestSpec(320, 180, 256)))
    assert res.status == 0
    server.close()
