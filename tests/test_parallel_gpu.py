"""Particle shards and the grid all-reduce on one B200.

A shard made with a global index offset must evolve exactly as those slots
of the unsharded system, and the integer grids of two shards must add up to
the unsharded grid bit for bit (exact and stochastic deposits). ShardedDisk
is then run under a one-rank NCCL group (device all-reduce on the context's
stream) and a one-rank gloo group (through the host): both must give the
volume one unsharded splat gives. More than one rank needs more GPUs than a
test here has; the multi-rank logic runs on the CPU in test_parallel.py.
The peer-memory reduce runs as two processes sharing the one GPU: each opens
the other's sums through CUDA IPC and deposits into both, ordered by gloo
barriers on the host (no kernel waits on another process's).
"""
import os
import socket
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COUNT = 300_001
SIZE = 64
SEED = 9


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.fixture(scope="module")
def ctx():
    import gargantua_b200 as g

    c = g.Context()
    yield c
    c.close()


def _shards(ctx, world=2):
    import gargantua_b200 as g
    from gargantua_b200 import parallel as P

    out = []
    for r in range(world):
        first, n = P.shard_bounds(COUNT, r, world)
        out.append(g.Particles(ctx, n, SEED, first_index=first))
    return out


def test_shards_match_unsharded_slots(ctx):
    import gargantua_b200 as g

    whole = g.Particles(ctx, COUNT, SEED)
    whole.advance(50, seed_first=True)
    shards = _shards(ctx)
    for s in shards:
        s.advance(50, seed_first=True)
    got = np.concatenate([s.read() for s in shards])
    ref = whole.read()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    for s in shards:
        s.close()
    whole.close()


@pytest.mark.parametrize("exact", [True, False])
def test_shard_grids_sum_to_the_unsharded_grid(ctx, exact):
    import torch

    import gargantua_b200 as g
    from gargantua_b200 import parallel as P

    whole = g.Particles(ctx, COUNT, SEED)
    whole.advance(30, seed_first=True)
    ref_vol = g.Volume(ctx, SIZE)
    ref_vol.bin(whole, exact, frame=5)
    ref = ref_vol.read_sums()
    shards = _shards(ctx)
    vols = []
    for s in shards:
        s.advance(30, seed_first=True)
        v = g.Volume(ctx, SIZE)
        v.bin(s, exact, frame=5)
        vols.append(v)
    ctx.synchronize()
    total = P.device_sums(vols[0]) + P.device_sums(vols[1])  # int32 adds wrap on the device
    torch.cuda.synchronize()
    P.device_sums(vols[0]).copy_(total)
    torch.cuda.synchronize()
    got = vols[0].read_sums()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    assert ref[2].any()
    for v in vols + [ref_vol]:
        v.close()
    for s in shards + [whole]:
        s.close()


@pytest.mark.parametrize("backend", ["nccl", "gloo"])
def test_sharded_disk_one_rank_matches_plain_splat(ctx, backend):
    import torch
    import torch.distributed as dist

    import gargantua_b200 as g
    from gargantua_b200 import parallel as P

    torch.cuda.set_device(0)
    dist.init_process_group(backend, init_method=f"tcp://127.0.0.1:{_port()}", rank=0, world_size=1)
    try:
        disk = P.ShardedDisk(ctx, COUNT, SIZE, seed=SEED)
        disk.advance(40, seed_first=True)
        disk.splat(exact=True)
        disk.splat(exact=False)
        ctx.synchronize()
        em, vel = disk.volume.read()
        whole = g.Particles(ctx, COUNT, SEED)
        whole.advance(40, seed_first=True)
        vol = g.Volume(ctx, SIZE)
        vol.splat(whole, exact=True)
        vol.splat(whole, exact=False)
        rem, rvel = vol.read()
        assert np.array_equal(em.view(np.uint16), rem.view(np.uint16))
        assert np.array_equal(vel.view(np.uint16), rvel.view(np.uint16))
        assert disk.volume.frame == vol.frame == 2
        disk.close()
        vol.close()
        whole.close()
    finally:
        dist.destroy_process_group()


def test_peer_attach_refusals(ctx):
    """gg_volume_attach_peers refuses more than GG_MAX_PEERS handles before
    opening any, leaving the volume unattached (it still bins like a plain
    volume); count 0 detaches nothing harmlessly; the volume exports a
    handle."""
    import ctypes as C

    import gargantua_b200 as g
    from gargantua_b200._lib import check

    vol = g.Volume(ctx, 16)
    lib = g.lib()
    handles = bytes(64 * (g.types.MAX_PEERS + 1))
    with pytest.raises(g.GargantuaError):
        check(lib.gg_volume_attach_peers(vol.handle, C.c_char_p(handles), g.types.MAX_PEERS + 1))
    check(lib.gg_volume_attach_peers(vol.handle, None, 0))
    handle = (C.c_uint8 * g.types.IPC_HANDLE_BYTES)()
    check(lib.gg_volume_ipc_handle(vol.handle, handle))
    assert any(bytes(handle))
    ps = g.Particles(ctx, 5000, SEED)
    ps.advance(5, seed_first=True)
    vol.bin(ps, exact=True)
    assert vol.read_sums()[2].any()
    ps.close()
    vol.close()


def _peer_rank(rank: int, world: int, port: int, outdir: str) -> None:
    """One rank of the peer-memory reduce on GPU 0: its shard deposited into
    every rank's sums (gg_volume_attach_peers), then two splats through
    ShardedDisk.splat. Writes its sums and textures to outdir."""
    import datetime

    import torch.distributed as dist

    import gargantua_b200 as g
    from gargantua_b200 import parallel as P

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        ctx = g.Context(0)
        disk = P.ShardedDisk(ctx, COUNT, SIZE, seed=SEED, reduce="peer")
        disk.advance(40, seed_first=True)
        disk.reduce_bin(exact=True)
        em, mo, ma = disk.volume.read_sums()
        np.savez(os.path.join(outdir, f"sums{rank}.npz"), em=em, mo=mo, ma=ma)
        disk.volume.clear()
        textures = []
        for exact in (False, True):  # frames 0 and 1: the resolve clears, the barriers order the ranks
            disk.splat(exact=exact)
            textures.extend(disk.volume.read())
        np.savez(os.path.join(outdir, f"tex{rank}.npz"), *textures)
        disk.close()
        ctx.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_peer_memory_reduce_matches_the_unsharded_grid(ctx, tmp_path):
    """reduce="peer": two ranks' deposits land in both grids over peer memory
    (CUDA IPC), and each rank's sums and resolved volume equal one unsharded
    splat's, exact and stochastic."""
    import torch.multiprocessing as mp

    import gargantua_b200 as g

    procs = mp.start_processes(_peer_rank, args=(2, _port(), str(tmp_path)), nprocs=2, start_method="spawn",
                               join=False)
    deadline = time.time() + 300
    while not procs.join(timeout=5):
        if time.time() > deadline:
            for p in procs.processes:
                p.kill()
            pytest.fail("the two ranks did not finish in 300 s")
    whole = g.Particles(ctx, COUNT, SEED)
    whole.advance(40, seed_first=True)
    vol = g.Volume(ctx, SIZE)
    vol.bin(whole, exact=True)
    ref = vol.read_sums()
    vol.clear()
    ref_tex = []
    for exact in (False, True):
        vol.splat(whole, exact=exact)
        ref_tex.extend(vol.read())
    assert ref[2].any()
    for rank in range(2):
        got = np.load(tmp_path / f"sums{rank}.npz")
        for name, r in zip(("em", "mo", "ma"), ref):
            assert np.array_equal(got[name], r), (rank, name)
        tex = np.load(tmp_path / f"tex{rank}.npz")
        for k, r in enumerate(ref_tex):
            assert np.array_equal(tex[f"arr_{k}"].view(np.uint16), r.view(np.uint16)), (rank, k)
    vol.close()
    whole.close()
