"""Multi-process host logic of gargantua_b200.parallel on the CPU (gloo).

Two ranks each seed, step and deposit their shard of a particle system with
the FP32 replicas of the kernels (the device kernels take the same global
index offset), then sum their integer grids with sum_words_. The result must
equal the unsharded system's grid bit for bit, and each shard's particles
must equal the matching slots of the unsharded system. Modular (2^32)
wrap-around of the sums is checked on words chosen to overflow.
"""
import os
import socket

import numpy as np
import pytest

from gargantua_b200 import parallel as P

N_PARTICLES = 6001  # odd: the shards differ in size
GRID = 24
SEED = 0x1234_5678_9ABC
DISPATCHES = 40
TEMPERATURE_SCALE = 7.5e3
DT, ALPHA = 0.1, 0.003


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _system(first: int, count: int):
    import oracle_ffi as O

    cdf = O.inverse_cdf(1024).astype(np.float32)
    parts = O.seed32(count, SEED, 1, cdf, TEMPERATURE_SCALE, first_index=first)
    O.step32(parts, SEED, 1, cdf, DT, ALPHA, TEMPERATURE_SCALE, DISPATCHES, threads=1, first_index=first)
    return parts


def _grids(parts, first: int):
    import oracle_ffi as O

    out = []
    for frame, exact in ((3, False), (4, True)):
        em, mo, ma = O.deposit32(parts, GRID, frame, exact, SEED, first_index=first)
        out.append(P.host_records(em, mo, ma))
    return out


def _rank_main(rank: int, world: int, port: int, outdir: str) -> None:
    import torch
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        first, count = P.shard_bounds(N_PARTICLES, rank, world)
        parts = _system(first, count)
        np.save(os.path.join(outdir, f"parts{rank}.npy"), parts)
        for k, words in enumerate(_grids(parts, first)):
            t = torch.from_numpy(words.copy())
            P.sum_words_(t)
            np.save(os.path.join(outdir, f"grid{k}_{rank}.npy"), t.numpy())
        # Words whose sum wraps: 0xFFFFFFF0 + 0x20 = 0x10 (mod 2^32), and
        # INT32_MAX + 1 = INT32_MIN.
        wrap = torch.tensor([-16 if rank == 0 else 32, 2**31 - 1 if rank == 0 else 1, rank], dtype=torch.int32)
        P.sum_words_(wrap)
        np.save(os.path.join(outdir, f"wrap{rank}.npy"), wrap.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def two_ranks(tmp_path_factory):
    import torch.multiprocessing as mp

    outdir = str(tmp_path_factory.mktemp("ranks"))
    mp.start_processes(_rank_main, args=(2, _free_port(), outdir), nprocs=2, start_method="spawn", join=True)
    return outdir


def test_shard_bounds_partition_the_range():
    for count in (0, 1, 7, 1000, 1_000_003):
        for world in (1, 2, 3, 8):
            spans = [P.shard_bounds(count, r, world) for r in range(world)]
            assert spans[0][0] == 0
            for (a, n), (b, _) in zip(spans, spans[1:]):
                assert a + n == b
            assert spans[-1][0] + spans[-1][1] == count
            sizes = [n for _, n in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        P.shard_bounds(10, 2, 2)


def test_sharded_disk_refuses_an_unknown_reduce():
    """reduce is "collective" (NCCL or the host) or "peer" (the deposit over
    peer memory); anything else is refused before a particle is made."""
    with pytest.raises(ValueError):
        P.ShardedDisk(None, 10, 8, rank=0, world=1, reduce="ring")


def test_rows_and_deal_cover_everything_once():
    rows = [P.rows_for_rank(1080, r, 8) for r in range(8)]
    assert rows[0][0] == 0 and rows[-1][1] == 1080
    assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
    items = list(range(37))
    dealt = [P.deal(items, r, 4) for r in range(4)]
    assert sorted(sum(dealt, [])) == items


def test_host_records_round_trip():
    rng = np.random.default_rng(5)
    n3 = 5 ** 3
    em = rng.integers(0, 2**32, 2 * n3, dtype=np.uint64).astype(np.uint32)
    mo = rng.integers(-2**31, 2**31, 3 * n3).astype(np.int32)
    ma = rng.integers(0, 2**32, n3, dtype=np.uint64).astype(np.uint32)
    a, b, c = P.split_records(P.host_records(em, mo, ma), n3)
    assert np.array_equal(a, em) and np.array_equal(b, mo) and np.array_equal(c, ma)


def test_shards_reproduce_the_unsharded_particles(two_ranks):
    whole = _system(0, N_PARTICLES)
    got = np.concatenate([np.load(os.path.join(two_ranks, f"parts{r}.npy")) for r in range(2)])
    assert got.shape == whole.shape
    assert np.array_equal(got.view(np.uint32), whole.view(np.uint32))


def test_summed_shard_grids_equal_the_unsharded_grid(two_ranks):
    whole = _system(0, N_PARTICLES)
    for k, ref in enumerate(_grids(whole, 0)):
        for r in range(2):
            got = np.load(os.path.join(two_ranks, f"grid{k}_{r}.npy"))
            assert np.array_equal(got, ref), (k, r)
        assert ref.any()


def test_sum_words_wraps_modulo_two_to_the_32(two_ranks):
    for r in range(2):
        got = np.load(os.path.join(two_ranks, f"wrap{r}.npy"))
        assert got.tolist() == [16, -2**31, 1]
