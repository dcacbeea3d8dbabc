"""One process per GPU: how the per-frame passes spread over several GPUs.

* Particles (sim.metal:6-79) write only their own slot and draw their random
  numbers from pcg4d keyed on the particle's index (sim.metal:7-8), so the
  index range [0, N) splits into contiguous shards with no exchange: the
  shard of a rank is a particle system whose slot i is global particle
  first_index + i, and it evolves exactly as those slots of the unsharded
  system do.
* The splat (splat.metal:16-88) is the one pass with an exchange. Each rank
  deposits its shard into a full private grid of integer sums; the sums are
  32-bit two's-complement integers, so one element-wise all-reduce (sum) of
  the 6 n^3 words gives the unsharded grid bit for bit, in any order. Every
  rank then resolves the combined grid into its own textures.
* Rays are independent: requests, or the rows of one image, are dealt to
  ranks with no exchange (the march reads the resolved volume only).

On GPUs the all-reduce runs on the sums in device memory over NCCL, ordered
on the context's stream between the bin and the resolve. Under the gloo
backend (CPU process groups) the words pass through the host, widened to 64
bits and folded back to 32, which is the same modular sum.

With reduce="peer" there is no separate all-reduce: every rank opens the
other ranks' sums through CUDA IPC (gg_volume_attach_peers), and the
deposit adds each word into its own grid and into every peer's over NVLink
(peer atomics), so when all ranks' bins are done every grid holds the total.
The ranks only order themselves on the host: a barrier before the bin (no
rank adds into a grid whose owner has not resolved and cleared the previous
frame) and one after it (no rank resolves before every deposit has landed).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import host as H
from . import types as T
from ._lib import check, lib


def shard_bounds(count: int, rank: int, world: int) -> tuple[int, int]:
    """(first_index, count) of rank's contiguous shard of [0, count): the
    first count % world ranks hold one more element."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} is not in a world of {world}")
    base, extra = divmod(count, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def rows_for_rank(height: int, rank: int, world: int) -> tuple[int, int]:
    """[row_begin, row_end) of an image's rows marched by rank."""
    first, n = shard_bounds(height, rank, world)
    return first, first + n


def deal(items: list, rank: int, world: int) -> list:
    """Round-robin share of a request list: rank takes items rank, rank +
    world, ... so every rank sees a similar mix of sizes and spins."""
    return items[rank::world]


def _backend(group) -> str:
    import torch.distributed as dist

    return dist.get_backend(group)


def sum_words_(words, group=None) -> None:
    """In-place modular (2^32) sum of a 1-D int32 tensor over the group.

    CUDA tensors go to the collective as they are (NCCL adds int32 words on
    the device, which wraps in two's complement); CPU tensors are widened to
    int64, summed and folded back to their low 32 bits, so the result is the
    same modular sum whatever the group's size."""
    import torch
    import torch.distributed as dist

    if words.dtype != torch.int32 or words.dim() != 1:
        raise TypeError("sum_words_ takes a 1-D int32 tensor")
    if words.is_cuda:
        dist.all_reduce(words, op=dist.ReduceOp.SUM, group=group)
        return
    wide = words.to(torch.int64) & 0xFFFFFFFF
    dist.all_reduce(wide, op=dist.ReduceOp.SUM, group=group)
    wide &= 0xFFFFFFFF
    words.copy_(torch.where(wide >= 1 << 31, wide - (1 << 32), wide).to(torch.int32))


def attach_peer_sums(vol: H.Volume, group=None) -> int:
    """Exchange the volumes' IPC handles over the group and attach every
    other rank's sums to `vol` (gg_volume_attach_peers); returns the number
    attached. Every rank's volume must have the same size."""
    import torch
    import torch.distributed as dist

    handle = (C.c_uint8 * T.IPC_HANDLE_BYTES)()
    check(lib().gg_volume_ipc_handle(vol.handle, handle))
    mine = torch.tensor(list(bytes(handle)) + [vol.size], dtype=torch.int64)
    if _backend(group) == "nccl":
        mine = mine.cuda(vol.ctx.device)
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    everyone = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(everyone, mine, group=group)
    others = [t.cpu() for r, t in enumerate(everyone) if r != rank]
    if any(int(t[-1]) != vol.size for t in others):
        raise ValueError("every rank's volume must have the same size")
    buf = bytes(b for t in others for b in t[:-1].to(torch.uint8).tolist())
    check(lib().gg_volume_attach_peers(vol.handle, C.c_char_p(buf) if buf else None, len(others)))
    return len(others)


def host_records(em: np.ndarray, mo: np.ndarray, ma: np.ndarray) -> np.ndarray:
    """The three reference arrays (emission u32[2 n^3], momentum i32[3 n^3],
    mass u32[n^3]) as one int32 word array (all emission, then momentum, then
    mass), the unit sum_words_ reduces on the host."""
    return np.concatenate([em.view(np.int32), mo.view(np.int32), ma.view(np.int32)])


def split_records(words: np.ndarray, n3: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    words = np.ascontiguousarray(words, np.int32)
    return (words[:2 * n3].view(np.uint32).copy(), words[2 * n3:5 * n3].copy(), words[5 * n3:].view(np.uint32).copy())


class _DeviceWords:
    """__cuda_array_interface__ over the volume's sums, so torch sees them as
    an int32 tensor without a copy."""

    def __init__(self, ptr: int, words: int):
        self.__cuda_array_interface__ = {"shape": (words,), "typestr": "<i4", "data": (ptr, False), "version": 3,
                                         "strides": None}


def device_sums(vol: H.Volume):
    """The volume's sums as a 1-D int32 CUDA tensor that aliases them."""
    import torch

    ptr, words = C.c_void_p(), C.c_uint64()
    check(lib().gg_volume_sums(vol.handle, C.byref(ptr), C.byref(words)))
    return torch.as_tensor(_DeviceWords(ptr.value, words.value), device=f"cuda:{vol.ctx.device}")


def combine_sums(vol: H.Volume, group=None) -> None:
    """Sum the volume's integer grid over the group, in place.

    NCCL: the all-reduce reads and writes the sums in device memory, issued
    with the context's stream as torch's current stream so it starts after
    the bin kernels and the resolve starts after it. Other backends: the sums
    go through the host."""
    import torch

    if _backend(group) == "nccl":
        stream = torch.cuda.ExternalStream(lib().gg_context_stream(vol.ctx.handle), device=vol.ctx.device)
        with torch.cuda.device(vol.ctx.device), torch.cuda.stream(stream):
            sum_words_(device_sums(vol), group)
        return
    em, mo, ma = vol.read_sums()
    words = torch.from_numpy(host_records(em, mo, ma))
    sum_words_(words, group)
    vol.write_sums(*split_records(words.numpy(), vol.size ** 3))


@dataclass
class Shard:
    rank: int
    world: int
    first_index: int
    count: int


class ShardedDisk:
    """A particle system of `count` particles spread over the ranks of a
    process group, with a full resolved volume on every rank.

    advance() steps each rank's shard with no exchange; splat() bins the
    shard into the rank's private sums, sums them over the group and
    resolves, so every rank ends with the volume one GPU would have made
    from all `count` particles (SplatPass.encode, SplatPass.swift:71-76)."""

    def __init__(self, ctx: H.Context, count: int, size: int, seed: int = 1,
                 potential: int = T.POTENTIAL_PACZYNSKI_WIITA, group=None, rank: int | None = None,
                 world: int | None = None, reduce: str = "collective"):
        if reduce not in ("collective", "peer"):
            raise ValueError(f"reduce is 'collective' or 'peer', not {reduce!r}")
        if rank is None or world is None:
            import torch.distributed as dist

            rank, world = dist.get_rank(group), dist.get_world_size(group)
        first, n = shard_bounds(count, rank, world)
        if n == 0:
            raise ValueError(f"{count} particles leave rank {rank} of {world} without a shard")
        self.shard = Shard(rank, world, first, n)
        self.count = count
        self.group = group
        self.ctx = ctx
        self.particles = H.Particles(ctx, n, seed, potential, first_index=first)
        self.volume = H.Volume(ctx, size)
        self.reduce = reduce
        if reduce == "peer":
            attach_peer_sums(self.volume, group)

    def advance(self, dispatches: int, seed_first: bool = False) -> None:
        self.particles.advance(dispatches, seed_first)

    def bin(self, exact: bool = True) -> None:
        self.volume.bin(self.particles, exact)

    def _barrier(self) -> None:
        import torch.distributed as dist

        self.ctx.synchronize()  # this rank's device work is done before it says so
        dist.barrier(group=self.group)

    def reduce_bin(self, exact: bool = True) -> None:
        """Every rank's shard binned into every rank's sums (reduce="peer"):
        after it, each rank's sums hold the unsharded grid."""
        self._barrier()
        self.bin(exact)
        self._barrier()

    def splat(self, exact: bool = True) -> None:
        if self.reduce == "peer":
            self.reduce_bin(exact)
        else:
            self.bin(exact)
            combine_sums(self.volume, self.group)
        self.volume.resolve()
        self.volume.frame += 1

    def close(self) -> None:
        if self.reduce == "peer" and self.volume.handle:
            # Unmap the other ranks' sums, and let every rank do so, before
            # any rank frees the sums the others have mapped.
            check(lib().gg_volume_attach_peers(self.volume.handle, None, 0))
            self._barrier()
        self.volume.close()
        self.particles.close()
