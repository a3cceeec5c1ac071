"""MSM over a key sharded across GPUs: each rank holds n_r consecutive points of the key and the
matching scalars, runs its own MSM, and the partial XYZZ results are gathered and added on the
host (zkg_xyzz_add_host). One point of 128 (G1) or 256 (G2) bytes per rank crosses the
interconnect, so the sum is the only collective; the result equals the single-GPU MSM of the
whole key. The process group is torch.distributed's (gloo or nccl), one process per GPU.

    lo, hi = shard_bounds(n, rank, world)        # this rank's points [lo, hi)
    words = msm_sharded(gpu, Group.G1, bases_r, scalars_r, hi - lo, c)   # full MSM, on every rank
"""
from __future__ import annotations

import numpy as np

from ._lib import check, lib, u32p
from .gpu import Buffer, Gpu
from .group import Group
from .msm import Msm


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """Rank `rank`'s points [lo, hi) of n, in near-equal consecutive ranges."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def xyzz_sum(group: Group, partials) -> np.ndarray:
    """Sum of XYZZ points (arrays of group.xyzz_words() words) on the host."""
    acc = np.zeros(group.xyzz_words(), dtype=np.uint32)
    for p in partials:
        q = np.ascontiguousarray(p, dtype=np.uint32)
        check(lib().zkg_xyzz_add_host(int(group), acc.ctypes.data_as(u32p), q.ctypes.data_as(u32p),
                                      acc.ctypes.data_as(u32p)))
    return acc


def gather_partials(local: np.ndarray, pg=None) -> list[np.ndarray]:
    """Every rank's partial result, in rank order (torch.distributed all_gather over the CPU)."""
    import torch
    import torch.distributed as dist

    if pg is None and not (dist.is_available() and dist.is_initialized()):
        return [local]
    t = torch.from_numpy(local.view(np.int32).copy())
    out = [torch.empty_like(t) for _ in range(dist.get_world_size(pg))]
    dist.all_gather(out, t, group=pg)
    return [o.numpy().view(np.uint32) for o in out]


def msm_sharded(gpu: Gpu, group: Group, bases: Buffer, scalars: Buffer, n_local: int, c: int, pg=None) -> np.ndarray:
    """This rank's MSM over its shard, then the sum of all ranks' partials (same on every rank)."""
    msm = Msm.for_group(gpu, group, n_local, c)
    local = gpu.read(msm.run(gpu, bases, scalars), group.xyzz_words())
    msm.close()
    return xyzz_sum(group, gather_partials(local, pg))
