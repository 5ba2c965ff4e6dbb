"""Sharding of independent units (bands, Poisson solves) over GPUs.

Bands of a band-batched operator and independent Poisson solves need no
communication, so N GPUs simply take contiguous shares of the units; the only
collectives are for bookkeeping (the maximum time over ranks, gathering
results for checks).  One process per GPU; torch.distributed supplies the
process group (NCCL on GPUs, gloo on CPU for tests).
"""
import torch
import torch.distributed as dist


def shard(n, rank, world):
    """Contiguous [start, stop) share of n units for `rank` of `world`;
    the first n % world ranks take one extra unit."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError('bad rank %d of %d' % (rank, world))
    base, extra = divmod(int(n), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _device_for_backend():
    if dist.is_initialized() and dist.get_backend() == 'nccl':
        return torch.device('cuda', torch.cuda.current_device())
    return torch.device('cpu')


def max_over_ranks(x):
    """Maximum of a float over all ranks (x itself without a process group)."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x):
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_shards(local, n_total):
    """All-gather the per-rank shards (leading axis = units) of a tensor that
    was split with shard(); every rank gets the full (n_total, ...) tensor."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return local
    world = dist.get_world_size()
    dev = _device_for_backend()
    sizes = [shard(n_total, r, world) for r in range(world)]
    width = max(b - a for a, b in sizes)
    buf = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=dev)
    buf[:local.shape[0]] = local.to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    return torch.cat([p[:b - a] for p, (a, b) in zip(parts, sizes)], 0)
