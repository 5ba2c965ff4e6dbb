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


# ---------------------------------------------------------------------------
# Independent Poisson solves over GPUs.  A stream of requests (grid size N,
# arrival time) is split without communication: every rank computes the same
# assignment from the same request list -- each request, in arrival order,
# goes to the rank with the least work assigned so far (cost ~ grid points,
# ties to the lower rank) -- and serves only its own share on its own GPU.
# Only the summaries are gathered, for reporting.
# ---------------------------------------------------------------------------
def solve_cost(N):
    """Relative cost of one solve on an N^3 grid (its point count)."""
    return float(N) ** 3


def assign_requests(requests, world, cost=None):
    """Rank of every request (same order): greedy least-loaded assignment in
    arrival order.  Deterministic, so every rank computes the same one."""
    if world < 1:
        raise ValueError('world must be >= 1')
    cost = cost or (lambda r: solve_cost(r.N))
    load = [0.0] * world
    order = sorted(range(len(requests)), key=lambda i: (requests[i].arrival, i))
    ranks = [0] * len(requests)
    for i in order:
        k = min(range(world), key=lambda j: (load[j], j))
        ranks[i] = k
        load[k] += cost(requests[i])
    return ranks


def merge_summaries(summaries):
    """One summary for the whole job from the per-rank ones (each a dict
    from PoissonServer.run plus the completed requests' latencies in
    'latencies_s'): counts add up, the wall time is the slowest rank's, the
    throughput is all completed solves over that time, the latency
    percentiles are over every completed request."""
    import numpy as np
    wall = max(s['wall_s'] for s in summaries)
    lat = np.concatenate([np.asarray(s.get('latencies_s', []), float) for s in summaries])
    completed = sum(s['completed'] for s in summaries)
    out = {'ranks': len(summaries), 'wall_s': wall, 'completed': completed,
           'solves_per_s': completed / wall if wall > 0 else 0.0}
    for k in ('requests', 'rejected', 'expired', 'cancelled', 'failed'):
        out[k] = sum(s.get(k, 0) for s in summaries)
    if lat.size:
        out['p50_ms'] = float(np.percentile(lat, 50) * 1e3)
        out['p99_ms'] = float(np.percentile(lat, 99) * 1e3)
    out['max_residual'] = max(s.get('max_residual', 0.0) for s in summaries)
    return out


class ShardedPoissonService:
    """Serves a request stream on all ranks: each rank runs `server` (a
    PoissonServer on its own GPU, or anything with the same run() method)
    on its share of the requests (assign_requests) and the summaries are
    gathered to every rank (torch.distributed, bookkeeping only).  Without a
    process group it serves everything on this process."""

    def __init__(self, server):
        self.server = server

    def run(self, requests):
        if dist.is_initialized():
            rank, world = dist.get_rank(), dist.get_world_size()
        else:
            rank, world = 0, 1
        ranks = assign_requests(requests, world)
        mine = [r for r, k in zip(requests, ranks) if k == rank]
        local = dict(self.server.run(mine))
        local['latencies_s'] = [r.done - r.arrival for r in mine if r.status == 'ok']
        if world == 1:
            return merge_summaries([local]), mine
        parts = [None] * world
        dist.all_gather_object(parts, local)
        return merge_summaries(parts), mine
