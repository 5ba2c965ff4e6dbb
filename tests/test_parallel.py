"""The N > 1 path on CPU: band sharding, gather and max-over-ranks timing
with world_size 2 over gloo (no GPU).  The per-rank compute is the oracle
stencil standing in for the GPU apply; the sharded, gathered result must
equal the unsharded one."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from gpaw_b200.parallel import shard


def test_shard_covers_every_unit_once():
    for n in (0, 1, 5, 512, 513):
        for world in (1, 2, 3, 8):
            spans = [shard(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, result_dir):
    import datetime
    import torch.distributed as dist
    from oracle import geometry as G
    from oracle import kernels as K
    from gpaw_b200.parallel import gather_shards, max_over_ranks, shard
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        gd = G.Grid((10, 8, 12), (3.0, 2.4, 3.6), 1)
        c, o = G.laplace_stencil(gd, -0.5, 3)
        rng = np.random.default_rng(0)
        bands = rng.standard_normal((5,) + tuple(gd.n_c)) + 1j * rng.standard_normal((5,) + tuple(gd.n_c))
        ph = G.bloch_phases(gd, (0.25, 0, 0))
        a, b = shard(len(bands), rank, world)
        local = K.fd_apply(c, o, gd.pbc_c, bands[a:b], ph)
        full = gather_shards(torch.from_numpy(local), len(bands)).numpy()
        ref = K.fd_apply(c, o, gd.pbc_c, bands, ph)
        ok = np.array_equal(full, ref)
        t = max_over_ranks(0.5 + rank)  # each rank's "time"; all must see the max
        np.save(os.path.join(result_dir, 'rank%d.npy' % rank), np.array([ok, t == 0.5 + world - 1]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo(tmp_path):
    world = 2
    port = _free_port()
    ctx = mp.get_context('spawn')
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        ok, tmax = np.load(tmp_path / ('rank%d.npy' % r))
        assert ok and tmax


class _Req:
    def __init__(self, rid, N, arrival):
        self.rid, self.N, self.arrival = rid, N, arrival
        self.status = self.done = self.result = None


def test_assign_requests_balances_and_covers():
    from gpaw_b200.parallel import assign_requests, solve_cost
    rng = np.random.default_rng(1)
    sizes = rng.choice([32, 48, 64, 96, 128, 160], 1000)
    reqs = [_Req(i, int(N), float(i) * 1e-3) for i, N in enumerate(sizes)]
    for world in (1, 2, 3, 8):
        ranks = assign_requests(reqs, world)
        assert ranks == assign_requests(reqs, world)  # deterministic
        assert set(ranks) == set(range(world))
        load = [sum(solve_cost(r.N) for r, k in zip(reqs, ranks) if k == j) for j in range(world)]
        assert max(load) - min(load) <= solve_cost(160)  # within the largest request
    with pytest.raises(ValueError):
        assign_requests(reqs, 0)


class _OracleServer:
    """Host stand-in for a PoissonServer: solves each request's small
    zero-boundary grid with the oracle V-cycle."""

    def run(self, requests):
        import time
        from oracle import geometry as G
        from oracle import poisson as OP
        t0 = time.perf_counter()
        for r in requests:
            og = G.Grid((r.N,) * 3, (r.N * 0.4,) * 3, 0)
            rng = np.random.default_rng(r.rid)
            rho = rng.standard_normal(tuple(og.n_c))
            ps = OP.PoissonSolver(1, 'J', 1e-8)
            ps.set_grid_descriptor(og)
            ps.initialize()
            phi = np.zeros(tuple(og.n_c))
            ps.solve(phi, rho - rho.mean())
            r.result = float(np.abs(phi).sum())
            r.status = 'ok'
            r.done = r.arrival + 1e-3 * (r.rid + 1)
        wall = time.perf_counter() - t0 + 1e-6
        return {'requests': len(requests), 'completed': len(requests), 'rejected': 0,
                'wall_s': wall, 'max_residual': 0.0}


def _serve_rank(rank, world, port, result_dir):
    import datetime
    import torch.distributed as dist
    from gpaw_b200.parallel import ShardedPoissonService
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        reqs = [_Req(i, N, 0.002 * i) for i, N in enumerate([8, 16, 8, 12, 16, 8, 12, 8, 16])]
        summary, mine = ShardedPoissonService(_OracleServer()).run(reqs)
        np.save(os.path.join(result_dir, 'serve%d.npy' % rank),
                np.array([[r.rid, r.result] for r in mine]))
        np.save(os.path.join(result_dir, 'summary%d.npy' % rank),
                np.array([summary['completed'], summary['requests'], summary['p50_ms']]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_serve_disjoint_shares(tmp_path):
    """Two gloo ranks serve one request stream: every request once, on one
    rank; the merged summary counts all of them on both ranks; each result
    equals the same request served by one process."""
    from gpaw_b200.parallel import ShardedPoissonService
    world = 2
    port = _free_port()
    ctx = mp.get_context('spawn')
    procs = [ctx.Process(target=_serve_rank, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    got = np.concatenate([np.load(tmp_path / ('serve%d.npy' % r)) for r in range(world)])
    assert sorted(got[:, 0].astype(int)) == list(range(9))
    assert all(len(np.load(tmp_path / ('serve%d.npy' % r))) > 0 for r in range(world))
    reqs = [_Req(i, N, 0.002 * i) for i, N in enumerate([8, 16, 8, 12, 16, 8, 12, 8, 16])]
    single, _ = ShardedPoissonService(_OracleServer()).run(reqs)
    by_id = {int(i): v for i, v in got}
    assert all(by_id[r.rid] == r.result for r in reqs)
    for r in range(world):
        completed, nreq, p50 = np.load(tmp_path / ('summary%d.npy' % r))
        assert completed == 9 and nreq == 9
        assert abs(p50 - single['p50_ms']) < 1e-9
