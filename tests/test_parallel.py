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
