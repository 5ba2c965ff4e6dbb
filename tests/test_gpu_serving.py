"""Many independent Poisson solves: one-launch batches of uneven grids and the
continuous-batching server.  Every result must equal the same request solved
alone (bit for bit: solves share no buffers and every reduction has a fixed
order), and agree with the CPU oracle (same V-cycle count, 1e-10 max-abs)."""
import numpy as np
import pytest

from oracle import geometry as G
from oracle import poisson as OP

pytestmark = pytest.mark.gpu
H = 0.2 / G.BOHR


def oracle_solve(N, rho_np):
    og = G.Grid((N,) * 3, (N * H,) * 3, 0)
    ps = OP.PoissonSolver(3, 'J', 2e-10)
    ps.set_grid_descriptor(og)
    ps.initialize()
    phi = np.zeros(rho_np.shape)
    n = ps.solve(phi, rho_np)
    return phi, n


def test_batch_of_uneven_grids(cuda):
    import torch
    from gpaw_b200.poisson import PoissonSolver
    from gpaw_b200.serving import PoissonBatch, grid_for, pair_density
    sizes = [16, 24, 32, 20, 24]
    solvers, rhos, phis = [], [], []
    for i, N in enumerate(sizes):
        gd = grid_for(N, H, device=cuda)
        ps = PoissonSolver(3, 'J', 2e-10)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        solvers.append(ps)
        rho = pair_density(gd, 100 + i)
        rhos.append(rho)
        phis.append(torch.zeros_like(rho))
    batch = PoissonBatch(solvers)
    res = batch.solve(phis, rhos)
    for i, N in enumerate(sizes):
        # alone, on a fresh solver
        ps = PoissonSolver(3, 'J', 2e-10)
        ps.set_grid_descriptor(grid_for(N, H, device=cuda))
        phi = torch.zeros_like(rhos[i])
        n = ps.solve(phi, rhos[i])
        assert n == res[i][0]
        assert torch.equal(phi, phis[i]), 'batch result differs from the solve alone'
        phi_o, n_o = oracle_solve(N, rhos[i].cpu().numpy())
        assert n == n_o
        assert np.abs(phi.cpu().numpy() - phi_o).max() < 1e-10
    # a second launch of the same batch gives the same results
    phis2 = [torch.zeros_like(r) for r in rhos]
    res2 = batch.solve(phis2, rhos)
    assert [r[0] for r in res2] == [r[0] for r in res]
    assert all(torch.equal(a, b) for a, b in zip(phis, phis2))


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_server_alone_vs_mix(cuda, precision):
    import torch
    from gpaw_b200.serving import PoissonServer, Request, grid_for, pair_density
    sizes = [16, 32, 24, 48, 16, 32, 24, 20, 48, 16]
    rhos = [pair_density(grid_for(N, H, device=cuda), 7 + i) for i, N in enumerate(sizes)]
    torch.cuda.synchronize()

    def serve(max_inflight, arrivals):
        srv = PoissonServer(H, precision=precision, max_inflight=max_inflight, nstreams=8,
                            device=cuda, keep_results=True)
        reqs = [Request(i, N, arrivals[i], rhos[i]) for i, N in enumerate(sizes)]
        stats = srv.run(reqs)
        torch.cuda.synchronize()
        return reqs, stats

    mix, s_mix = serve(8, [0.0] * len(sizes))               # all at once, overlapping
    alone, s_alone = serve(1, [0.0] * len(sizes))           # one at a time
    staggered, _ = serve(4, [0.002 * i for i in range(len(sizes))])  # arriving over time
    assert s_mix['completed'] == len(sizes) and s_alone['completed'] == len(sizes)
    for a, b, c in zip(mix, alone, staggered):
        assert a.status == 'ok' and a.niter == b.niter == c.niter
        assert torch.equal(a.phi, b.phi) and torch.equal(a.phi, c.phi)
        assert a.error <= 2e-10
    # one request against the oracle
    k = 3
    phi_o, n_o = oracle_solve(sizes[k], rhos[k].cpu().numpy())
    tol = 1e-10 if precision == 'fp64' else 1e-9
    assert np.abs(mix[k].phi.cpu().numpy() - phi_o).max() < tol


def test_server_memory_budget_rejects(cuda):
    import torch
    from gpaw_b200.serving import PoissonServer, Request, grid_for, pair_density
    rho = pair_density(grid_for(32, H, device=cuda), 3)
    torch.cuda.synchronize()
    srv = PoissonServer(H, budget_bytes=1 << 20, device=cuda)  # 1 MiB: too small
    reqs = [Request(0, 32, 0.0, rho)]
    stats = srv.run(reqs)
    assert stats['rejected'] == 1 and reqs[0].status.startswith('rejected')
