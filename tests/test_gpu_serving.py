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


def make_batch(cuda, sizes, relax='J', precision='fp64', seed=300):
    import torch
    from gpaw_b200.poisson import PoissonSolver
    from gpaw_b200.serving import PoissonBatch, grid_for, pair_density
    solvers, rhos = [], []
    for i, N in enumerate(sizes):
        ps = PoissonSolver(3, relax, 2e-10, precision=precision)
        ps.set_grid_descriptor(grid_for(N, H, device=cuda))
        ps.initialize()
        solvers.append(ps)
        rhos.append(pair_density(grid_for(N, H, device=cuda), seed + i))
    return PoissonBatch(solvers), solvers, rhos


def solve_alone(cuda, N, rho, relax='J', precision='fp64', eps=2e-10):
    import torch
    from gpaw_b200.poisson import PoissonSolver
    from gpaw_b200.serving import grid_for
    ps = PoissonSolver(3, relax, eps, precision=precision)
    ps.set_grid_descriptor(grid_for(N, H, device=cuda))
    phi = torch.zeros_like(rho)
    n = ps.solve(phi, rho)
    return phi, n


@pytest.mark.parametrize('relax', ['J', 'GS'])
def test_grouped_batch_matches_alone(cuda, relax):
    """Small solvers of one structure are grouped: one launch per V-cycle
    step over all their grids.  Here 24^3 (three coarsenings) and 32^3 (four)
    form two groups; 20^3 (two coarsenings) and 48^3 (above the 32768-point
    default) run alone beside them.  Every result equals the solve alone bit
    for bit, and the oracle's (Jacobi: same V-cycle count, 1e-10)."""
    import torch
    sizes = [24, 32, 20, 24, 48, 32]
    batch, solvers, rhos = make_batch(cuda, sizes, relax)
    assert batch.grouped == 4
    phis = [torch.zeros_like(r) for r in rhos]
    res = batch.solve(phis, rhos)
    for i, N in enumerate(sizes):
        phi, n = solve_alone(cuda, N, rhos[i], relax)
        assert n == res[i][0], (N, n, res[i][0])
        assert res[i][1] <= 2e-10
        assert torch.equal(phi, phis[i]), N
        if relax == 'J' and N <= 48:
            phi_o, n_o = oracle_solve(N, rhos[i].cpu().numpy())
            assert n == n_o
            assert np.abs(phis[i].cpu().numpy() - phi_o).max() < 1e-10
    phis2 = [torch.zeros_like(r) for r in rhos]
    res2 = batch.solve(phis2, rhos)
    assert [r[0] for r in res2] == [r[0] for r in res]
    assert all(torch.equal(a, b) for a, b in zip(phis, phis2))


_LARGE_GROUP = r"""
import sys, torch
sys.path.insert(0, 'tests')
from test_gpu_serving import make_batch, solve_alone
for relax in ('J', 'GS'):
    sizes = [48, 80, 64]
    batch, solvers, rhos = make_batch('cuda', sizes, relax, seed=700)
    assert batch.grouped == 3, batch.grouped
    phis = [torch.zeros_like(r) for r in rhos]
    res = batch.solve(phis, rhos)
    for i, N in enumerate(sizes):
        phi, n = solve_alone('cuda', N, rhos[i], relax)
        assert n == res[i][0], (relax, N, n, res[i][0])
        d = float((phi - phis[i]).abs().max()) / float(phi.abs().max())
        assert d < 1e-12, (relax, N, d)
print('ok')
"""


def test_grouped_batch_with_large_grids(cuda):
    """GFD_GROUP_MAX_POINTS raises the size limit: 48^3 to 80^3 join the
    group; 80^3 runs one-thread-per-point kernels where alone it marches, so
    it matches the solve alone to rounding (1e-12 relative), same count."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, GFD_GROUP_MAX_POINTS='100000000')
    r = subprocess.run([sys.executable, '-c', _LARGE_GROUP], cwd=root, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and 'ok' in r.stdout, r.stdout + r.stderr


def test_grouped_batch_charged_and_maxiter(cuda):
    """Per-solve outcomes inside one grouped launch: a charged zero-boundary
    request whose solver has not loaded the compensating Gaussian is refused
    (NotImplementedError, phi untouched) without touching the others; once
    that solver loads it, the same launch solves the charged request as a
    solve alone does.  maxiter stops every solve at that count
    (PoissonConvergenceError)."""
    import torch
    from gpaw_b200.errors import PoissonConvergenceError
    sizes = [32, 32, 32]
    batch, solvers, rhos = make_batch(cuda, sizes, seed=410)
    assert batch.grouped == 3
    rhos[1] = rhos[1] + 1e-3          # net charge
    phis = [torch.zeros_like(r) for r in rhos]
    with pytest.raises(NotImplementedError):
        batch.solve(phis, rhos)
    assert not phis[1].any()
    for i in (0, 2):
        n, err = solvers[i].result()
        phi, n_alone = solve_alone(cuda, sizes[i], rhos[i])
        assert n == n_alone and err <= 2e-10
        assert torch.equal(phi, phis[i])
    solvers[1].load_gauss()
    phis = [torch.zeros_like(r) for r in rhos]
    res = batch.solve(phis, rhos)
    phi, n_alone = solve_alone(cuda, sizes[1], rhos[1])
    assert res[1][0] == n_alone and torch.equal(phi, phis[1])
    phi_o, n_o = oracle_solve(sizes[1], rhos[1].cpu().numpy())
    assert n_alone == n_o and np.abs(phi.cpu().numpy() - phi_o).max() < 1e-10
    rhos[1] = rhos[1] - rhos[1].mean()
    phis = [torch.zeros_like(r) for r in rhos]
    with pytest.raises(PoissonConvergenceError):
        batch.solve(phis, rhos, maxiter=2)
    for s in solvers:
        with pytest.raises(PoissonConvergenceError):
            s.result()
        assert s.niter == 2


@pytest.mark.parametrize('group', [True, False])
def test_batch_unused_slots(cuda, group):
    """A batch captured once serves fewer requests than it has slots: unused
    slots (None) run nothing, and the used ones give the results alone."""
    import torch
    from gpaw_b200.serving import PoissonBatch
    sizes = [32, 32, 32, 32]
    _, solvers, rhos = make_batch(cuda, sizes, seed=610)
    batch = PoissonBatch(solvers, group=group)
    assert batch.grouped == (4 if group else 0)
    for used in ([0, 2], [3], [0, 1, 2, 3]):
        phis = [torch.zeros_like(r) if i in used else None for i, r in enumerate(rhos)]
        res = batch.solve(phis, [r if i in used else None for i, r in enumerate(rhos)])
        for i in range(4):
            if i not in used:
                assert res[i] is None
                continue
            phi, n = solve_alone(cuda, 32, rhos[i])
            assert res[i][0] == n and torch.equal(phi, phis[i])
    with pytest.raises(ValueError):
        batch.solve([None] * 4, [None] * 4)


def test_mixed_precision_batch_uses_branches(cuda):
    import torch
    sizes = [24, 32]
    batch, solvers, rhos = make_batch(cuda, sizes, precision='mixed', seed=500)
    assert batch.grouped == 0
    phis = [torch.zeros_like(r) for r in rhos]
    res = batch.solve(phis, rhos)
    for i, N in enumerate(sizes):
        phi, n = solve_alone(cuda, N, rhos[i], precision='mixed')
        assert n == res[i][0] and torch.equal(phi, phis[i])


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_server_alone_vs_mix(cuda, precision):
    import torch
    from gpaw_b200.serving import PoissonServer, Request, grid_for, pair_density
    sizes = [16, 32, 24, 48, 16, 32, 24, 20, 48, 16]
    rhos = [pair_density(grid_for(N, H, device=cuda), 7 + i) for i, N in enumerate(sizes)]
    torch.cuda.synchronize()

    def serve(max_inflight, arrivals, slots=8):
        srv = PoissonServer(H, precision=precision, max_inflight=max_inflight, nstreams=8,
                            device=cuda, keep_results=True, slots=slots)
        reqs = [Request(i, N, arrivals[i], rhos[i]) for i, N in enumerate(sizes)]
        stats = srv.run(reqs)
        torch.cuda.synchronize()
        return reqs, stats

    mix, s_mix = serve(8, [0.0] * len(sizes))               # all at once, overlapping
    alone, s_alone = serve(1, [0.0] * len(sizes), slots=1)  # one at a time
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


def test_server_deadline_and_cancel(cuda):
    """Host-side request failures: with one launch in flight at a time, the
    requests queued behind it with a zero admission deadline expire; a
    request cancelled before it arrives never runs, one cancelled right after
    the start is dropped whether it still waits or already runs (its result
    discarded); the other requests finish and equal their solves alone."""
    import torch
    from gpaw_b200.serving import PoissonServer, Request, grid_for, pair_density
    sizes = [64] * 8
    rhos = [pair_density(grid_for(N, H, device=cuda), 50 + i) for i, N in enumerate(sizes)]
    torch.cuda.synchronize()
    srv = PoissonServer(H, max_inflight=1, nstreams=2, device=cuda, keep_results=True, slots=1)
    reqs = [Request(i, N, 0.0, rhos[i]) for i, N in enumerate(sizes)]
    for r in reqs[5:7]:
        r.deadline = 0.0                      # must be admitted at once: they cannot be
    reqs[3].arrival, reqs[3].cancel_at = 0.5, 0.0   # cancelled before it arrives
    reqs[1].cancel_at = 1e-4                  # cancelled right after the start
    stats = srv.run(reqs)
    assert [r.status for r in reqs[5:7]] == ['expired', 'expired']
    assert reqs[3].status == 'cancelled' and reqs[3].admit is None
    assert reqs[1].status == 'cancelled' and reqs[1].phi is None
    assert stats['expired'] == 2 and stats['cancelled'] == 2
    for i in (0, 2, 4, 7):
        assert reqs[i].status == 'ok'
        phi, n = solve_alone(cuda, sizes[i], rhos[i])
        assert reqs[i].niter == n and torch.equal(reqs[i].phi, phi)


def test_server_device_allocation_failure(cuda):
    """A failing device allocation (planned through gfd_test_fail_alloc, on
    the host): the pod cannot be created, the request is rejected with
    nothing in flight, and the server goes on to serve the next requests.
    The same planned failure surfaces as MemoryError from the solver, the
    relaxation scratch and the preconditioner."""
    import torch
    from gpaw_b200 import _lib
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.poisson import PoissonSolver
    from gpaw_b200.preconditioner import Preconditioner
    from gpaw_b200.serving import PoissonServer, Request, grid_for, pair_density
    rho = pair_density(grid_for(32, H, device=cuda), 5)
    torch.cuda.synchronize()
    srv = PoissonServer(H, device=cuda, keep_results=True, slots=1)
    try:
        assert _lib.lib.gfd_test_fail_alloc(1) == 0
        stats = srv.run([Request(0, 32, 0.0, rho)])
        assert stats['rejected'] == 1 and srv.alloc_failures == 1
        reqs = [Request(1, 32, 0.0, rho), Request(2, 32, 0.0, rho)]
        stats = srv.run(reqs)
        assert stats['completed'] == 2 and all(r.status == 'ok' for r in reqs)
        phi, n = solve_alone(cuda, 32, rho)
        assert torch.equal(reqs[0].phi, phi)

        gd = grid_for(40, H, device=cuda)
        ps = PoissonSolver(3, 'J', 2e-10)
        ps.set_grid_descriptor(gd)
        assert _lib.lib.gfd_test_fail_alloc(1) == 0
        with pytest.raises(MemoryError):
            ps.initialize()
        ps.initialize()                       # the next allocation succeeds
        lap = Laplace(gd, -0.25 / np.pi, 3)
        f = torch.zeros(tuple(int(x) for x in gd.n_c), dtype=torch.float64, device=cuda)
        assert _lib.lib.gfd_test_fail_alloc(1) == 0
        with pytest.raises(MemoryError):
            lap.relax(2, f, f.clone(), 1, 1.0)
        kin = Laplace(gd, -0.5, 3, complex)
        assert _lib.lib.gfd_test_fail_alloc(1) == 0
        with pytest.raises(MemoryError):
            Preconditioner(gd, kin, complex, block=2)
    finally:
        _lib.lib.gfd_test_fail_alloc(0)


def test_server_metrics_and_cuda_timer(cuda):
    """The JSON-lines stream of a served run has one record per request,
    carrying its status and V-cycle count, and a summary equal to the
    returned one; a CudaTimer around solves reports device time for the
    nested regions (positive, outer >= inner)."""
    import io
    import json
    import torch
    from gpaw_b200.serving import PoissonServer, Request, grid_for, pair_density
    from gpaw_b200.timing import CudaTimer, MetricsLog
    rhos = [pair_density(grid_for(32, H, device=cuda), 70 + i) for i in range(4)]
    srv = PoissonServer(H, device=cuda, slots=2, nstreams=2,
                        keep_results=lambda r: r.rid in (1, 2))
    reqs = [Request(i, 32, 0.0, rhos[i]) for i in range(4)]
    buf = io.StringIO()
    stats = srv.run(reqs, metrics=MetricsLog(buf))
    # only the selected requests' potentials are kept, and they are theirs
    assert reqs[0].phi is None and reqs[3].phi is None
    for i in (1, 2):
        phi, n = solve_alone(cuda, 32, rhos[i])
        assert reqs[i].niter == n and torch.equal(reqs[i].phi, phi)
    recs = [json.loads(line) for line in buf.getvalue().splitlines()]
    per = [r for r in recs if r['kind'] == 'request']
    assert sorted(r['rid'] for r in per) == [0, 1, 2, 3]
    for r, q in zip(sorted(per, key=lambda r: r['rid']), reqs):
        assert r['status'] == 'ok' and r['niter'] == q.niter and r['done_s'] >= r['arrival_s']
    summ = [r for r in recs if r['kind'] == 'summary']
    assert len(summ) == 1 and summ[0]['completed'] == stats['completed'] == 4

    timer = CudaTimer()
    ps, phi = solve_timer_setup(cuda, rhos[0])
    timer.start('Poisson')
    for _ in range(3):
        timer.start('solve')
        phi.zero_()
        ps.solve(phi, rhos[0])
        timer.stop('solve')
    timer.stop('Poisson')
    outer, inner = timer.get_time('Poisson'), timer.get_time('Poisson', 'solve')
    assert 0 < inner <= outer
    buf = io.StringIO()
    MetricsLog(buf).timer(timer)
    regions = {json.loads(line)['region'] for line in buf.getvalue().splitlines()}
    assert {'Poisson', 'Poisson.solve', 'Other', 'Total'} <= regions


def solve_timer_setup(cuda, rho):
    import torch
    from gpaw_b200.poisson import PoissonSolver
    from gpaw_b200.serving import grid_for
    ps = PoissonSolver(3, 'J', 2e-10)
    ps.set_grid_descriptor(grid_for(32, H, device=cuda))
    ps.initialize()
    return ps, torch.zeros_like(rho)
