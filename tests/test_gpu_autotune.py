"""Launch-plan autotuning: every plan the tuner can pick gives the oracle's
results (1e-13 relative in FP64), the marching plans bit-identical ones,
and tuned Poisson solves keep the reference's V-cycle count and potential.

Plans are forced by loading a one-line cache file, so every candidate form
(one thread per point; marching with each tile and axis-0 split) runs."""
import numpy as np
import pytest

from oracle import geometry as G
from oracle import kernels as K
from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-13

# (form, tile, ctas_per_sm): form 0 one thread per point, 1 marching;
# tile 0/1/2 = 32/16/8 columns (16 and 8 only for radius <= 2), 3 = 32 columns
# by 8 rows (complex128 apply only; other launches fall back to the built-in tile),
# 4 = complex bands with re / im on lane pairs (radius <= 3), 5 = the same for
# complex128 on full rows staged by TMA.
PLANS = [(0, 0, 4), (1, 0, 1), (1, 0, 2), (1, 0, 8), (1, 1, 4), (1, 2, 2), (1, 3, 2),
         (1, 4, 2), (1, 4, 8), (1, 5, 1), (1, 5, 4)]


def family(plan, cplx):
    """Marching plans that share one summation order give bit-identical
    results: star_kernel's tiles, and each lane-pair kernel on its own
    (complex only; real launches of tiles 4 and 5 fall back to star_kernel)."""
    return 'tile%d' % plan[1] if cplx and plan[1] in (4, 5) else 'star'


@pytest.fixture
def plans(tmp_path):
    from gpaw_b200 import autotune
    autotune.clear()
    yield tmp_path
    autotune.clear()


def force(path, kind, dtype, mode, n, order, per, nbands, plan):
    from gpaw_b200 import autotune
    nbc = int(np.floor(np.log2(nbands)))
    with open(path, 'w') as f:
        f.write('gfd-tune 1\n')
        f.write('%d %d %d %d %d %d %d %d %d %d %d %d 1.0\n'
                % ((kind, dtype, mode) + tuple(n) + (order, per, nbc) + tuple(plan)))
    autotune.clear()
    autotune.load(path)


def per_mask(pbc):
    return sum(1 << c for c in range(3) if pbc[c])


@pytest.mark.parametrize('n', [1, 3])
@pytest.mark.parametrize('cplx', [False, True])
def test_forced_stencil_plans_match_oracle(cuda, plans, n, cplx):
    import torch
    from gpaw_b200 import autotune
    from gpaw_b200.fd_operators import FDOperator
    from gpaw_b200.grid_descriptor import GridDescriptor
    N, pbc = (20, 26, 40), (1, 0, 1)
    og = G.Grid(N, np.array(N) * 0.25, pbc)
    gd = GridDescriptor(og.N_c, og.cell_cv, og.pbc_c)
    c, o = G.laplace_stencil(og, 1.3, n)
    rng = np.random.default_rng(5 + n)
    a = rng.standard_normal((3,) + tuple(og.n_c))
    ph = None
    if cplx:
        a = a + 1j * rng.standard_normal(a.shape)
        ph = G.bloch_phases(og, (0.25, 0.0, -0.13))
    ref = K.fd_apply(c, o, og.pbc_c, a, ph)
    t = torch.from_numpy(a).to(cuda)
    op = FDOperator(c, o, gd, t.dtype)
    march = {}
    for plan in PLANS:
        if n > 2 and plan[1] in (1, 2):
            continue
        force(plans / 'p.txt', 0, 1 if cplx else 0, 0, og.n_c, n, per_mask(pbc), 3, plan)
        got = autotune.operator_plan(op, 3)
        assert got is not None and got['form'] == ('direct', 'march')[plan[0]]
        out = torch.full_like(t, float('nan'))
        op.apply(t, out, ph)
        torch.cuda.synchronize()
        res = out.cpu().numpy()
        assert rel_err(res, ref) < TOL, plan
        if plan[0] == 1:
            fam = family(plan, cplx)
            march.setdefault(fam, res)
            assert np.array_equal(res, march[fam]), plan


def test_forced_jacobi_plans_match_oracle(cuda, plans):
    import torch
    from gpaw_b200.fd_operators import FDOperator
    from gpaw_b200.grid_descriptor import GridDescriptor
    N, pbc = (24, 30, 36), (0, 0, 0)
    og = G.Grid(N, np.array(N) * 0.3, pbc)
    gd = GridDescriptor(og.N_c, og.cell_cv, og.pbc_c)
    c, o = G.laplace_stencil(og, -0.25 / np.pi, 3)
    rng = np.random.default_rng(9)
    phi = rng.standard_normal(tuple(og.n_c))
    rho = rng.standard_normal(tuple(og.n_c))
    ref = phi.copy()
    K.relax(2, c, o, og.pbc_c, ref, rho, 3, 2.0 / 3.0)
    op = FDOperator(c, o, gd, torch.float64)
    for plan in [(0, 0, 4), (1, 0, 1), (1, 0, 8)]:
        force(plans / 'p.txt', 0, 0, 1, og.n_c, 3, 0, 1, plan)
        f = torch.from_numpy(phi).to(cuda)
        op.relax(2, f, torch.from_numpy(rho).to(cuda), 3, 2.0 / 3.0)
        torch.cuda.synchronize()
        assert rel_err(f.cpu().numpy(), ref) < TOL, plan


@pytest.mark.parametrize('interp', [False, True])
def test_forced_transfer_plans_match_oracle(cuda, plans, interp):
    import torch
    from gpaw_b200 import autotune
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.transformers import Transformer
    N, pbc = (24, 16, 40), (1, 0, 1)
    og = G.Grid(N, np.array(N) * 0.3, pbc)
    gd = GridDescriptor(og.N_c, og.cell_cv, og.pbc_c)
    g2 = gd.refine() if interp else gd.coarsen()
    og2 = og.refine() if interp else og.coarsen()
    rng = np.random.default_rng(13)
    a = rng.standard_normal((2,) + tuple(og.n_c))
    ref = K.transform(og, og2, 3, a)
    t = torch.from_numpy(a).to(cuda)
    tr = Transformer(gd, g2, 3, t.dtype)
    march = None
    for plan in [(0, 0, 4), (1, 0, 1), (1, 0, 2), (1, 0, 8)]:
        force(plans / 'p.txt', 2 if interp else 1, 0, 0, og.n_c, 3, per_mask(pbc), 2, plan)
        assert autotune.transformer_plan(tr, 2)['ctas_per_sm'] == plan[2]
        out = torch.full((2,) + tuple(int(x) for x in g2.n_c), float('nan'),
                         dtype=t.dtype, device=cuda)
        tr.apply(t, out)
        torch.cuda.synchronize()
        res = out.cpu().numpy()
        assert rel_err(res, ref) < TOL, plan
        if plan[0] == 1:
            if march is None:
                march = res
            assert np.array_equal(res, march), plan


def test_tune_operator_cache_roundtrip(cuda, plans):
    """tune_operator picks a plan, later launches use it, and the cache
    survives save / clear / load."""
    import torch
    from gpaw_b200 import autotune
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    og = G.Grid((40, 40, 40), (40 * 0.18 / G.BOHR,) * 3, 1)
    gd = GridDescriptor(og.N_c, og.cell_cv, og.pbc_c)
    ph = G.bloch_phases(og, (0.25, 0.0, 0.0))
    lap = Laplace(gd, -0.5, 3, complex)
    assert autotune.operator_plan(lap, 8) is None
    plan = autotune.tune_operator(lap, nbands=8, phase_cd=ph, reps=2)
    assert plan['form'] in ('direct', 'march') and plan['us'] > 0
    assert autotune.operator_plan(lap, 8) == plan
    assert autotune.operator_plan(lap, 15) == plan   # same band-count class
    assert autotune.operator_plan(lap, 16) is None
    pot = autotune.tune_operator(lap, nbands=8, mode='potential', phase_cd=ph, reps=1)
    assert autotune.operator_plan(lap, 8, mode='potential') == pot
    assert autotune.count() == 2
    autotune.save(plans / 'c.txt')
    autotune.clear()
    assert autotune.count() == 0 and autotune.operator_plan(lap, 8) is None
    autotune.load(plans / 'c.txt')
    got = autotune.operator_plan(lap, 8)
    assert got['form'] == plan['form'] and got['tile'] == plan['tile']
    assert got['ctas_per_sm'] == plan['ctas_per_sm']
    rng = np.random.default_rng(21)
    a = rng.standard_normal((8,) + tuple(og.n_c)) + 1j * rng.standard_normal((8,) + tuple(og.n_c))
    t = torch.from_numpy(a).to(cuda)
    out = torch.empty_like(t)
    lap.apply(t, out, ph)
    torch.cuda.synchronize()
    ref = K.fd_apply(lap.coef_p, lap.offset_pc, og.pbc_c, a, ph, nthreads=8)
    assert rel_err(out.cpu().numpy(), ref) < TOL


def test_tuned_poisson_keeps_vcycles_and_potential(cuda, plans):
    import torch
    from test_gpu_poisson import gaussians_rho, solve_oracle
    from gpaw_b200 import autotune
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.poisson import PoissonSolver
    og = G.Grid((48,) * 3, (48 * 0.2 / G.BOHR,) * 3, 0)
    rho = gaussians_rho(og, 16, 3)
    phi_o, n_o, _ = solve_oracle(og, rho)
    gd = GridDescriptor(og.N_c, og.cell_cv, og.pbc_c)
    for precision, tol in (('fp64', 1e-10), ('mixed', 1e-9)):
        ps = PoissonSolver(3, 'J', 2e-10, precision=precision)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        r = torch.from_numpy(rho).to(cuda)
        phi0 = torch.zeros_like(r)
        n0 = ps.solve(phi0, r)        # captured with the built-in rules
        ps.autotune(reps=2)
        assert autotune.count() > 0
        phi1 = torch.zeros_like(r)
        n1 = ps.solve(phi1, r)        # recaptured with the tuned plans
        assert ps.error <= 2e-10
        if precision == 'fp64':
            assert n0 == n_o and n1 == n_o
        assert np.abs(phi1.cpu().numpy() - phi_o).max() < tol
        autotune.clear()


def test_autotune_argument_errors(cuda, plans):
    import torch
    from gpaw_b200 import autotune
    from gpaw_b200.fd_operators import FDOperator, Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    gd = GridDescriptor((16, 16, 16), np.eye(3) * 3.0, (1, 1, 1))
    lap = Laplace(gd, 1.0, 2)
    with pytest.raises(ValueError):
        autotune.tune_operator(lap, 2, mode='jacobi', w=0.0)
    with pytest.raises(ValueError):
        autotune.tune_operator(lap, 2, mode='bogus')
    with pytest.raises(ValueError):
        autotune.tune_operator(lap, 2, dtype=torch.complex128)
    cross = FDOperator([1.0, 0.5, 0.5], [(0, 0, 0), (1, 1, 0), (-1, -1, 0)], gd)
    with pytest.raises(NotImplementedError):
        autotune.tune_operator(cross, 1)
    assert autotune.count() == 0


@pytest.mark.parametrize('nn', [1, 3, 4])
@pytest.mark.parametrize('N,pbc', [((12, 20, 96), (1, 1, 1)), ((10, 17, 192), (1, 0, 1)),
                                   ((9, 24, 97), (0, 1, 0)), ((8, 16, 48), (1, 1, 1))])
def test_tile48_matches_oracle(cuda, plans, nn, N, pbc):
    """The 48-column tile (plan tile 6, the built-in choice where axis 2 is
    a multiple of 48) for complex128 apply and apply with a potential:
    against the oracle (Bloch phases on every periodic axis, so the wrapped
    axis-2 halo carries its phase; zero boundaries on the others) and bit
    for bit equal to the short tile (tile 3), which sums in the same
    order."""
    import torch
    from gpaw_b200 import autotune
    from gpaw_b200.fd_operators import FDOperator
    from gpaw_b200.grid_descriptor import GridDescriptor
    og = G.Grid(N, np.array(N) * 0.25, pbc)
    gd = GridDescriptor(og.N_c, og.cell_cv, og.pbc_c)
    c, o = G.laplace_stencil(og, -0.5, nn)
    rng = np.random.default_rng(21 + nn)
    a = rng.standard_normal((3,) + tuple(og.n_c)) + 1j * rng.standard_normal((3,) + tuple(og.n_c))
    v = rng.uniform(-1, 1, tuple(og.n_c))
    ph = G.bloch_phases(og, (0.25, -0.1, 0.3))
    ref = K.fd_apply(c, o, og.pbc_c, a, ph)
    t = torch.from_numpy(a).to(cuda)
    vt = torch.from_numpy(v).to(cuda)
    op = FDOperator(c, o, gd, t.dtype)
    res = {}
    for tile in (6, 3):
        for mode in (0, 3):
            force(plans / 'p.txt', 0, 1, mode, og.n_c, nn, per_mask(pbc), 3, (1, tile, 1))
            got = autotune.operator_plan(op, 3, mode='potential' if mode == 3 else 'apply')
            assert got is not None and got['tile'] == {6: '48x8', 3: '32x8'}[tile]
            out = torch.full_like(t, float('nan'))
            if mode == 0:
                op.apply(t, out, ph)
            else:
                op.apply_with_potential(t, out, vt, ph)
            torch.cuda.synchronize()
            res[tile, mode] = out.cpu().numpy()
            want = ref if mode == 0 else ref + v * a
            assert rel_err(res[tile, mode], want) < TOL, (tile, mode)
    for mode in (0, 3):
        assert np.array_equal(res[6, mode], res[3, mode]), mode
    # complex64 bands: the 48-column tile (now built-in there) against the
    # 32 x 16 tile (plan tile 0, same summation order) and the FP64 oracle
    t64 = t.to(torch.complex64)
    op64 = FDOperator(c, o, gd, t64.dtype)
    r64 = {}
    for tile in (6, 0):
        force(plans / 'p.txt', 0, 3, 0, og.n_c, nn, per_mask(pbc), 3, (1, tile, 1))
        out = torch.full_like(t64, float('nan'))
        op64.apply(t64, out, ph)
        torch.cuda.synchronize()
        r64[tile] = out.cpu().numpy()
    assert np.array_equal(r64[6], r64[0])
    assert rel_err(r64[6].astype(complex), ref) < 2e-6
