"""The CPU oracle, pinned before it is trusted (no GPU needed).

1. Against the golden vectors in tests/golden/fd_golden.npz, which GPAW's own
   unmodified C kernels produced (tests/golden/make_golden.py).
2. Against the reference's known-answer tests, re-expressed here:
   gpaw/test/laplace.py:51-87 (polynomial exactness),
   gpaw/test/gradient.py:15-63 (exact ramp derivatives),
   gpaw/test/transformations.py:9-48 and gpaw/test/non_periodic.py:5-24
   (integral conservation).
3. Against the reference library itself when it was built here.
"""
from math import cos, pi, sin

import numpy as np
import pytest

from oracle import geometry as G
from oracle import kernels as K
from oracle import poisson as P
from conftest import rel_err


def _grid(d, prefix):
    return G.Grid(d[prefix + '_N'], d[prefix + '_cell'], d[prefix + '_pbc'])


@pytest.mark.parametrize('tag', ['np', 'p', 'mx'])
def test_stencils_match_golden(golden, tag):
    d = golden
    gd = _grid(d, 'stencil_' + tag)
    a_r, a_c, ph = d['stencil_%s_in_r' % tag], d['stencil_%s_in_c' % tag], d['stencil_%s_phase' % tag]
    for n in (1, 2, 3):
        c, o = d['lap%d_%s_coefs' % (n, tag)], d['lap%d_%s_offsets' % (n, tag)]
        assert rel_err(K.fd_apply(c, o, gd.pbc_c, a_r), d['lap%d_%s_out_r' % (n, tag)]) < 1e-15
        assert rel_err(K.fd_apply(c, o, gd.pbc_c, a_c, ph), d['lap%d_%s_out_c' % (n, tag)]) < 1e-15
        # the oracle's own coefficient builder reproduces the stored ones
        c2, o2 = G.laplace_stencil(gd, -0.5, n)
        assert np.array_equal(o2, o) and np.abs(c2 - c).max() <= 1e-15 * np.abs(c).max()
    for v in range(3):
        c, o = d['grad%d_%s_coefs' % (v, tag)], d['grad%d_%s_offsets' % (v, tag)]
        assert rel_err(K.fd_apply(c, o, gd.pbc_c, a_c, ph), d['grad%d_%s_out_c' % (v, tag)]) < 1e-15


def test_cross_stencil_matches_golden(golden):
    d = golden
    gd = G.Grid(d['hex_N'], d['hex_cell'], 1)
    out = K.fd_apply(d['hex_coefs'], d['hex_offsets'], gd.pbc_c, d['hex_in'], d['hex_phase'])
    assert rel_err(out, d['hex_out']) < 1e-15


@pytest.mark.parametrize('tag', ['np', 'p'])
def test_relax_matches_golden(golden, tag):
    d = golden
    gd = _grid(d, 'relax_' + tag)
    c, o = d['relax_%s_coefs' % tag], d['relax_%s_offsets' % tag]
    p = d['relax_%s_phi0' % tag].copy()
    K.relax(2, c, o, gd.pbc_c, p, d['relax_%s_rho' % tag], 3, 2.0 / 3.0)
    assert np.abs(p - d['relax_%s_jacobi3' % tag]).max() == 0.0
    p = d['relax_%s_phi0' % tag].copy()
    K.relax(1, c, o, gd.pbc_c, p, d['relax_%s_rho' % tag], 2, 1.0)
    assert np.abs(p - d['relax_%s_gs2' % tag]).max() == 0.0


@pytest.mark.parametrize('tag', ['np', 'p'])
def test_transformers_match_golden(golden, tag):
    d = golden
    gd = _grid(d, 'tr_' + tag)
    for nn in (1, 2, 3, 4):
        for name, g2 in (('restrict', gd.coarsen()), ('interp', gd.refine())):
            out_r = K.transform(gd, g2, nn, d['tr_%s_in_r' % tag])
            assert rel_err(out_r, d['tr_%s_%s%d_r' % (tag, name, nn)]) < 1e-15
            out_c = K.transform(gd, g2, nn, d['tr_%s_in_c' % tag], d['tr_%s_phase' % tag])
            assert rel_err(out_c, d['tr_%s_%s%d_c' % (tag, name, nn)]) < 1e-15


@pytest.mark.parametrize('tag', ['j16', 'j16p', 'gs16'])
def test_poisson_matches_golden(golden, tag):
    d = golden
    gd = _grid(d, 'ps_' + tag)
    ps = P.PoissonSolver(int(d['ps_%s_nn' % tag]), str(d['ps_%s_relax' % tag]), 2e-10)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    phi = np.zeros(tuple(gd.n_c))
    niter = ps.solve(phi, d['ps_%s_rho' % tag])
    assert niter == int(d['ps_%s_niter' % tag])
    assert np.abs(phi - d['ps_%s_phi' % tag]).max() < 1e-13


# -- known-answer tests of the reference, re-expressed -----------------------

CELLS = [
    ('hexagonal', [(1, 0, 0), (0.5, 3 ** 0.5 / 2, 0), (0, 0, 1.1)]),
    ('fcc', [(0, 1, 1), (1, 0, 1), (1, 1, 0)]),
    ('bcc', [(-1, 1, 1), (1, -1, 1), (1, 1, -1)]),
    ('sc', [1.1, 1.02, 1.03]),
    ('distorted hexagonal', [(1, 0, 0), (1.02 * cos(pi / 3 - 0.02), 1.02 * sin(pi / 3 - 0.02), 0),
                             (0, 0, 1.0)]),
]


@pytest.mark.parametrize('name,cell', CELLS)
def test_laplace_gradient_polynomial_exactness(name, cell):
    """gpaw/test/laplace.py:51-87: exact on monomials of degree <= 2n at the
    centre point, within 2e-12."""
    for n in range(1, 4):
        N = 2 * n + 2
        gd = G.Grid((N, N, N), cell)
        r_gv = gd.coords().transpose((1, 2, 3, 0)) - gd.cell_cv.sum(0) / 2
        lap = G.laplace_stencil(gd, 1.0, n)
        grads = [G.gradient_stencil(gd, v, 1.0, n) for v in range(3)]
        for m in range(0, 2 * n + 1):
            for ix in range(m + 1):
                for iy in range(m - ix + 1):
                    iz = m - ix - iy
                    a = (r_gv ** (ix, iy, iz)).prod(3)
                    r = 2.0 if (m == 2 and max(ix, iy, iz) == 2) else 0.0
                    b = K.fd_apply(*lap, gd.pbc_c, a)
                    assert abs(b[n + 1, n + 1, n + 1] - r) < 2e-12
                    for v in range(3):
                        b = K.fd_apply(*grads[v], gd.pbc_c, a)
                        r = 1.0 if (m == 1 and (ix, iy, iz)[v] == 1) else 0.0
                        assert abs(b[n + 1, n + 1, n + 1] - r) < 2e-12


def test_gradient_exact_values():
    """gpaw/test/gradient.py:15-63."""
    gd = G.Grid((8, 1, 1), (8.0, 1.0, 1.0))
    a = np.zeros(tuple(gd.n_c))
    a[:, 0, 0] = np.arange(8)
    dadx = K.fd_apply(*G.gradient_stencil(gd, 0), gd.pbc_c, a)
    assert dadx[3, 0, 0] == 1.0 and np.sum(dadx[:, 0, 0]) == 0.0
    gd = G.Grid((1, 8, 1), (1.0, 8.0, 1.0), (1, 0, 1))
    a = np.zeros(tuple(gd.n_c))
    a[0, :, 0] = np.arange(gd.beg_c[1], gd.end_c[1]) - 1
    dady = K.fd_apply(*G.gradient_stencil(gd, 1), gd.pbc_c, a)
    assert dady[0, 0, 0] == 0.5 and np.sum(dady[0, :, 0]) == 3.0
    gd = G.Grid((1, 7, 1), ((1.0, 0.0, 0.0), (5.0, 5.0, 0.0), (0.0, 0.0, 0.7)))
    a = np.zeros(tuple(gd.n_c))
    a[0, :, 0] = np.arange(gd.beg_c[1], gd.end_c[1]) - 1
    dady = K.fd_apply(*G.gradient_stencil(gd, 1), gd.pbc_c, a)
    assert dady[0, 0, 0] == -3.5 and abs(np.sum(dady[0, :, 0])) < 1e-12


def test_transformations_conserve_integral():
    """gpaw/test/transformations.py:9-48 (periodic, K = 2..8, real and complex)."""
    gd = G.Grid((20, 20, 20))
    rng = np.random.RandomState(8)
    a = rng.random_sample(tuple(gd.n_c))
    ac = rng.random_sample(tuple(gd.n_c)) + 1j * rng.random_sample(tuple(gd.n_c))
    for g2 in (gd.refine(), gd.coarsen()):
        for k in (2, 4, 6, 8):
            b = K.transform(gd, g2, k // 2, a)
            assert abs(gd.integrate(a) - g2.integrate(b)) < 1e-14
            b = K.transform(gd, g2, k // 2, ac, np.ones((3, 2), complex))
            assert abs(gd.integrate(ac) - g2.integrate(b)) < 1e-14


def test_non_periodic_conserves_integral():
    """gpaw/test/non_periodic.py:5-24."""
    gd1 = G.Grid((20, 20, 20), (8.0, 8.0, 8.0), 0)
    rng = np.random.RandomState(8)
    a1 = rng.random_sample(tuple(gd1.n_c))
    gd2 = gd1.refine()
    a2 = K.transform(gd1, gd2, 1, a1)
    assert abs(gd1.integrate(a1) - gd2.integrate(a2)) < 1e-10
    a2[0] = a2[:, 0] = a2[:, :, 0] = 0.0
    a2[-1] = a2[:, -1] = a2[:, :, -1] = 0.0
    a1 = K.transform(gd2, gd1, 1, a2)
    assert abs(gd1.integrate(a1) - gd2.integrate(a2)) < 1e-10


@pytest.mark.skipif(not K.have_ref(), reason='reference library not built here')
def test_port_equals_reference_library():
    """Port and the unmodified reference agree bit for bit on real data."""
    rng = np.random.default_rng(5)
    for pbc in (0, 1, (1, 0, 0)):
        gd = G.Grid((13, 9, 11), (13 * 0.3, 9 * 0.3, 11 * 0.3), pbc)
        c, o = G.laplace_stencil(gd, -0.5, 3)
        a = rng.standard_normal((3,) + tuple(gd.n_c))
        assert np.array_equal(K.fd_apply(c, o, gd.pbc_c, a), K.fd_apply(c, o, gd.pbc_c, a, impl='ref'))
        ac = a + 1j * rng.standard_normal(a.shape)
        ph = G.bloch_phases(gd, (0.3, -0.1, 0.2))
        assert rel_err(K.fd_apply(c, o, gd.pbc_c, ac, ph),
                       K.fd_apply(c, o, gd.pbc_c, ac, ph, impl='ref')) < 1e-15


def test_oracle_preconditioner_is_linear():
    """The restated preconditioner (gpaw/preconditioner.py:45-70) is a linear
    map of the residuals: P(a R1 + b R2) = a P(R1) + b P(R2), periodic with
    Bloch phases and zero boundary."""
    from oracle.preconditioner import Preconditioner as OraclePC
    rng = np.random.default_rng(12)
    for N, pbc, k in (((16, 16, 16), 1, (0.25, 0.0, 0.1)), ((16, 12, 20), 0, None)):
        gd = G.Grid(N, np.array(N) * 0.4, pbc)
        c, o = G.laplace_stencil(gd, -0.5, 2)
        pc = OraclePC(gd, (c, o))
        shape = (2,) + tuple(gd.n_c)
        R1 = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        R2 = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        ph = G.bloch_phases(gd, k) if k else np.ones((3, 2), complex)
        lhs = pc(2.0 * R1 - 0.5 * R2, ph)
        rhs = 2.0 * pc(R1, ph) - 0.5 * pc(R2, ph)
        assert rel_err(lhs, rhs) < 1e-13


@pytest.mark.parametrize('tag', ['m16', 'm16p'])
def test_mehrstellen_poisson_matches_golden(golden, tag):
    """nn='M' (LaplaceA phi = LaplaceB rho, gpaw/poisson.py:53-59, 196-199)
    against the solve run on the reference's own C kernels."""
    d = golden
    gd = _grid(d, 'mehr_' + tag)
    ps = P.PoissonSolver('M', 'J', 2e-10)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    phi = np.zeros(tuple(gd.n_c))
    niter = ps.solve(phi, d['mehr_%s_rho' % tag])
    assert niter == int(d['mehr_%s_niter' % tag])
    assert np.abs(phi - d['mehr_%s_phi' % tag]).max() < 1e-13


@pytest.mark.skipif(not K.have_ref(), reason='reference library not built here')
def test_cross_term_relax_port_equals_reference():
    """Relaxation with a cross-term stencil (LaplaceA: the operator's cfd flag
    is 0, so halo corners are filled) bit for bit against GPAW's C."""
    rng = np.random.default_rng(6)
    for pbc in (0, 1, (1, 0, 1)):
        gd = G.Grid((12, 10, 14), (3.0, 2.5, 3.5), pbc)
        c, o = G.laplace_a_stencil(gd, 0.25 / pi)
        a = rng.standard_normal(tuple(gd.n_c))
        rho = rng.standard_normal(tuple(gd.n_c))
        for method, w in ((2, 2.0 / 3.0), (1, 1.0)):
            p1, p2 = a.copy(), a.copy()
            K.relax(method, c, o, gd.pbc_c, p1, rho, 2, w)
            K.relax(method, c, o, gd.pbc_c, p2, rho, 2, w, impl='ref')
            assert np.array_equal(p1, p2), (pbc, method)


def symmetric_blobs(N, h):
    """Two identical radial blobs at (0, 0, 0) and the centre of a periodic
    N^3 grid, mean removed (the geometry of gpaw/test/poisson.py:8-30)."""
    rc = N / 2.0 * 0.9 * h
    i = np.arange(N)
    a = np.zeros((N,) * 3)
    for centre in (0, N // 2):
        d = np.minimum(np.abs(i - centre), N - np.abs(i - centre)) * h
        r2 = d[:, None, None] ** 2 + d[None, :, None] ** 2 + d[None, None, :] ** 2
        # the spline through (0, 1), (rc/2, 0.5), (rc, 0) times Y_00
        a += np.where(r2 < rc * rc, 1 - np.sqrt(r2) / rc, 0.0) / np.sqrt(4 * np.pi)
    return a - a.mean()


@pytest.mark.parametrize('relax,tol', [('J', 6e-16), ('GS', 3e-6)])
def test_oracle_poisson_symmetry(relax, tol):
    """gpaw/test/poisson.py:31-41 on the oracle: phi[0,0,0] == phi[8,8,8]
    (nn = 1, periodic 16^3, cell 2.87 A; lexicographic Gauss-Seidel breaks
    the symmetry up to the reference's 3e-6)."""
    N, L = 16, 2.87 / 0.529177
    og = G.Grid((N,) * 3, (L,) * 3, 1)
    ps = P.PoissonSolver(1, relax, 2e-10)
    ps.set_grid_descriptor(og)
    ps.initialize()
    b = np.zeros((N,) * 3)
    ps.solve(b, symmetric_blobs(N, L / N), charge=0)
    assert abs(b[0, 0, 0] - b[8, 8, 8]) < tol
