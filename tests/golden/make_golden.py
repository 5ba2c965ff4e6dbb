"""Generate the golden fixtures in fd_golden.npz from GPAW's own C kernels.

Runs in a checkout where oracle/_ref/libgpawref.so was built from the
reference tree (make -C oracle); every output below comes from the
reference's unmodified c/bmgs + c/bc code (impl='ref'), driven through the
oracle's restated band loops and V-cycle.  Inputs are seeded and stored next
to the outputs, so the tests need neither the reference nor the seeds.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import geometry as G  # noqa: E402
from oracle import kernels as K  # noqa: E402
from oracle import poisson as P  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'fd_golden.npz')


def main():
    if not K.have_ref():
        raise SystemExit('oracle/_ref/libgpawref.so missing: run make -C oracle first')
    rng = np.random.default_rng(20240601)
    d = {}

    def grid(N, h, pbc, cell=None):
        if cell is None:
            cell = np.array(N, float) * h
        return G.Grid(N, cell, pbc)

    # Stencils: Laplace nn=1..3 and Gradient nn=3, real and Bloch-phased complex.
    for tag, pbc in [('np', (0, 0, 0)), ('p', (1, 1, 1)), ('mx', (1, 0, 1))]:
        gd = grid((10, 8, 12), 0.3, pbc)
        shape = (1,) + tuple(gd.n_c)
        a_r = rng.uniform(-1, 1, shape)
        a_c = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        ph = G.bloch_phases(gd, (0.25, 0.1, -0.3))
        d['stencil_%s_in_r' % tag] = a_r
        d['stencil_%s_in_c' % tag] = a_c
        d['stencil_%s_phase' % tag] = ph
        d['stencil_%s_pbc' % tag] = np.array(pbc)
        d['stencil_%s_N' % tag] = gd.N_c
        d['stencil_%s_cell' % tag] = gd.cell_cv
        for n in (1, 2, 3):
            c, o = G.laplace_stencil(gd, -0.5, n)
            d['lap%d_%s_coefs' % (n, tag)] = c
            d['lap%d_%s_offsets' % (n, tag)] = o
            d['lap%d_%s_out_r' % (n, tag)] = K.fd_apply(c, o, gd.pbc_c, a_r, impl='ref')
            d['lap%d_%s_out_c' % (n, tag)] = K.fd_apply(c, o, gd.pbc_c, a_c, ph, impl='ref')
        for v in range(3):
            c, o = G.gradient_stencil(gd, v, 1.0, 3)
            d['grad%d_%s_coefs' % (v, tag)] = c
            d['grad%d_%s_offsets' % (v, tag)] = o
            d['grad%d_%s_out_c' % (v, tag)] = K.fd_apply(c, o, gd.pbc_c, a_c, ph, impl='ref')

    # Non-orthogonal (hexagonal) periodic cell: cross-term stencil, n=2.
    hexcell = np.array([(1, 0, 0), (0.5, 3 ** 0.5 / 2, 0), (0, 0, 1.1)]) * 4.0
    gd = G.Grid((8, 8, 8), hexcell, 1)
    c, o = G.laplace_stencil(gd, 1.0, 2)
    a = rng.standard_normal((1,) + tuple(gd.n_c)) + 1j * rng.standard_normal((1,) + tuple(gd.n_c))
    ph = G.bloch_phases(gd, (0.1, -0.2, 0.3))
    d.update(hex_cell=hexcell, hex_N=gd.N_c, hex_coefs=c, hex_offsets=o, hex_in=a, hex_phase=ph,
             hex_out=K.fd_apply(c, o, gd.pbc_c, a, ph, impl='ref'))

    # Relaxation: 3 weighted-Jacobi sweeps and 2 lexicographic Gauss-Seidel sweeps.
    for tag, pbc in [('np', 0), ('p', 1)]:
        gd = grid((10, 8, 12), 0.25, pbc)
        c, o = G.laplace_stencil(gd, -0.25 / np.pi, 3)
        phi0 = rng.uniform(-1, 1, tuple(gd.n_c))
        rho = rng.uniform(-1, 1, tuple(gd.n_c))
        d['relax_%s_N' % tag] = gd.N_c
        d['relax_%s_pbc' % tag] = np.array([pbc] * 3)
        d['relax_%s_cell' % tag] = gd.cell_cv
        d['relax_%s_coefs' % tag] = c
        d['relax_%s_offsets' % tag] = o
        d['relax_%s_phi0' % tag] = phi0
        d['relax_%s_rho' % tag] = rho
        p = phi0.copy()
        K.relax(2, c, o, gd.pbc_c, p, rho, 3, 2.0 / 3.0, impl='ref')
        d['relax_%s_jacobi3' % tag] = p
        p = phi0.copy()
        K.relax(1, c, o, gd.pbc_c, p, rho, 2, 1.0, impl='ref')
        d['relax_%s_gs2' % tag] = p

    # Transformers: K = 2, 4, 6, 8 restriction and interpolation.
    for tag, pbc in [('np', 0), ('p', 1)]:
        gd = grid((8, 8, 10), 0.4, pbc)
        a_r = rng.uniform(0, 1, (1,) + tuple(gd.n_c))
        a_c = rng.uniform(0, 1, (1,) + tuple(gd.n_c)) + 1j * rng.uniform(0, 1, (1,) + tuple(gd.n_c))
        ph = G.bloch_phases(gd, (0.25, 0.0, 0.1))
        d['tr_%s_N' % tag] = gd.N_c
        d['tr_%s_pbc' % tag] = np.array([pbc] * 3)
        d['tr_%s_cell' % tag] = gd.cell_cv
        d['tr_%s_in_r' % tag] = a_r
        d['tr_%s_in_c' % tag] = a_c
        d['tr_%s_phase' % tag] = ph
        for nn in (1, 2, 3, 4):
            for name, g2 in (('restrict', gd.coarsen()), ('interp', gd.refine())):
                d['tr_%s_%s%d_r' % (tag, name, nn)] = K.transform(gd, g2, nn, a_r, impl='ref')
                d['tr_%s_%s%d_c' % (tag, name, nn)] = K.transform(gd, g2, nn, a_c, ph, impl='ref')

    # Multigrid Poisson solves (Jacobi and lexicographic GS), nn=3 and nn=1.
    for tag, N, pbc, nn, relax in [('j16', 16, 0, 3, 'J'), ('j16p', 16, 1, 3, 'J'),
                                   ('gs16', 16, 0, 1, 'GS')]:
        gd = grid((N, N, N), 0.2 / G.BOHR, pbc)
        r = gd.coords()
        L = gd.cell_cv.diagonal()
        rho = np.zeros(tuple(gd.n_c))
        for q in (1.0, -1.0):
            R = rng.uniform(0.3, 0.7, 3) * L
            s = 0.5 / G.BOHR
            rho += q * np.exp(-sum((r[c] - R[c]) ** 2 for c in range(3)) / (2 * s * s))
        rho -= rho.mean()
        ps = P.PoissonSolver(nn, relax, 2e-10, impl='ref')
        ps.set_grid_descriptor(gd)
        ps.initialize()
        phi = np.zeros(tuple(gd.n_c))
        niter = ps.solve(phi, rho)
        d['ps_%s_N' % tag] = gd.N_c
        d['ps_%s_pbc' % tag] = np.array([pbc] * 3)
        d['ps_%s_cell' % tag] = gd.cell_cv
        d['ps_%s_nn' % tag] = np.array(nn)
        d['ps_%s_relax' % tag] = np.array(relax)
        d['ps_%s_rho' % tag] = rho
        d['ps_%s_phi' % tag] = phi
        d['ps_%s_niter' % tag] = np.array(niter)
        d['ps_%s_err' % tag] = np.array(ps.errors[-1])

    # Mehrstellen Poisson (nn='M': LaplaceA phi = LaplaceB rho), Jacobi.
    for tag, N, pbc in [('m16', 16, 0), ('m16p', 16, 1)]:
        gd = grid((N, N, N), 0.2 / G.BOHR, pbc)
        r = gd.coords()
        L = gd.cell_cv.diagonal()
        rho = np.zeros(tuple(gd.n_c))
        for q in (1.0, -1.0):
            R = rng.uniform(0.3, 0.7, 3) * L
            s = 0.5 / G.BOHR
            rho += q * np.exp(-sum((r[c] - R[c]) ** 2 for c in range(3)) / (2 * s * s))
        rho -= rho.mean()
        ps = P.PoissonSolver('M', 'J', 2e-10, impl='ref')
        ps.set_grid_descriptor(gd)
        ps.initialize()
        phi = np.zeros(tuple(gd.n_c))
        niter = ps.solve(phi, rho)
        d['mehr_%s_N' % tag] = gd.N_c
        d['mehr_%s_pbc' % tag] = np.array([pbc] * 3)
        d['mehr_%s_cell' % tag] = gd.cell_cv
        d['mehr_%s_rho' % tag] = rho
        d['mehr_%s_phi' % tag] = phi
        d['mehr_%s_niter' % tag] = np.array(niter)

    np.savez_compressed(OUT, **d)
    print('wrote', OUT, os.path.getsize(OUT), 'bytes,', len(d), 'arrays')


if __name__ == '__main__':
    main()
