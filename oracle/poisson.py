"""Multigrid Poisson solver restated from gpaw/poisson.py -- TEST
INFRASTRUCTURE ONLY.

PoissonSolver(nn, relax, eps) with set_grid_descriptor / initialize / solve
as in gpaw/poisson.py:21-218, V-cycle iterate2 as in gpaw/poisson.py:245-276,
on top of the oracle kernels (impl 'port' or 'ref').  Only the charge-neutral
branch of solve() is restated (gpaw/poisson.py:136-138); the charged branches
need Ewald / Gaussian-multipole machinery that is outside this path.
"""
from math import pi

import numpy as np

from . import geometry, kernels


class PoissonConvergenceError(RuntimeError):
    pass


class PoissonSolver:
    def __init__(self, nn=3, relax='J', eps=2e-10, impl='port'):
        self.nn = nn
        self.eps = eps
        self.relax = relax
        self.maxiter = 1000
        self.impl = impl
        if relax == 'GS':
            self.relax_method = 1
        elif relax == 'J':
            self.relax_method = 2
        else:
            raise NotImplementedError('Relaxation method %s' % relax)

    def set_grid_descriptor(self, gd):
        self.gd = gd
        self.dv = gd.dv
        scale = -0.25 / pi
        self.grids = [gd]
        if self.nn == 'M':
            # Mehrstellen: A phi = B rho (gpaw/poisson.py:53-59)
            self.stencils = [geometry.laplace_a_stencil(gd, -scale)]
            self.B = geometry.laplace_b_stencil()
        else:
            self.stencils = [geometry.laplace_stencil(gd, scale, self.nn)]
            self.B = None
        self.presmooths = [2]
        self.postsmooths = [1]
        self.weights = [2.0 / 3.0]
        level = 0
        while level < 4:
            try:
                gd2 = gd.coarsen()
            except ValueError:
                break
            self.grids.append(gd2)
            self.stencils.append(geometry.laplace_stencil(gd2, scale, 1))
            self.presmooths.append(4)
            self.postsmooths.append(4)
            self.weights.append(1.0)
            level += 1
            gd = gd2
        self.levels = level

    def initialize(self):
        self.rhos = [np.empty(tuple(g.n_c)) for g in self.grids]
        self.phis = [None] + [np.empty(tuple(g.n_c)) for g in self.grids[1:]]
        self.residuals = [np.empty(tuple(g.n_c)) for g in self.grids]
        self.presmooths[self.levels] = 8
        self.postsmooths[self.levels] = 8

    # -- kernels -------------------------------------------------------------
    def _apply(self, level, a):
        c, o = self.stencils[level]
        return kernels.fd_apply(c, o, self.grids[level].pbc_c, a, impl=self.impl)

    def _relax(self, level, nsweeps):
        c, o = self.stencils[level]
        kernels.relax(self.relax_method, c, o, self.grids[level].pbc_c, self.phis[level],
                      self.rhos[level], nsweeps, self.weights[level], impl=self.impl)

    def solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6):
        if eps is None:
            eps = self.eps
        actual_charge = self.gd.integrate(rho)
        background = actual_charge / self.gd.dv / self.gd.global_size().prod()
        if charge is None:
            charge = actual_charge
        if abs(charge) > maxcharge:
            raise NotImplementedError('charged systems are outside the oracle')
        return self.solve_neutral(phi, rho - background, eps=eps)

    def solve_neutral(self, phi, rho, eps=2e-10):
        self.phis[0] = phi
        if self.B is None:
            self.rhos[0][:] = rho
        else:
            # gpaw/poisson.py:196-199
            self.rhos[0][:] = kernels.fd_apply(self.B[0], self.B[1], self.gd.pbc_c, rho,
                                               impl=self.impl)
        niter = 1
        self.errors = []
        while self.iterate2() > eps and niter < self.maxiter:
            niter += 1
        if niter == self.maxiter:
            raise PoissonConvergenceError(
                'Poisson solver did not converge in %d iterations!' % self.maxiter)
        if self.gd.pbc_c.all():
            phi -= phi.sum() / np.prod(self.gd.global_size())
        return niter

    def iterate2(self, level=0):
        if level < self.levels:
            self._relax(level, self.presmooths[level])
            r = self._apply(level, self.phis[level]) - self.rhos[level]
            self.rhos[level + 1][:] = kernels.transform(
                self.grids[level], self.grids[level + 1], 1, r, impl=self.impl)
            self.phis[level + 1][:] = 0.0
            self.iterate2(level + 1)
            corr = kernels.transform(self.grids[level + 1], self.grids[level], 1,
                                     self.phis[level + 1], impl=self.impl)
            self.phis[level] -= corr
        self._relax(level, self.postsmooths[level])
        if level == 0:
            r = self._apply(0, self.phis[0]) - self.rhos[0]
            error = float(np.dot(r.ravel(), r.ravel())) * self.dv
            self.errors.append(error)
            return error
