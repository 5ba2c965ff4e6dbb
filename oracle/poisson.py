"""Multigrid Poisson solver restated from gpaw/poisson.py -- TEST
INFRASTRUCTURE ONLY.

PoissonSolver(nn, relax, eps) with set_grid_descriptor / initialize / solve
as in gpaw/poisson.py:21-218, V-cycle iterate2 as in gpaw/poisson.py:245-276,
on top of the oracle kernels (impl 'port' or 'ref').  solve() has the
reference's three branches (gpaw/poisson.py:124-191): charge neutral; charged
and fully periodic (a Madelung shift, gpaw/utilities/ewald.py); charged and
non-periodic (an L = 0 generalised Gaussian carries the monopole,
gpaw/utilities/gauss.py).
"""
from math import pi, sqrt

import numpy as np
from scipy.special import erf, erfc

from . import geometry, kernels


def gauss_coordinates(gd, origin=None, tiny=1e-12):
    """Cartesian coordinates relative to the cell centre and their squared
    length, clamped away from zero (gpaw/utilities/tools.py:92-118)."""
    if origin is None:
        origin = 0.5 * gd.cell_cv.sum(0)
    r_vG = gd.coords() - np.asarray(origin, float)[:, None, None, None]
    for c in range(3):
        if gd.pbc_c[c]:
            L = gd.cell_cv[c, c]
            r_vG[c] = np.where(r_vG[c] > 0.5 * L, r_vG[c] - L, r_vG[c])
            r_vG[c] = np.where(r_vG[c] < -0.5 * L, r_vG[c] + L, r_vG[c])
    r2_G = np.sum(r_vG ** 2, axis=0)
    return r_vG, np.where(r2_G < tiny, tiny, r2_G)


def gauss_width(gd, a=19.0):
    """Exponent of the generalised Gaussians: exp(-a) at the boundary
    (Gaussian.set_width, gpaw/utilities/gauss.py:63-65)."""
    return 4 * a * (gd.icell_cv ** 2).sum(1).max()


def gauss_l0(gd):
    """The L = 0 generalised Gaussian and its potential
    (gpaw/utilities/gauss.py:22, 35, 67-82):
    g = sqrt(4 a^3) / pi exp(-a r^2), v = 2 sqrt(pi) erf(sqrt(a) r) / r."""
    a = gauss_width(gd)
    _, r2 = gauss_coordinates(gd)
    r = np.sqrt(r2)
    return (np.sqrt(a ** 3 * 4) / pi * np.exp(-a * r2),
            2.0 * 1.7724538509055159 * erf(np.sqrt(a) * r) / r)


def madelung(cell_cv, G=5, Ng=(9, 9, 9), Nl=(3, 3, 3)):
    """Potential at a probe charge -1 from its own periodic images in a
    neutralising background, by Ewald summation (gpaw/utilities/ewald.py:
    26-37, 44-91, 94-148 with r = r_B = 0 and the l = 0 charge excluded)."""
    cell = np.asarray(cell_cv, float)
    vol = abs(np.linalg.det(cell))
    recip = np.linalg.inv(cell).T
    G = G / np.sqrt((cell ** 2).sum(1).max())
    q = -1.0
    # real-space sum over l != 0 of erfc(G |l|) / |l|
    e_r = 0.0
    for i in range(-Nl[0], Nl[0] + 1):
        for j in range(-Nl[1], Nl[1] + 1):
            for k in range(-Nl[2], Nl[2] + 1):
                l_v = i * cell[0] + j * cell[1] + k * cell[2]
                d = np.linalg.norm(l_v)
                if d > 1e-5:
                    e_r += erfc(G * d) / d
    # reciprocal-space sum over g != 0
    e_g = 0.0
    for i in range(-Ng[0], Ng[0] + 1):
        for j in range(-Ng[1], Ng[1] + 1):
            for k in range(-Ng[2], Ng[2] + 1):
                g_v = 2 * pi * (i * recip[0] + j * recip[1] + k * recip[2])
                g2 = np.dot(g_v, g_v)
                if g2 > 1e-10:
                    x = 0.25 * g2 / G ** 2
                    e_g += np.exp(-x) / x
    e = q * e_r + q * pi / (vol * G ** 2) * e_g
    e -= q * 2.0 * G / np.sqrt(pi)        # the excluded l = 0 charge
    e += -q * pi / (G ** 2 * vol)         # compensating homogeneous background
    return e


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

    def solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6,
              zero_initial_phi=False):
        """gpaw/poisson.py:124-191."""
        if eps is None:
            eps = self.eps
        actual_charge = self.gd.integrate(rho)
        background = actual_charge / self.gd.dv / self.gd.global_size().prod()
        if charge is None:
            charge = actual_charge
        if abs(charge) <= maxcharge:
            return self.solve_neutral(phi, rho - background, eps=eps)
        if self.gd.pbc_c.all():
            # charged and periodic: shift by the Madelung potential
            if getattr(self, 'charged_periodic_correction', None) is None:
                self.charged_periodic_correction = madelung(self.gd.cell_cv)
            if zero_initial_phi:
                phi[:] = 0.0
            else:
                phi -= charge * self.charged_periodic_correction
            niter = self.solve_neutral(phi, rho - background, eps=eps)
            phi += charge * self.charged_periodic_correction
            return niter
        if not self.gd.pbc_c.any():
            # charged and non-periodic: a Gaussian carries the monopole
            if not hasattr(self, 'rho_gauss'):
                self.rho_gauss, self.phi_gauss = gauss_l0(self.gd)
            q = actual_charge / np.sqrt(4 * pi)
            rho_neutral = rho - q * self.rho_gauss
            if zero_initial_phi:
                phi[:] = 0.0
            else:
                phi -= q * self.phi_gauss
            niter = self.solve_neutral(phi, rho_neutral, eps=eps)
            phi += q * self.phi_gauss
            return niter
        raise NotImplementedError('charged system with mixed boundary conditions')

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
