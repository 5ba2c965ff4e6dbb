"""Band preconditioner restated from gpaw/preconditioner.py -- TEST
INFRASTRUCTURE ONLY.

The reference's sequence of nineteen array operations
(gpaw/preconditioner.py:45-70), step by step and in the same order, on top
of the oracle's stencil and transformer kernels (impl 'port' or 'ref').
"""
import numpy as np

from . import geometry, kernels


class Preconditioner:
    def __init__(self, gd0, kin0, impl='port'):
        """gd0: oracle Grid; kin0: (coefs, offsets) of the fine kinetic
        operator, coefs[0] the diagonal (gpaw/preconditioner.py:14-23)."""
        self.gd0 = gd0
        self.gd1 = gd0.coarsen()
        self.gd2 = self.gd1.coarsen()
        self.kin0 = kin0
        self.kin1 = geometry.laplace_stencil(self.gd1, -0.5, 1)
        self.kin2 = geometry.laplace_stencil(self.gd2, -0.5, 1)
        self.step = 0.66666666 / kin0[0][0]
        self.impl = impl

    def _kin(self, k, gd, a, phases):
        return kernels.fd_apply(k[0], k[1], gd.pbc_c, a, phases, nthreads=8, impl=self.impl)

    def _tr(self, gin, gout, a, phases):
        return kernels.transform(gin, gout, 1, a, phases, nthreads=8, impl=self.impl)

    def __call__(self, residuals, phases=None):
        """gpaw/preconditioner.py:45-70 with kpt.phase_cd = phases."""
        step = self.step
        g0, g1, g2 = self.gd0, self.gd1, self.gd2
        r1 = self._tr(g0, g1, -residuals, phases)
        d1 = 4 * step * r1
        q1 = self._kin(self.kin1, g1, d1, phases)
        q1 -= r1
        r2 = self._tr(g1, g2, q1, phases)
        d2 = 16 * step * r2
        q2 = self._kin(self.kin2, g2, d2, phases)
        q2 -= r2
        d2 -= 16 * step * q2
        q1 = self._tr(g2, g1, d2, phases)
        d1 -= q1
        q1 = self._kin(self.kin1, g1, d1, phases)
        q1 -= r1
        d1 -= 4 * step * q1
        d0 = self._tr(g1, g0, -d1, phases)
        q0 = self._kin(self.kin0, g0, d0, phases)
        q0 -= residuals
        d0 += -step * q0
        d0 *= -1.0
        return d0
