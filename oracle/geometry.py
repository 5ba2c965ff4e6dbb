"""Grid geometry, stencil coefficients and transformer paddings -- TEST
INFRASTRUCTURE ONLY (the oracle's own restatement, independent of the
product's host layer).

Follows, for a single domain (no domain decomposition):
  gpaw/domain.py:22-150            cell, inverse cell, neighbor_cd, sdisp_cd
  gpaw/grid_descriptor.py:65-150   N_c, beg_c/end_c, n_c, h_cv, dv
  gpaw/grid_descriptor.py:217-238  coarsen / refine
  gpaw/grid_descriptor.py:494-501  grid point coordinates
  gpaw/fd_operators.py:21-66       FDOperator offsets, padding, cfd flag
  gpaw/fd_operators.py:123-144     Gradient coefficients
  gpaw/fd_operators.py:231-292     NewGUCLaplace coefficients + table
  gpaw/transformers.py:19-62       transformer paddings and skips
"""
from fractions import Fraction
from math import factorial

import numpy as np

BOHR = 0.52917721092  # Angstrom per Bohr

# Chelikowsky et al. central-difference Laplacian weights, orders 1..6
# (gpaw/fd_operators.py:286-292), built from exact fractions.
_LAP = [[Fraction(0)],
        [Fraction(-2), Fraction(1)],
        [Fraction(-5, 2), Fraction(4, 3), Fraction(-1, 12)],
        [Fraction(-49, 18), Fraction(3, 2), Fraction(-3, 20), Fraction(1, 90)],
        [Fraction(-205, 72), Fraction(8, 5), Fraction(-1, 5), Fraction(8, 315),
         Fraction(-1, 560)],
        [Fraction(-5269, 1800), Fraction(5, 3), Fraction(-5, 21), Fraction(5, 126),
         Fraction(-5, 1008), Fraction(1, 3150)],
        [Fraction(-5369, 1800), Fraction(12, 7), Fraction(-15, 56), Fraction(10, 189),
         Fraction(-1, 112), Fraction(2, 1925), Fraction(-1, 16632)]]
LAPLACE = [[float(x) for x in row] for row in _LAP]


class Grid:
    """Single-domain uniform grid (gpaw/grid_descriptor.py:65-150)."""

    def __init__(self, N_c, cell_cv=(1.0, 1.0, 1.0), pbc_c=True):
        if isinstance(pbc_c, (int, bool, np.integer, np.bool_)):
            pbc_c = (bool(pbc_c),) * 3
        cell = np.array(cell_cv, float)
        if cell.ndim == 1:
            self.cell_cv = np.diag(cell)
            cell_c = cell
        else:
            self.cell_cv = cell
            cell_c = (cell ** 2).sum(1) ** 0.5
        self.icell_cv = np.linalg.inv(self.cell_cv).T
        self.xxxucell_cv = np.array([self.cell_cv[x] / cell_c[x] for x in range(3)])
        self.xxxiucell_cv = np.linalg.inv(self.xxxucell_cv.T)
        self.pbc_c = np.asarray(pbc_c, bool)
        self.N_c = np.array(N_c, int)
        self.beg_c = np.where(self.pbc_c, 0, 1)
        self.end_c = self.N_c.copy()
        if (self.end_c - self.beg_c <= 0).any():
            raise ValueError('Grid too small!')
        self.n_c = self.end_c - self.beg_c
        self.h_cv = self.cell_cv / self.N_c[:, np.newaxis]
        self.dv = abs(np.linalg.det(self.cell_cv)) / self.N_c.prod()
        self.orthogonal = not (self.cell_cv - np.diag(self.cell_cv.diagonal())).any()
        L_c = (np.linalg.inv(self.cell_cv) ** 2).sum(0) ** -0.5
        h_c = L_c / self.N_c
        if max(h_c) / min(h_c) > 1.3:
            raise ValueError('Very anisotropic grid spacings: %s' % h_c)
        # One domain: the neighbour is this domain itself (periodic) or none.
        self.neighbor_cd = np.where(self.pbc_c[:, None], 0, -1) * np.ones((3, 2), int)
        self.sdisp_cd = np.where(self.pbc_c[:, None], np.array([[1, -1]]), 0)

    def coarsen(self):
        if (self.N_c % 2).any():
            raise ValueError('Grid %s not divisible by 2!' % self.N_c)
        return Grid(self.N_c // 2, self.cell_cv, self.pbc_c)

    def refine(self):
        return Grid(self.N_c * 2, self.cell_cv, self.pbc_c)

    def global_size(self):
        return self.N_c - 1 + self.pbc_c

    def coords(self):
        """Cartesian coordinates r_vG (gpaw/grid_descriptor.py:494-501)."""
        return np.dot(np.indices(self.n_c, float).T + self.beg_c, self.h_cv).T.copy()

    def integrate(self, a):
        a = np.asarray(a)
        if a.ndim == 3:
            return a.sum() * self.dv
        return a.reshape(a.shape[:-3] + (-1,)).sum(-1) * self.dv


def laplace_stencil(gd, scale=1.0, n=1):
    """NewGUCLaplace coefficients/offsets (gpaw/fd_operators.py:231-282)."""
    M_ic = np.indices((3, 3, 3)).reshape((3, -1)).T[-13:] - 1
    u_cv = gd.h_cv / (gd.h_cv ** 2).sum(1)[:, np.newaxis] ** 0.5
    u2_i = (np.dot(M_ic, u_cv) ** 2).sum(1)
    i_d = u2_i.argsort(kind='stable')
    m_mv = np.array([(2, 0, 0), (0, 2, 0), (0, 0, 2), (0, 1, 1), (1, 0, 1), (1, 1, 0)])
    for D in range(3, 7):
        h_dv = np.dot(M_ic[i_d[:D]], gd.h_cv)
        A_md = (h_dv ** m_mv[:, np.newaxis, :]).prod(2)
        a_d, residual, rank, s = np.linalg.lstsq(A_md, [1, 1, 1, 0, 0, 0], rcond=-1)
        if residual.sum() < 1e-14:
            assert rank == D
            break
    a_d = a_d * scale
    offsets = [(0, 0, 0)]
    coefs = [LAPLACE[n][0] * a_d.sum()]
    for d in range(D):
        M_c = M_ic[i_d[d]]
        offsets.extend(np.arange(1, n + 1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(LAPLACE[n][1:]))
        offsets.extend(np.arange(-1, -n - 1, -1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(LAPLACE[n][1:]))
    return np.array(coefs, float), np.array(offsets, np.int64).reshape(-1, 3)


def laplace_a_stencil(gd, scale):
    """Mehrstellen left-hand operator LaplaceA (gpaw/fd_operators.py:192-216):
    centre, six face neighbours and twelve edge neighbours of an orthogonal
    cell (the module divides with true division)."""
    c = (-1.0 / 12.0) / gd.h_cv.diagonal() ** 2 * scale
    c0, c1, c2 = c[1] + c[2], c[0] + c[2], c[1] + c[0]
    a = -16.0 * np.sum(c)
    b = 10.0 * c + 0.125 * a
    coefs = [a, b[0], b[0], b[1], b[1], b[2], b[2]] + [c0] * 4 + [c1] * 4 + [c2] * 4
    offsets = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1),
               (0, -1, -1), (0, -1, 1), (0, 1, -1), (0, 1, 1),
               (-1, 0, -1), (-1, 0, 1), (1, 0, -1), (1, 0, 1),
               (-1, -1, 0), (-1, 1, 0), (1, -1, 0), (1, 1, 0)]
    return np.array(coefs, float), np.array(offsets, np.int64)


def laplace_b_stencil():
    """Mehrstellen right-hand operator LaplaceB (gpaw/fd_operators.py:218-229)."""
    b = 1.0 / 12.0
    return (np.array([0.5, b, b, b, b, b, b]),
            np.array([(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1),
                      (0, 0, 1)], np.int64))


def gradient_stencil(gd, v, scale=1.0, n=1):
    """Gradient coefficients/offsets (gpaw/fd_operators.py:123-144)."""
    h = (gd.h_cv ** 2).sum(1) ** 0.5
    d = gd.xxxiucell_cv[:, v]
    A = np.zeros((2 * n + 1, 2 * n + 1))
    for i, io in enumerate(range(-n, n + 1)):
        for j in range(2 * n + 1):
            A[i, j] = io ** j / float(factorial(j))
    A[n, 0] = 1.0
    coefs = np.linalg.inv(A)[1]
    coefs = np.delete(coefs, len(coefs) // 2)
    offs = np.delete(np.arange(-n, n + 1), n)
    coef_p, offset_pc = [], []
    for i in range(3):
        if abs(d[i]) > 1e-11:
            coef_p.extend(list(coefs * d[i] / h[i] * scale))
            offset = np.zeros((2 * n, 3), int)
            offset[:, i] = offs
            offset_pc.extend(offset)
    return np.array(coef_p, float), np.array(offset_pc, np.int64).reshape(-1, 3)


def fd_layout(offsets_pc, n_c):
    """Padding, flat offsets and cfd flag as FDOperator builds them
    (gpaw/fd_operators.py:21-66)."""
    offsets_pc = np.asarray(offsets_pc, np.int64).reshape(-1, 3)
    cfd = all((o != 0).sum() < 2 for o in offsets_pc)
    maxoffset_c = [max(o[c] for o in offsets_pc) for c in range(3)]
    mp = maxoffset_c[0]
    if maxoffset_c[1] != mp or maxoffset_c[2] != mp:
        mp = max(maxoffset_c)
    M_c = np.asarray(n_c) + 2 * mp
    stride_c = np.array([M_c[1] * M_c[2], M_c[2], 1])
    return int(mp), np.dot(offsets_pc, stride_c).astype(np.int64), cfd


def transformer_layout(gdin, gdout, nn):
    """Paddings, neighbour paddings and skips (gpaw/transformers.py:31-49)."""
    pad_cd = np.empty((3, 2), int)
    npad_cd = np.empty((3, 2), int)
    skip_cd = np.zeros((3, 2), int)
    if (gdin.N_c == 2 * gdout.N_c).all():
        pad_cd[:, 0] = 2 * nn - 1 - 2 * gdout.beg_c + gdin.beg_c
        pad_cd[:, 1] = 2 * nn - 2 + 2 * gdout.end_c - gdin.end_c
        npad_cd[:, 0] = 2 * nn - 2 + 2 * gdout.beg_c - gdin.beg_c
        npad_cd[:, 1] = 2 * nn - 1 - 2 * gdout.end_c + gdin.end_c
        interpolate = False
    else:
        assert (gdout.N_c == 2 * gdin.N_c).all()
        pad_cd[:, 0] = nn - 1 - gdout.beg_c // 2 + gdin.beg_c
        pad_cd[:, 1] = nn + gdout.end_c // 2 - gdin.end_c
        npad_cd[:, 0] = nn + gdout.beg_c // 2 - gdin.beg_c
        npad_cd[:, 1] = nn - 1 - gdout.end_c // 2 + gdin.end_c
        skip_cd[:, 0] = gdout.beg_c % 2
        skip_cd[:, 1] = gdout.end_c % 2
        interpolate = True
        # The reference runs its first interpolation pass into the output
        # array and guards its size (gpaw/transformers.py:50-51).
        assert ((gdin.n_c[0] + 2 * nn - 1) * (gdin.n_c[1] + 2 * nn - 1) <=
                gdout.n_c[0] * gdout.n_c[1])
    assert (pad_cd >= 0).all()
    return pad_cd, npad_cd, skip_cd, interpolate


def bloch_phases(gd, k_c):
    """phase_cd = exp(2 pi i sdisp_cd k_c) (gpaw/kpt_descriptor.py:164-166)."""
    return np.exp(2j * np.pi * gd.sdisp_cd * np.asarray(k_c, float)[:, np.newaxis])
