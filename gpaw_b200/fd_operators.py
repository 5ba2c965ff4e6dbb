"""Finite-difference operators on the GPU (drop-in for gpaw.fd_operators).

FDOperator(coef_p, offset_pc, gd, dtype).apply(in_xg, out_xg, phase_cd) and
.relax(relax_method, f_g, s_g, n, w) keep the reference signatures
(gpaw/fd_operators.py:20-96); the arrays are CUDA torch tensors and the work
runs in libgpawfd.  Coefficient builders:

* Laplace(gd, scale, n, dtype) -> NewGUCLaplace (the reference default,
  gpaw/fd_operators.py:147-153): least-squares weights of 3..6 lattice
  directions (gpaw/fd_operators.py:231-282), centre weight first.
* Gradient(gd, v, scale, n, dtype): order-2n central first derivative
  (gpaw/fd_operators.py:123-144).
* GUCLaplace, LaplaceA / LaplaceB (Mehrstellen) as in
  gpaw/fd_operators.py:192-229, 317-367.
"""
from fractions import Fraction
from math import factorial

import numpy as np
import torch

from . import _lib
from .tensors import dtype_code, is_complex, nbands, require_device, stream_of, torch_dtype

# Central-difference second-derivative weights of order 2, 4, ..., 12
# (Chelikowsky et al., PRB 50, 11355 (1994)); row n holds the centre weight
# followed by the weights of distance 1..n.
_LAPLACE_FRACTIONS = {
    1: ('-2', '1'),
    2: ('-5/2', '4/3', '-1/12'),
    3: ('-49/18', '3/2', '-3/20', '1/90'),
    4: ('-205/72', '8/5', '-1/5', '8/315', '-1/560'),
    5: ('-5269/1800', '5/3', '-5/21', '5/126', '-5/1008', '1/3150'),
    6: ('-5369/1800', '12/7', '-15/56', '10/189', '-1/112', '2/1925', '-1/16632'),
}
laplace = [[0.0]] + [[float(Fraction(x)) for x in _LAPLACE_FRACTIONS[n]] for n in range(1, 7)]

# Cross-derivative weights (gpaw/fd_operators.py:304-313), used by GUCLaplace.
_CROSS = {
    1: ['1/4'],
    2: ['4/9', '-1/18', '1/144'],
    3: ['9/16', '-9/80', '1/80', '9/400', '-1/400', '1/3600'],
}
cross = [[0.0]] + [[float(Fraction(x)) for x in _CROSS[n]] for n in sorted(_CROSS)]


class FDOperator:
    """A stencil on grid gd; offsets are integer (d0, d1, d2) triples."""

    def __init__(self, coef_p, offset_pc, gd, dtype=float, allocate=True):
        offset_pc = np.asarray(offset_pc, np.int64).reshape(-1, 3)
        coef_p = np.ascontiguousarray(coef_p, float).ravel()
        if coef_p.shape[0] != offset_pc.shape[0]:
            raise ValueError('one coefficient per offset')
        self.cfd = bool(all((o != 0).sum() < 2 for o in offset_pc))
        self.mp = int(np.abs(offset_pc).max()) if len(offset_pc) else 0
        self.coef_p = coef_p
        self.offset_pc = offset_pc
        self.gd = gd
        self.dtype = torch_dtype(dtype)
        self.shape = tuple(int(x) for x in gd.n_c)
        self.npoints = len(coef_p)
        self.operator = None
        self.allocated = False
        if allocate:
            self.allocate()

    def __str__(self):
        return '<%d point finite-difference stencil>' % self.npoints

    def allocate(self):
        if self.allocated:
            raise RuntimeError('already allocated')
        coefs, cp = _lib.f64(self.coef_p)
        offs, op = _lib.i64(self.offset_pc)
        size, sp = _lib.i64(self.gd.n_c)
        nbr, np_ = _lib.i64(self.gd.neighbor_cd)
        handle = _lib._vp()
        _lib.check(_lib.lib.gfd_operator_create(
            len(coefs), cp, op, sp, self.mp, np_, int(not is_complex(self.dtype)), int(self.cfd),
            _lib.ctypes.byref(handle)), 'Operator')
        self.operator = handle
        self.allocated = True

    def is_allocated(self):
        return self.allocated

    def __del__(self):
        h = getattr(self, 'operator', None)
        lib = getattr(_lib, 'lib', None) if _lib is not None else None
        if h and lib is not None:  # at interpreter exit the module may be gone
            lib.gfd_operator_destroy(h)
            self.operator = None

    def _check_arrays(self, a, b):
        require_device(a, 'in_xg')
        require_device(b, 'out_xg')
        if tuple(a.shape) != tuple(b.shape):
            raise ValueError('input and output shapes differ: %s %s' % (a.shape, b.shape))
        if tuple(a.shape[-3:]) != self.shape:
            raise ValueError('array shape %s does not match the grid %s'
                             % (tuple(a.shape), self.shape))
        if a.dtype != b.dtype:
            raise ValueError('input and output dtypes differ')
        if is_complex(a.dtype) != is_complex(self.dtype):
            raise ValueError('operator built for %s arrays, got %s' % (self.dtype, a.dtype))

    def apply(self, in_xg, out_xg, phase_cd=None):
        """out_xg = operator applied to in_xg (band-batched over leading axes).
        Complex arrays take Bloch phases phase_cd[3, 2]."""
        self._check_arrays(in_xg, out_xg)
        _, pp = _lib.phases_arg(phase_cd if is_complex(in_xg.dtype) else None)
        _lib.check(_lib.lib.gfd_operator_apply(
            self.operator, dtype_code(in_xg), in_xg.data_ptr(), out_xg.data_ptr(),
            nbands(in_xg), pp, stream_of(in_xg)), 'apply')

    def apply_with_potential(self, in_xg, out_xg, vt_g, phase_cd=None):
        """out_xg = operator(in_xg) + vt_g * in_xg in one pass: the kinetic
        operator and the local potential of FDWaveFunctions.
        apply_pseudo_hamiltonian (gpaw/wavefunctions/fd.py:50-52 with
        gpaw/hamiltonian.py:371-398).  vt_g: one real grid on the device,
        float64 for float64/complex128 bands, float32 for float32/complex64."""
        self._check_arrays(in_xg, out_xg)
        require_device(vt_g, 'vt_g')
        if tuple(vt_g.shape) != self.shape:
            raise ValueError('vt_g must have the grid shape %s' % (self.shape,))
        want = torch.float32 if in_xg.dtype in (torch.float32, torch.complex64) else torch.float64
        if vt_g.dtype != want or not vt_g.is_contiguous():
            raise ValueError('vt_g must be a contiguous %s grid' % want)
        _, pp = _lib.phases_arg(phase_cd if is_complex(in_xg.dtype) else None)
        _lib.check(_lib.lib.gfd_operator_apply_potential(
            self.operator, dtype_code(in_xg), in_xg.data_ptr(), out_xg.data_ptr(),
            nbands(in_xg), pp, vt_g.data_ptr(), stream_of(in_xg)), 'apply_with_potential')

    def relax(self, relax_method, f_g, s_g, n, w=None):
        """n relaxation sweeps for 'operator f_g = s_g', in place on f_g.
        relax_method 1: multicolour Gauss-Seidel; otherwise weighted Jacobi."""
        require_device(f_g, 'f_g')
        require_device(s_g, 's_g')
        if tuple(f_g.shape) != self.shape or tuple(s_g.shape) != self.shape:
            raise ValueError('relax works on one grid array')
        if f_g.dtype != s_g.dtype:
            raise ValueError('f_g and s_g dtypes differ')
        _lib.check(_lib.lib.gfd_operator_relax(
            self.operator, dtype_code(f_g), int(relax_method), f_g.data_ptr(), s_g.data_ptr(),
            int(n), 1.0 if w is None else float(w), stream_of(f_g)), 'relax')

    def get_diagonal_element(self):
        d = _lib.ctypes.c_double()
        _lib.check(_lib.lib.gfd_operator_get_diagonal_element(self.operator,
                                                              _lib.ctypes.byref(d)))
        return d.value

    def estimate_memory(self, mem):
        mem.setsize(0)


def gradient_coefficients(n):
    """First-derivative weights at offsets -n..-1, 1..n of the order-2n
    central difference: row 1 of the inverse Taylor matrix."""
    A = np.array([[io ** j / float(factorial(j)) for j in range(2 * n + 1)]
                  for io in range(-n, n + 1)])
    A[n, 0] = 1.0
    c = np.linalg.inv(A)[1]
    return np.delete(c, n), np.delete(np.arange(-n, n + 1), n)


class Gradient(FDOperator):
    def __init__(self, gd, v, scale=1.0, n=1, dtype=float, allocate=True):
        length_c = np.sqrt((gd.h_cv ** 2).sum(1))
        d_c = gd.xxxiucell_cv[:, v]
        w_k, off_k = gradient_coefficients(n)
        coef_p, offset_pc = [], []
        for c in range(3):
            if abs(d_c[c]) > 1e-11:
                coef_p.extend(w_k * d_c[c] / length_c[c] * scale)
                o = np.zeros((2 * n, 3), int)
                o[:, c] = off_k
                offset_pc.extend(o)
        FDOperator.__init__(self, coef_p, offset_pc, gd, dtype, allocate)


# The 13 lattice directions with a positive first nonzero component, in the
# order np.indices((3, 3, 3)) lists them.
_DIRECTIONS = np.indices((3, 3, 3)).reshape((3, -1)).T[-13:] - 1
# Second-order monomials x^2, y^2, z^2, yz, xz, xy.
_MONOMIALS = np.array([(2, 0, 0), (0, 2, 0), (0, 0, 2), (0, 1, 1), (1, 0, 1), (1, 1, 0)])


def guc_direction_weights(h_cv):
    """Fewest lattice directions d (3 to 6, shortest first) and weights a_d
    with sum_d a_d (d . grad)^2 = nabla^2 exactly for quadratics."""
    unit_cv = h_cv / np.sqrt((h_cv ** 2).sum(1))[:, None]
    order = np.argsort((np.dot(_DIRECTIONS, unit_cv) ** 2).sum(1), kind='stable')
    target = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])
    for D in range(3, 7):
        h_dv = np.dot(_DIRECTIONS[order[:D]], h_cv)
        A = np.prod(h_dv[None, :, :] ** _MONOMIALS[:, None, :], axis=2)
        a_d, residual, rank, _ = np.linalg.lstsq(A, target, rcond=-1)
        if residual.sum() < 1e-14:
            if rank != D:
                raise ValueError('degenerate lattice directions')
            return _DIRECTIONS[order[:D]], a_d
    raise ValueError('no Laplacian stencil fits this cell')


class NewGUCLaplace(FDOperator):
    """Laplacian for general (non-orthorhombic) grids with O(h^2n) error."""

    def __init__(self, gd, scale=1.0, n=1, dtype=float, allocate=True):
        if not 1 <= n <= 6:
            raise ValueError('stencil range n must be 1..6')
        dirs, a_d = guc_direction_weights(gd.h_cv)
        a_d = a_d * scale
        w = np.array(laplace[n])
        offsets = [(0, 0, 0)]
        coefs = [w[0] * a_d.sum()]
        for M_c, a in zip(dirs, a_d):
            for sign in (1, -1):
                for k in range(1, n + 1):
                    offsets.append(tuple(sign * k * M_c))
                    coefs.append(a * w[k])
        FDOperator.__init__(self, coefs, offsets, gd, dtype, allocate)
        self.n = n

    def __str__(self):
        return ('<%d*%d+1=%d point O(h^%d) finite-difference Laplacian>' %
                ((self.npoints - 1) // self.n, self.n, self.npoints, 2 * self.n))


class GUCLaplace(FDOperator):
    """Central-difference Laplacian with explicit cross terms
    (gpaw/fd_operators.py:317-367); n <= 3 here."""

    def __init__(self, gd, scale=1.0, n=1, dtype=float, allocate=True):
        n = int(n)
        if n not in _CROSS:
            raise NotImplementedError('GUCLaplace is provided for n = 1..3')
        h = np.sqrt((gd.h_cv ** 2).sum(1))
        iu = gd.xxxiucell_cv
        d2 = (iu ** 2).sum(1)
        offsets = [(0, 0, 0)]
        coefs = [scale * np.sum(d2 * laplace[n][0] / h ** 2)]
        for d in range(1, n + 1):
            c = scale * d2 * laplace[n][d] / h ** 2
            offsets.extend([(-d, 0, 0), (d, 0, 0), (0, -d, 0), (0, d, 0), (0, 0, -d), (0, 0, d)])
            coefs.extend([c[0], c[0], c[1], c[1], c[2], c[2]])
        ci = 0
        for d1 in range(n):
            for d2_ in range(d1, n):
                quad = [[(d1 + 1, d2_ + 1, 0), (-d1 - 1, d2_ + 1, 0), (d1 + 1, -d2_ - 1, 0),
                         (-d1 - 1, -d2_ - 1, 0)],
                        [(0, d1 + 1, d2_ + 1), (0, -d1 - 1, d2_ + 1), (0, d1 + 1, -d2_ - 1),
                         (0, -d1 - 1, -d2_ - 1)],
                        [(d2_ + 1, 0, d1 + 1), (d2_ + 1, 0, -d1 - 1), (-d2_ - 1, 0, d1 + 1),
                         (-d2_ - 1, 0, -d1 - 1)]]
                for i in range(3):
                    j = (i + 1) % 3
                    c = scale * 2.0 * cross[n][ci] * np.dot(iu[i], iu[j]) / (h[i] * h[j])
                    if abs(c) > 1e-11:
                        offsets.extend(quad[i])
                        coefs.extend([c, -c, -c, c])
                        if d2_ > d1:
                            perm = [0, 1, 2]
                            perm[i], perm[j] = j, i
                            offsets.extend([tuple(np.take(o, perm)) for o in quad[i]])
                            coefs.extend([c, -c, -c, c])
                ci += 1
        FDOperator.__init__(self, coefs, offsets, gd, dtype, allocate)


class LaplaceA(FDOperator):
    """Mehrstellen left-hand operator (gpaw/fd_operators.py:192-216)."""

    def __init__(self, gd, scale, dtype=float, allocate=True):
        if not gd.orthogonal:
            raise RuntimeError('Mehrstellen stencil needs an orthogonal cell')
        c = (-1.0 / 12) / gd.h_cv.diagonal() ** 2 * scale
        c0, c1, c2 = c[1] + c[2], c[0] + c[2], c[1] + c[0]
        a = -16.0 * np.sum(c)
        b = 10.0 * c + 0.125 * a
        coefs = [a, b[0], b[0], b[1], b[1], b[2], b[2]] + [c0] * 4 + [c1] * 4 + [c2] * 4
        offsets = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1),
                   (0, -1, -1), (0, -1, 1), (0, 1, -1), (0, 1, 1),
                   (-1, 0, -1), (-1, 0, 1), (1, 0, -1), (1, 0, 1),
                   (-1, -1, 0), (-1, 1, 0), (1, -1, 0), (1, 1, 0)]
        FDOperator.__init__(self, coefs, offsets, gd, dtype, allocate)


class LaplaceB(FDOperator):
    """Mehrstellen right-hand operator (gpaw/fd_operators.py:218-229)."""

    def __init__(self, gd, dtype=float, allocate=True):
        b = 1.0 / 12.0
        FDOperator.__init__(self, [0.5, b, b, b, b, b, b],
                            [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0),
                             (0, 0, -1), (0, 0, 1)], gd, dtype, allocate)


def Laplace(gd, scale=1.0, n=1, dtype=float, allocate=True):
    """Laplace factory (gpaw/fd_operators.py:147-153).  n=9 selects the FFT
    Laplacian, which is not part of the finite-difference path."""
    if n == 9:
        raise NotImplementedError('FTLaplace (n=9) is an FFT operator, not provided')
    return NewGUCLaplace(gd, scale, n, dtype, allocate)


def apply_pseudo_hamiltonian(kin, psit_xG, Htpsit_xG, vt_G, phase_cd=None):
    """Htpsit_xG = kin psit_xG + vt_G psit_xG over a band batch: GPAW's
    FDWaveFunctions.apply_pseudo_hamiltonian (gpaw/wavefunctions/fd.py:50-52),
    the kinetic apply followed by Hamiltonian.apply_local_potential
    (gpaw/hamiltonian.py:371-398, Htpsit += psit * vt), as one kernel pass:
    the potential joins the stencil's centre weight, so each band is read
    once and written once (FDOperator.apply_with_potential).

    kin: the kinetic FDOperator (Laplace(gd, -0.5, nn, dtype)); vt_G: the spin
    channel's local potential on the same grid (float64 for float64/complex128
    bands, float32 for float32/complex64); phase_cd: the k-point's Bloch phases
    for complex bands."""
    if not isinstance(kin, FDOperator):
        raise TypeError('kin must be an FDOperator')
    kin.apply_with_potential(psit_xG, Htpsit_xG, vt_G, phase_cd)
