"""Multigrid Poisson solver on the GPU (drop-in for gpaw.poisson.PoissonSolver).

PoissonSolver(nn=3, relax='J', eps=2e-10) with set_grid_descriptor(gd),
initialize() and solve(phi, rho, charge=None, eps=None, maxcharge=1e-6,
zero_initial_phi=False) -> number of V-cycles, as gpaw/poisson.py:21-218.
The level hierarchy is the reference's (gpaw/poisson.py:45-89, 111-113):

  level 0      Laplace(gd, -1/(4 pi), nn), 2 pre- / 1 post-smoothing sweeps,
               Jacobi weight 2/3
  levels 1..L  Laplace(gd_l, -1/(4 pi), 1), 4 / 4 sweeps, weight 1, at most
               four coarsenings; the coarsest level smooths 8 / 8 times
  transfers    Transformer(nn=1) restriction and interpolation

relax='J' is weighted Jacobi as in the reference; relax='GS' is multicolour
Gauss-Seidel (the reference's lexicographic sweep is sequential).  The whole
V-cycle, the residual norm and the convergence test run in libgpawfd on the
device; phi and rho are float64 CUDA tensors.

precision='mixed' keeps the float64 residual, update and norm and runs the
V-cycle in float32 (defect correction); precision='fp64' is the plain form.
"""
from math import pi

import numpy as np

from . import _lib
from .errors import PoissonConvergenceError  # noqa: F401  (re-exported)
from .fd_operators import Laplace, LaplaceA, LaplaceB
from .tensors import require_device, stream_of, stream_of_device
from .transformers import Transformer


def madelung(cell_cv):
    """Potential shift per unit charge of a charged periodic system:
    madelung(cell_cv) of gpaw/utilities/ewald.py:148 (Ewald sum, computed by
    libgpawfd on the host)."""
    c, cp = _lib.f64(np.asarray(cell_cv, float).reshape(3, 3))
    out = _lib.ctypes.c_double(0.0)
    _lib.check(_lib.lib.gfd_madelung(cp, _lib.ctypes.byref(out)), 'madelung')
    return out.value


class PoissonSolver:
    def __init__(self, nn=3, relax='J', eps=2e-10, precision='fp64'):
        self.relax = relax
        self.nn = nn
        self.eps = eps
        self.maxiter = 1000
        self.charged_periodic_correction = None
        if relax == 'GS':
            self.relax_method = _lib.GFD_RELAX_GS
        elif relax == 'J':
            self.relax_method = _lib.GFD_RELAX_JACOBI
        else:
            raise NotImplementedError('Relaxation method %s' % relax)
        if precision not in ('fp64', 'mixed'):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        self.solver = None

    def get_method(self):
        return ['Gauss-Seidel', 'Jacobi'][self.relax_method - 1]

    def get_stencil(self):
        return self.nn

    def set_grid_descriptor(self, gd):
        self.gd = gd
        self.dv = gd.dv
        scale = -0.25 / pi
        if self.nn == 'M':
            # Mehrstellen: LaplaceA phi = LaplaceB rho (gpaw/poisson.py:53-59)
            if not gd.orthogonal:
                raise RuntimeError('Cannot use Mehrstellen stencil with non orthogonal cell.')
            self.operators = [LaplaceA(gd, -scale, allocate=False)]
            self.B = LaplaceB(gd, allocate=False)
        else:
            self.operators = [Laplace(gd, scale, self.nn, allocate=False)]
            self.B = None
        self.interpolators = []
        self.restrictors = []
        self.presmooths = [2]
        self.postsmooths = [1]
        self.weights = [2.0 / 3.0]
        level = 0
        while level < 4:
            try:
                gd2 = gd.coarsen()
            except ValueError:
                break
            self.operators.append(Laplace(gd2, scale, 1, allocate=False))
            self.interpolators.append(Transformer(gd2, gd, allocate=False))
            self.restrictors.append(Transformer(gd, gd2, allocate=False))
            self.presmooths.append(4)
            self.postsmooths.append(4)
            self.weights.append(1.0)
            level += 1
            gd = gd2
        self.levels = level

    def initialize(self, load_gauss=False):
        extra = [self.B] if self.B is not None else []
        for obj in self.operators + self.interpolators + self.restrictors + extra:
            if not obj.allocated:
                obj.allocate()
        self.presmooths[self.levels] = 8
        self.postsmooths[self.levels] = 8
        self.step = 0.66666666 / self.operators[0].get_diagonal_element()
        L = self.levels
        ops = (_lib._vp * (L + 1))(*[o.operator for o in self.operators])
        rs = (_lib._vp * max(L, 1))(*[t.transformer for t in self.restrictors])
        ips = (_lib._vp * max(L, 1))(*[t.transformer for t in self.interpolators])
        pre = (_lib.ctypes.c_int * (L + 1))(*self.presmooths)
        post = (_lib.ctypes.c_int * (L + 1))(*self.postsmooths)
        w = (_lib.ctypes.c_double * (L + 1))(*self.weights)
        handle = _lib._vp()
        mode = _lib.GFD_POISSON_MIXED if self.precision == 'mixed' else _lib.GFD_POISSON_FP64
        _lib.check(_lib.lib.gfd_poisson_create(
            L, ops, rs, ips, pre, post, w, self.relax_method, float(self.gd.dv),
            int(self.gd.pbc_c.all()), mode, _lib.ctypes.byref(handle)), 'PoissonSolver')
        self.solver = handle
        if self.B is not None:
            _lib.check(_lib.lib.gfd_poisson_set_rhs_operator(handle, self.B.operator),
                       'PoissonSolver')
        if self.gd.pbc_c.all():
            # charged periodic systems: the Madelung shift per unit charge
            # (charged_periodic_correction, gpaw/poisson.py:143-151)
            if self.charged_periodic_correction is None:
                self.charged_periodic_correction = madelung(self.gd.cell_cv)
            _lib.check(_lib.lib.gfd_poisson_set_madelung(handle,
                                                         self.charged_periodic_correction),
                       'PoissonSolver')
        if load_gauss:
            self.load_gauss()

    def load_gauss(self):
        """The compensating L = 0 Gaussian of charged non-periodic systems
        and its potential, on the device (gpaw/poisson.py:118-123;
        Gaussian(gd) of gpaw/utilities/gauss.py:47-82: exponent
        4 * 19 * max_c sum_v icell_cv^2, centred in the cell)."""
        if self.solver is None:
            self.initialize()
        if getattr(self, '_gauss_loaded', False):
            return
        gd = self.gd
        a = 4 * 19.0 * (gd.icell_cv ** 2).sum(1).max()
        center = 0.5 * gd.cell_cv.sum(0)
        h, hp = _lib.f64(gd.h_cv)
        b, bp = _lib.i64(gd.beg_c)
        c, cp = _lib.f64(center)
        _lib.check(_lib.lib.gfd_poisson_load_gauss(self.solver, hp, bp, cp, float(a),
                                                   stream_of_device(gd.device)),
                   'PoissonSolver.load_gauss')
        self._gauss_loaded = True

    def __del__(self):
        h = getattr(self, 'solver', None)
        lib = getattr(_lib, 'lib', None) if _lib is not None else None
        if h and lib is not None:  # at interpreter exit the module may be gone
            lib.gfd_poisson_destroy(h)
            self.solver = None

    def solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6, zero_initial_phi=False):
        """Solve nabla^2 phi = -4 pi rho; phi holds the initial guess and
        receives the solution.  Returns the number of V-cycles.  The
        reference's three branches (gpaw/poisson.py:124-191): neutral, charged
        periodic (Madelung shift), charged non-periodic (compensating
        Gaussian, loaded on first need); charged with mixed boundary
        conditions raises NotImplementedError.  zero_initial_phi starts the
        charged branches from phi = 0, as the reference (the neutral branch
        keeps phi).  Raises PoissonConvergenceError after maxiter V-cycles."""
        if self.solver is None:
            self.initialize()
        self._check_arrays(phi, rho)
        if eps is None:
            eps = self.eps
        flags = _lib.GFD_SOLVE_ZERO_INITIAL_PHI if zero_initial_phi else 0
        niter = _lib.ctypes.c_int(0)
        err = _lib.ctypes.c_double(0.0)
        for attempt in range(2):
            status = _lib.lib.gfd_poisson_solve_ex(
                self.solver, phi.data_ptr(), rho.data_ptr(),
                _lib.nan() if charge is None else float(charge), float(eps), float(maxcharge),
                int(self.maxiter), flags, _lib.ctypes.byref(niter), _lib.ctypes.byref(err),
                stream_of(phi))
            if status != _lib.GFD_ENEEDGAUSS or attempt:
                break
            # A charged non-periodic rho: phi is unchanged; load the Gaussian
            # (gpaw/poisson.py:162-164) and solve again.
            self.load_gauss()
        self.niter = niter.value
        self.error = err.value
        _lib.check(status, 'PoissonSolver.solve')
        return niter.value

    def prepare(self):
        """Allocate the hierarchy and capture the solve graph now (a solve of
        rho = 0, which stops after one V-cycle), so the first real solve
        does not pay for them."""
        import torch
        if self.solver is None:
            self.initialize()
        z = torch.zeros(tuple(int(x) for x in self.gd.n_c), dtype=torch.float64,
                        device=self.gd.device)
        self.solve(z, torch.zeros_like(z))

    def autotune(self, reps=5):
        """Tune the launch plans of every level's Jacobi sweep, restriction
        and interpolation on the solver's own buffers
        (gpaw_b200.autotune); the next solve captures its graph with them."""
        import torch
        if self.solver is None:
            self.initialize()
        _lib.check(_lib.lib.gfd_poisson_autotune(
            self.solver, int(reps), torch.cuda.current_stream(self.gd.device).cuda_stream),
            'PoissonSolver.autotune')
        torch.cuda.current_stream(self.gd.device).synchronize()

    def solve_async(self, phi, rho, charge=None, eps=None, maxcharge=1e-6):
        """Enqueue a solve on the current stream and return at once; call
        result() after the stream has passed it (e.g. a recorded event)."""
        if self.solver is None:
            self.initialize()
        self._check_arrays(phi, rho)
        if eps is None:
            eps = self.eps
        _lib.check(_lib.lib.gfd_poisson_solve_async(
            self.solver, phi.data_ptr(), rho.data_ptr(),
            _lib.nan() if charge is None else float(charge), float(eps), float(maxcharge),
            int(self.maxiter), stream_of(phi)), 'PoissonSolver.solve_async')

    def result(self):
        """(niter, error) of the last completed solve_async; raises as solve."""
        niter = _lib.ctypes.c_int(0)
        err = _lib.ctypes.c_double(0.0)
        status = _lib.lib.gfd_poisson_result(self.solver, _lib.ctypes.byref(niter),
                                             _lib.ctypes.byref(err))
        self.niter = niter.value
        self.error = err.value
        _lib.check(status, 'PoissonSolver.result')
        return niter.value, err.value

    def _check_arrays(self, phi, rho):
        import torch
        require_device(phi, 'phi')
        require_device(rho, 'rho')
        if phi.dtype != torch.float64 or rho.dtype != torch.float64:
            raise ValueError('phi and rho must be float64')
        shape = tuple(int(x) for x in self.gd.n_c)
        if tuple(phi.shape) != shape or tuple(rho.shape) != shape:
            raise ValueError('phi and rho must have the grid shape %s' % (shape,))

    def nbytes(self):
        """Device memory held by the solver's level hierarchy (bytes)."""
        esz = 4 if self.precision == 'mixed' else 8
        n = int(np.prod(self.gd.n_c))
        total = n * 8 * (4 if self.precision == 'mixed' else 1)
        g = self.gd
        for level in range(self.levels + 1):
            total += 4 * int(np.prod(g.n_c)) * esz
            if level < self.levels:
                g = g.coarsen()
        return total

    def estimate_memory(self, mem):
        nbytes = 0
        g = int(np.prod(self.gd.n_c)) * 8
        for _ in range(self.levels + 1):
            nbytes += 4 * g
            g //= 8
        mem.subnode('rho, phi (x2), residual [%d levels]' % self.levels, nbytes)

    def __repr__(self):
        return 'PoissonSolver(relax=\'%s\', nn=%s, eps=%e)' % (self.relax, repr(self.nn),
                                                              self.eps)
