"""Band preconditioner on the GPU: gpaw.preconditioner.Preconditioner
(gpaw/preconditioner.py:13-70).

Same construction (two coarsenings, nn = 1 kinetic operators and
transformers, step = 0.66666666 / kin0.get_diagonal_element()) and the same
call, residuals -> preconditioned residuals, with the k-point's Bloch phases.
The reference's nineteen array operations per call run as eight device
passes (gfd_preconditioner_apply); the arithmetic is the same up to the
order of the floating-point operations.
"""
import torch

from . import _lib
from .fd_operators import Laplace
from .tensors import dtype_code, is_complex, require_device, stream_of, torch_dtype
from .transformers import Transformer


class Preconditioner:
    def __init__(self, gd0, kin0, dtype=float, block=1):
        gd1 = gd0.coarsen()
        gd2 = gd1.coarsen()
        self.gd0 = gd0
        self.kin0 = kin0
        self.kin1 = Laplace(gd1, -0.5, 1, dtype)
        self.kin2 = Laplace(gd2, -0.5, 1, dtype)
        self.dtype = torch_dtype(dtype)
        self.block = int(block)
        self.step = 0.66666666 / kin0.get_diagonal_element()
        self.restrictor_object0 = Transformer(gd0, gd1, 1, dtype)
        self.restrictor_object1 = Transformer(gd1, gd2, 1, dtype)
        self.interpolator_object2 = Transformer(gd2, gd1, 1, dtype)
        self.interpolator_object1 = Transformer(gd1, gd0, 1, dtype)
        self.handle = None
        self.out = None
        self.allocated = False
        self.allocate()

    def allocate(self):
        if self.allocated:
            return
        for k in (self.kin0, self.kin1, self.kin2):
            if k.operator is None:
                k.allocate()
        ts = (self.restrictor_object0, self.restrictor_object1, self.interpolator_object2,
              self.interpolator_object1)
        for t in ts:
            if not t.allocated:
                t.allocate()
        h = _lib._vp()
        code = dtype_code(torch.empty(0, dtype=self.dtype))
        _lib.check(_lib.lib.gfd_preconditioner_create(
            self.kin0.operator, self.kin1.operator, self.kin2.operator,
            *[t.transformer for t in ts], code, self.block, _lib.ctypes.byref(h)),
            'Preconditioner')
        self.handle = h
        shape = (self.block,) + tuple(int(x) for x in self.gd0.n_c)
        self.out = torch.empty(shape, dtype=self.dtype, device=self.gd0.device)
        self.allocated = True

    def __del__(self):
        h = getattr(self, 'handle', None)
        lib = getattr(_lib, 'lib', None) if _lib is not None else None
        if h and lib is not None:  # at interpreter exit the module may be gone
            lib.gfd_preconditioner_destroy(h)
            self.handle = None

    def __call__(self, residuals, kpt=None):
        """Preconditioned residuals of the bands in `residuals` (nb x grid, or
        one grid).  Returns a view of the preconditioner's own output array,
        as the reference returns its scratch (valid until the next call)."""
        require_device(residuals, 'residuals')
        if residuals.dtype != self.dtype:
            raise ValueError('residuals dtype %s, preconditioner built for %s'
                             % (residuals.dtype, self.dtype))
        grid = tuple(int(x) for x in self.gd0.n_c)
        single = residuals.dim() == 3
        if tuple(residuals.shape[-3:]) != grid or residuals.dim() not in (3, 4):
            raise ValueError('residuals must have shape (nb,) + %s' % (grid,))
        if not residuals.is_contiguous():
            raise ValueError('residuals must be contiguous')
        nb = 1 if single else int(residuals.shape[0])
        if nb > self.block:
            raise ValueError('%d bands exceed the block of %d' % (nb, self.block))
        phases = getattr(kpt, 'phase_cd', None) if kpt is not None else None
        _, pp = _lib.phases_arg(phases if is_complex(self.dtype) else None)
        out = self.out[:nb]
        _lib.check(_lib.lib.gfd_preconditioner_apply(
            self.handle, dtype_code(residuals), residuals.data_ptr(), out.data_ptr(), nb, pp,
            stream_of(residuals)), 'Preconditioner')
        return out[0] if single else out
