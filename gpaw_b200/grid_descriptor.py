"""Uniform 3-D grid for one GPU (no domain decomposition).

Mirrors the subset of gpaw.grid_descriptor.GridDescriptor / gpaw.domain.Domain
that the finite-difference path uses (gpaw/grid_descriptor.py:65-238,
gpaw/domain.py:22-150):

* N_c grid points per axis; a non-periodic axis stores N_c - 1 points
  (beg_c = 1), a periodic one N_c (gpaw/grid_descriptor.py:113-126);
* h_cv = cell_cv / N_c, dv = |det cell| / prod(N_c);
* neighbor_cd = 0 (this domain: periodic wrap) or -1 (zero boundary) and
  sdisp_cd = (+1, -1) on periodic axes (gpaw/domain.py:122-150);
* coarsen() raises ValueError for odd N_c or a grid with no points, which is
  what stops the Poisson level hierarchy (gpaw/poisson.py:75-79).

Arrays are torch tensors on the current CUDA device.
"""
import numpy as np
import torch

from . import _lib
from .tensors import require_device, stream_of, torch_dtype


class GridDescriptor:
    def __init__(self, N_c, cell_cv=(1.0, 1.0, 1.0), pbc_c=True, comm=None, parsize=None,
                 device=None):
        if comm is not None and getattr(comm, 'size', 1) != 1:
            raise NotImplementedError('domain decomposition is not provided: one GPU per grid')
        if isinstance(pbc_c, (bool, int, np.integer, np.bool_)):
            pbc_c = (bool(pbc_c),) * 3
        self.pbc_c = np.array(pbc_c, bool)
        self.N_c = np.array(N_c, int)
        if self.N_c.shape != (3,):
            raise ValueError('N_c needs three entries')
        cell = np.array(cell_cv, float)
        if cell.ndim == 1:
            self.cell_cv = np.diag(cell)
            length_c = cell.copy()
        else:
            self.cell_cv = cell
            length_c = np.sqrt((cell ** 2).sum(1))
        self.icell_cv = np.linalg.inv(self.cell_cv).T
        self.xxxucell_cv = self.cell_cv / length_c[:, None]
        self.xxxiucell_cv = np.linalg.inv(self.xxxucell_cv.T)
        self.beg_c = np.array([0 if p else 1 for p in self.pbc_c])
        self.end_c = self.N_c.copy()
        self.n_c = self.end_c - self.beg_c
        if (self.n_c <= 0).any():
            raise ValueError('Grid too small!')
        self.h_cv = self.cell_cv / self.N_c[:, None]
        self.dv = abs(np.linalg.det(self.cell_cv)) / self.N_c.prod()
        self.orthogonal = not (self.cell_cv - np.diag(self.cell_cv.diagonal())).any()
        spacing_c = (np.linalg.inv(self.cell_cv) ** 2).sum(0) ** -0.5 / self.N_c
        if spacing_c.max() / spacing_c.min() > 1.3:
            raise ValueError('Very anisotropic grid spacings: %s' % spacing_c)
        self.neighbor_cd = np.array([[0, 0] if p else [-1, -1] for p in self.pbc_c], int)
        self.sdisp_cd = np.array([[1, -1] if p else [0, 0] for p in self.pbc_c], int)
        self.comm = None
        self.device = torch.device(device) if device is not None else torch.device('cuda')

    # -- hierarchy -----------------------------------------------------------
    def coarsen(self):
        if (self.N_c % 2).any():
            raise ValueError('Grid %s not divisible by 2!' % self.N_c)
        return GridDescriptor(self.N_c // 2, self.cell_cv, self.pbc_c, device=self.device)

    def refine(self):
        return GridDescriptor(self.N_c * 2, self.cell_cv, self.pbc_c, device=self.device)

    # -- arrays --------------------------------------------------------------
    def get_size_of_global_array(self, pad=False):
        return self.N_c if pad else self.N_c - 1 + self.pbc_c

    def _shape(self, n):
        if isinstance(n, int):
            n = (n,)
        return tuple(n) + tuple(int(x) for x in self.n_c)

    def zeros(self, n=(), dtype=float, global_array=False, pad=False):
        return torch.zeros(self._shape(n), dtype=torch_dtype(dtype), device=self.device)

    def empty(self, n=(), dtype=float, global_array=False, pad=False):
        return torch.empty(self._shape(n), dtype=torch_dtype(dtype), device=self.device)

    def bytecount(self, dtype=float):
        return int(np.prod(self.n_c)) * torch.empty((), dtype=torch_dtype(dtype)).element_size()

    def integrate(self, a_xg, b_xg=None, global_integral=True):
        """sum(a) dv per 3-D array (gpaw/grid_descriptor.py:197-215).  float64
        3-D arrays use the library's deterministic reduction."""
        require_device(a_xg, 'a_xg')
        if b_xg is not None:
            require_device(b_xg, 'b_xg')
            return (torch.vdot(a_xg.reshape(-1), b_xg.reshape(-1)) * self.dv).item()
        if a_xg.ndim == 3 and a_xg.dtype == torch.float64:
            out = (_lib.ctypes.c_double * 1)()
            _lib.check(_lib.lib.gfd_grid_sum(a_xg.data_ptr(), a_xg.numel(), self.dv, out,
                                             stream_of(a_xg)), 'integrate')
            return out[0]
        s = a_xg.reshape(a_xg.shape[:-3] + (-1,)).sum(-1) * self.dv
        return s.item() if a_xg.ndim == 3 else s

    def get_grid_point_coordinates(self, dtype=float, global_array=False):
        """Cartesian coordinates r_vG of the grid points (host numpy array),
        gpaw/grid_descriptor.py:494-501."""
        return np.dot(np.indices(self.n_c, float).T + self.beg_c, self.h_cv).T.copy()

    def __repr__(self):
        return 'GridDescriptor(N_c=%s, pbc_c=%s)' % (list(self.N_c), list(self.pbc_c))
