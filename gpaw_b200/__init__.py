"""gpaw_b200 -- GPAW's real-space finite-difference path on NVIDIA B200.

Drop-in Python 3 versions of the reference calls, backed by libgpawfd.so
(hand-written sm_100a CUDA behind the C ABI in include/gpaw_fd.h):

    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace, Gradient
    from gpaw_b200.transformers import Transformer
    from gpaw_b200.poisson import PoissonSolver

Arrays are CUDA torch tensors in the reference's C-contiguous layout.
"""
from .errors import ConvergenceError, PoissonConvergenceError  # noqa: F401

__version__ = '0.1'


def library_version():
    from . import _lib
    return _lib.lib.gfd_version().decode()
