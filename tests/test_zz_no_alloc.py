"""gfd_operator_relax_noalloc, the relaxation entry point that allocates no
device memory, for callers that cannot call cudaMalloc (a graph capture in
progress, an application-owned memory pool, allocation-free loops).

Through the C ABI it must give the same result as gfd_operator_relax,
within the 1e-13 relaxation tolerance of the other tests, on two calls in a
row (the second call reuses the shared scratch array the first one left
behind), and reject a grid larger than its 16 MiB scratch with an error.
This file is collected last so a failure here does not stop the rest of the
GPU suite.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _relax(lib_fn, op, phi, rho, method, nrelax, w, stream):
    from gpaw_b200 import _lib
    status = lib_fn(op.operator, _lib.GFD_FLOAT64, method, phi.data_ptr(), rho.data_ptr(),
                    nrelax, w, stream)
    assert status == _lib.GFD_OK, _lib.last_error()


@pytest.mark.parametrize('pbc', [0, 1])
def test_noalloc_relax_matches_relax(cuda, pbc):
    import torch
    from gpaw_b200 import _lib
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    gd = GridDescriptor((48, 40, 56), (48 * 0.38, 40 * 0.38, 56 * 0.38), pbc)
    op = Laplace(gd, -0.25 / np.pi, 3)
    rng = np.random.default_rng(7 + pbc)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # two calls in a row share the scratch array
        phi0 = torch.from_numpy(rng.uniform(-1, 1, tuple(gd.n_c))).to(cuda)
        rho = torch.from_numpy(rng.uniform(-1, 1, tuple(gd.n_c))).to(cuda)
        for method, nrelax, w in ((_lib.GFD_RELAX_JACOBI, 3, 2.0 / 3.0),
                                  (_lib.GFD_RELAX_JACOBI, 2, 1.0),
                                  (_lib.GFD_RELAX_GS, 2, 1.0)):
            a = phi0.clone()
            b = phi0.clone()
            _relax(_lib.lib.gfd_operator_relax, op, a, rho, method, nrelax, w, stream)
            _relax(_lib.lib.gfd_operator_relax_noalloc, op, b, rho, method, nrelax, w, stream)
            torch.cuda.synchronize()
            assert rel_err(b.cpu().numpy(), a.cpu().numpy()) < TOL, (call, method, nrelax)


def test_noalloc_relax_rejects_oversized_grid(cuda):
    import torch
    from gpaw_b200 import _lib
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    gd = GridDescriptor((132, 132, 132), (50.0, 50.0, 50.0), 0)  # 131^3 float64 > 16 MiB
    op = Laplace(gd, -0.25 / np.pi, 1)
    phi = torch.zeros(tuple(int(x) for x in gd.n_c), dtype=torch.float64, device=cuda)
    status = _lib.lib.gfd_operator_relax_noalloc(op.operator, _lib.GFD_FLOAT64,
                                                 _lib.GFD_RELAX_JACOBI, phi.data_ptr(),
                                                 phi.data_ptr(), 1, 1.0,
                                                 ctypes.c_void_p(None))
    assert status == _lib.GFD_EINVAL
    assert 'at most' in _lib.last_error()
