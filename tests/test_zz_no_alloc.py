"""gfd_operator_relax_noalloc, the relaxation entry point that allocates no
device memory, for callers that cannot call cudaMalloc (a graph capture in
progress, an application-owned memory pool, allocation-free loops).

Through the C ABI it must give the same result as gfd_operator_relax, and
its Jacobi sweeps the oracle's (the reference's relaxation restated in C),
within the 1e-13 relaxation tolerance of the other tests (2e-6 for float32
against the float64 oracle), on two calls in a row: the second call reuses
the shared scratch array the first one left behind.  Grids up to the 16 MiB
scratch are accepted (128^3 float64; 150^3 only in float32), larger ones are
rejected with an error.  This file is collected last so a failure here does
not stop the rest of the GPU suite.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-13
TOL32 = 2e-6


def _call(lib_fn, op, dtype, phi, rho, method, nrelax, w, stream):
    from gpaw_b200 import _lib
    return lib_fn(op.operator, dtype, method, phi.data_ptr(), rho.data_ptr(), nrelax, w, stream)


def _relax(lib_fn, op, dtype, phi, rho, method, nrelax, w, stream):
    from gpaw_b200 import _lib
    status = _call(lib_fn, op, dtype, phi, rho, method, nrelax, w, stream)
    assert status == _lib.GFD_OK, _lib.last_error()


@pytest.mark.parametrize('pbc', [0, 1])
def test_noalloc_relax_matches_relax_and_oracle(cuda, pbc):
    import torch
    from gpaw_b200 import _lib
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    from oracle import kernels as K
    gd = GridDescriptor((48, 40, 56), (48 * 0.38, 40 * 0.38, 56 * 0.38), pbc)
    op = Laplace(gd, -0.25 / np.pi, 3)
    rng = np.random.default_rng(7 + pbc)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # two calls in a row share the scratch array
        phi0_h = rng.uniform(-1, 1, tuple(gd.n_c))
        rho_h = rng.uniform(-1, 1, tuple(gd.n_c))
        phi0 = torch.from_numpy(phi0_h).to(cuda)
        rho = torch.from_numpy(rho_h).to(cuda)
        for method, nrelax, w in ((_lib.GFD_RELAX_JACOBI, 3, 2.0 / 3.0),
                                  (_lib.GFD_RELAX_JACOBI, 2, 1.0),
                                  (_lib.GFD_RELAX_GS, 2, 1.0)):
            a = phi0.clone()
            b = phi0.clone()
            _relax(_lib.lib.gfd_operator_relax, op, _lib.GFD_FLOAT64, a, rho, method, nrelax, w,
                   stream)
            _relax(_lib.lib.gfd_operator_relax_noalloc, op, _lib.GFD_FLOAT64, b, rho, method,
                   nrelax, w, stream)
            torch.cuda.synchronize()
            got = b.cpu().numpy()
            assert rel_err(got, a.cpu().numpy()) < TOL, (call, method, nrelax)
            if method == _lib.GFD_RELAX_JACOBI:
                # The reference's lexicographic Gauss-Seidel is a sequential
                # sweep and the GPU's is multicolour, so only Jacobi iterates
                # are comparable point for point.
                ref = phi0_h.copy()
                K.relax(method, op.coef_p, op.offset_pc, gd.pbc_c, ref, rho_h, nrelax, w)
                assert rel_err(got, ref) < TOL, (call, nrelax, w)


def test_noalloc_relax_float32(cuda):
    """The float32 branch: the same as gfd_operator_relax in float32 on two
    calls in a row, and within 2e-6 of the float64 oracle's Jacobi sweeps."""
    import torch
    from gpaw_b200 import _lib
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    from oracle import kernels as K
    gd = GridDescriptor((64, 64, 64), (64 * 0.38,) * 3, 0)
    op = Laplace(gd, -0.25 / np.pi, 3)
    rng = np.random.default_rng(11)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        phi0_h = rng.uniform(-1, 1, tuple(gd.n_c))
        rho_h = rng.uniform(-1, 1, tuple(gd.n_c))
        phi0 = torch.from_numpy(phi0_h).to(cuda, torch.float32)
        rho = torch.from_numpy(rho_h).to(cuda, torch.float32)
        a = phi0.clone()
        b = phi0.clone()
        _relax(_lib.lib.gfd_operator_relax, op, _lib.GFD_FLOAT32, a, rho, _lib.GFD_RELAX_JACOBI,
               3, 2.0 / 3.0, stream)
        _relax(_lib.lib.gfd_operator_relax_noalloc, op, _lib.GFD_FLOAT32, b, rho,
               _lib.GFD_RELAX_JACOBI, 3, 2.0 / 3.0, stream)
        torch.cuda.synchronize()
        got = b.cpu().numpy().astype(np.float64)
        assert rel_err(got, a.cpu().numpy().astype(np.float64)) < TOL, call
        ref = phi0.cpu().numpy().astype(np.float64)  # the float32-rounded inputs
        K.relax(_lib.GFD_RELAX_JACOBI, op.coef_p, op.offset_pc, gd.pbc_c, ref,
                rho.cpu().numpy().astype(np.float64), 3, 2.0 / 3.0)
        assert rel_err(got, ref) < TOL32, call


def test_noalloc_relax_size_limit(cuda):
    """128^3 float64 (exactly the 16 MiB scratch) is accepted; 129^3 float64
    is rejected with a message; 150^3 is accepted in float32 (4 bytes per
    point) and rejected in float64."""
    import torch
    from gpaw_b200 import _lib
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    null = ctypes.c_void_p(None)

    def grid(n):
        gd = GridDescriptor((n + 1,) * 3, ((n + 1) * 0.4,) * 3, 0)  # n^3 points
        return gd, Laplace(gd, -0.25 / np.pi, 1)

    gd, op = grid(128)
    phi = torch.zeros((128,) * 3, dtype=torch.float64, device=cuda)
    rho = torch.ones_like(phi)
    assert _call(_lib.lib.gfd_operator_relax_noalloc, op, _lib.GFD_FLOAT64, phi, rho,
                 _lib.GFD_RELAX_JACOBI, 1, 1.0, null) == _lib.GFD_OK, _lib.last_error()
    torch.cuda.synchronize()
    # one Jacobi sweep from zero with weight 1: phi = rho / c0 everywhere
    assert torch.allclose(phi, rho / op.get_diagonal_element(), rtol=1e-15, atol=0)
    del phi, rho

    gd, op = grid(129)
    phi = torch.zeros((129,) * 3, dtype=torch.float64, device=cuda)
    assert _call(_lib.lib.gfd_operator_relax_noalloc, op, _lib.GFD_FLOAT64, phi, phi,
                 _lib.GFD_RELAX_JACOBI, 1, 1.0, null) == _lib.GFD_EINVAL
    assert 'at most' in _lib.last_error()
    del phi

    gd, op = grid(150)
    phi = torch.zeros((150,) * 3, dtype=torch.float32, device=cuda)
    rho = torch.ones_like(phi)
    assert _call(_lib.lib.gfd_operator_relax_noalloc, op, _lib.GFD_FLOAT32, phi, rho,
                 _lib.GFD_RELAX_JACOBI, 1, 1.0, null) == _lib.GFD_OK, _lib.last_error()
    torch.cuda.synchronize()
    assert torch.allclose(phi, rho / op.get_diagonal_element(), rtol=1e-6, atol=0)
    phi64 = torch.zeros((150,) * 3, dtype=torch.float64, device=cuda)
    assert _call(_lib.lib.gfd_operator_relax_noalloc, op, _lib.GFD_FLOAT64, phi64, phi64,
                 _lib.GFD_RELAX_JACOBI, 1, 1.0, null) == _lib.GFD_EINVAL
