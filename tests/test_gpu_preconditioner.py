"""The band preconditioner (gpaw/preconditioner.py:13-70) on the GPU against
its step-by-step restatement in the oracle: 1e-13 relative in FP64 (the
device regroups the nineteen array operations into eight passes, so the
results agree to rounding), 2e-6 for the FP32 variants."""
import numpy as np
import pytest

from oracle import geometry as G
from oracle.preconditioner import Preconditioner as OraclePC
from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-13
BOHR = G.BOHR


class KPoint:
    def __init__(self, phase_cd):
        self.phase_cd = phase_cd


CASES = [('c128_p48', (48, 48, 48), 1, complex, (0.25, 0.0, 0.0), 4, 3),
         ('c128_mixed', (40, 32, 48), (1, 0, 1), complex, (0.1, 0.0, -0.3), 3, 2),
         ('f64_np40', (40, 40, 40), 0, float, None, 2, 3),
         ('f64_p96', (96, 96, 96), 1, float, None, 2, 3)]


@pytest.mark.parametrize('tag,N,pbc,dtype,k,nb,nn', CASES)
def test_preconditioner_matches_oracle(cuda, tag, N, pbc, dtype, k, nb, nn):
    import torch
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.preconditioner import Preconditioner
    og = G.Grid(N, np.array(N) * 0.2 / BOHR, pbc)
    gd = GridDescriptor(og.N_c, og.cell_cv, og.pbc_c)
    rng = np.random.default_rng(sum(map(ord, tag)))
    shape = (nb,) + tuple(og.n_c)
    R = rng.standard_normal(shape)
    if dtype is complex:
        R = R + 1j * rng.standard_normal(shape)
    ph = G.bloch_phases(og, k) if k is not None else None
    kin0 = Laplace(gd, -0.5, nn, dtype)
    ref = OraclePC(og, (kin0.coef_p, kin0.offset_pc))(R, ph)
    pc = Preconditioner(gd, kin0, dtype, block=nb + 1)
    t = torch.from_numpy(R).to(cuda)
    out = pc(t, KPoint(ph))
    torch.cuda.synchronize()
    assert out.shape == t.shape
    assert rel_err(out.cpu().numpy(), ref) < TOL
    # one band at a time gives the same bands
    one = pc(t[1].contiguous(), KPoint(ph)).cpu().numpy()
    assert rel_err(one, ref[1]) < TOL
    # FP32 variant against the FP64 oracle
    d32 = np.complex64 if dtype is complex else np.float32
    kin32 = Laplace(gd, -0.5, nn, d32)
    pc32 = Preconditioner(gd, kin32, d32, block=nb)
    o32 = pc32(t.to(torch.complex64 if dtype is complex else torch.float32), KPoint(ph))
    assert rel_err(o32.cpu().numpy().astype(ref.dtype), ref) < 2e-6


def test_preconditioner_rejects_bad_input(cuda):
    import torch
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.preconditioner import Preconditioner
    gd = GridDescriptor((16, 16, 16), (4.0, 4.0, 4.0), 1)
    pc = Preconditioner(gd, Laplace(gd, -0.5, 2, complex), complex, block=2)
    with pytest.raises(ValueError):
        pc(torch.zeros((3, 16, 16, 16), dtype=torch.complex128, device=cuda))  # > block
    with pytest.raises(ValueError):
        pc(torch.zeros((2, 16, 16, 16), dtype=torch.float64, device=cuda))  # dtype
    with pytest.raises(ValueError):
        pc(torch.zeros((2, 8, 16, 16), dtype=torch.complex128, device=cuda))  # shape
