"""GPU parity of the finite-difference operators against the CPU oracle.

Bar (FP64): max|gpu - oracle| / max|oracle| <= 1e-13, the tolerance of
the stencil path; FP32 variants are checked against the FP64 oracle at 2e-6.
"""
import numpy as np
import pytest

from oracle import geometry as G
from oracle import kernels as K
from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-13
BOHR = G.BOHR


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def host(t):
    return t.detach().cpu().numpy()


def gpu_apply(cuda, gd_args, coefs, offsets, a, phase=None, dtype=None):
    import torch
    from gpaw_b200.fd_operators import FDOperator
    from gpaw_b200.grid_descriptor import GridDescriptor
    gd = GridDescriptor(*gd_args)
    t = dev(a, cuda)
    if dtype is not None:
        t = t.to(dtype)
    op = FDOperator(coefs, offsets, gd, t.dtype)
    out = torch.empty_like(t)
    op.apply(t, out, phase)
    torch.cuda.synchronize()
    return host(out)


@pytest.mark.parametrize('tag', ['np', 'p', 'mx'])
def test_golden_stencils(golden, cuda, tag):
    d = golden
    args = (d['stencil_%s_N' % tag], d['stencil_%s_cell' % tag], d['stencil_%s_pbc' % tag])
    a_r, a_c, ph = d['stencil_%s_in_r' % tag], d['stencil_%s_in_c' % tag], d['stencil_%s_phase' % tag]
    for n in (1, 2, 3):
        c, o = d['lap%d_%s_coefs' % (n, tag)], d['lap%d_%s_offsets' % (n, tag)]
        assert rel_err(gpu_apply(cuda, args, c, o, a_r), d['lap%d_%s_out_r' % (n, tag)]) < TOL
        assert rel_err(gpu_apply(cuda, args, c, o, a_c, ph), d['lap%d_%s_out_c' % (n, tag)]) < TOL
    for v in range(3):
        c, o = d['grad%d_%s_coefs' % (v, tag)], d['grad%d_%s_offsets' % (v, tag)]
        assert rel_err(gpu_apply(cuda, args, c, o, a_c, ph), d['grad%d_%s_out_c' % (v, tag)]) < TOL


def test_golden_cross_stencil(golden, cuda):
    d = golden
    out = gpu_apply(cuda, (d['hex_N'], d['hex_cell'], 1), d['hex_coefs'], d['hex_offsets'],
                    d['hex_in'], d['hex_phase'])
    assert rel_err(out, d['hex_out']) < TOL


def test_plain_fp64_laplace_48(cuda):
    """16 float64 bands on a 48^3 zero-boundary grid, h = 0.2 A, nn = 3,
    scale = -0.5, values U[-1, 1] from seed 1."""
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    import torch
    N = 48
    gd = GridDescriptor((N,) * 3, (N * 0.2 / BOHR,) * 3, 0)
    a = np.random.default_rng(1).uniform(-1, 1, (16,) + tuple(gd.n_c))
    lap = Laplace(gd, -0.5, 3)
    t = dev(a, cuda)
    out = torch.empty_like(t)
    lap.apply(t, out)
    ref = K.fd_apply(lap.coef_p, lap.offset_pc, gd.pbc_c, a, nthreads=8)
    assert rel_err(host(out), ref) < TOL


@pytest.mark.parametrize('kind', ['laplace', 'gradient0', 'gradient1', 'gradient2'])
def test_bloch_complex_96(cuda, kind):
    """Complex128 bands on a 96^3 periodic grid, h = 0.18 A, phases for
    k = (0.25, 0, 0); a few bands of the band-batched workload."""
    from gpaw_b200.fd_operators import Gradient, Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    import torch
    N = 96
    gd = GridDescriptor((N,) * 3, (N * 0.18 / BOHR,) * 3, 1)
    rng = np.random.default_rng(2)
    a = rng.standard_normal((3,) + tuple(gd.n_c)) + 1j * rng.standard_normal((3,) + tuple(gd.n_c))
    ph = np.exp(2j * np.pi * gd.sdisp_cd * np.array([0.25, 0, 0])[:, None])
    assert abs(ph[0, 0] - 1j) < 1e-15 and abs(ph[0, 1] + 1j) < 1e-15
    op = Laplace(gd, -0.5, 3, complex) if kind == 'laplace' else Gradient(gd, int(kind[-1]), 1.0, 3, complex)
    t = dev(a, cuda)
    out = torch.empty_like(t)
    op.apply(t, out, ph)
    ref = K.fd_apply(op.coef_p, op.offset_pc, gd.pbc_c, a, ph, nthreads=8)
    assert rel_err(host(out), ref) < TOL
    # FP32 variant (complex64) against the FP64 oracle
    op32 = Laplace(gd, -0.5, 3, np.complex64) if kind == 'laplace' else \
        Gradient(gd, int(kind[-1]), 1.0, 3, np.complex64)
    t32 = t.to(torch.complex64)
    o32 = torch.empty_like(t32)
    op32.apply(t32, o32, ph)
    assert rel_err(host(o32).astype(complex), ref) < 2e-6


SHAPES = [((5, 7, 9), 0), ((5, 7, 9), 1), ((33, 17, 65), (1, 0, 1)), ((3, 40, 3), 1),
          ((2, 2, 8), (0, 0, 1)), ((70, 9, 31), 0), ((12, 12, 12), 1)]


@pytest.mark.parametrize('N,pbc', SHAPES)
@pytest.mark.parametrize('n', [1, 2, 3, 4, 5, 6])
def test_ragged_shapes_all_orders(cuda, N, pbc, n):
    """Partial tiles, tiny and odd grids, every stencil order, real and
    phased complex, several bands and one bare 3-D array."""
    gd = G.Grid(N, np.array(N) * 0.25, pbc)
    mp = n
    if any(p and s < mp for p, s in zip(gd.pbc_c, gd.n_c)):
        pytest.skip('periodic axis shorter than the stencil')
    c, o = G.laplace_stencil(gd, 1.3, n)
    rng = np.random.default_rng(n)
    a = rng.standard_normal((2,) + tuple(gd.n_c))
    args = (gd.N_c, gd.cell_cv, gd.pbc_c)
    assert rel_err(gpu_apply(cuda, args, c, o, a), K.fd_apply(c, o, gd.pbc_c, a)) < TOL
    ac = a + 1j * rng.standard_normal(a.shape)
    ph = G.bloch_phases(gd, (0.17, -0.31, 0.4))
    assert rel_err(gpu_apply(cuda, args, c, o, ac, ph), K.fd_apply(c, o, gd.pbc_c, ac, ph)) < TOL
    assert rel_err(gpu_apply(cuda, args, c, o, a[0]), K.fd_apply(c, o, gd.pbc_c, a[0])) < TOL


def test_empty_band_batch_and_errors(cuda):
    import torch
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    gd = GridDescriptor((8, 8, 8), (2.0, 2.0, 2.0), 1)
    lap = Laplace(gd, -0.5, 2)
    a = torch.zeros((0, 8, 8, 8), dtype=torch.float64, device=cuda)
    lap.apply(a, torch.empty_like(a))  # nothing to do
    b = torch.zeros((8, 8, 8), dtype=torch.float64, device=cuda)
    with pytest.raises(ValueError):
        lap.apply(b, torch.zeros((8, 8, 7), dtype=torch.float64, device=cuda))
    with pytest.raises(ValueError):
        lap.apply(b.to(torch.complex128), torch.zeros_like(b.to(torch.complex128)))
    with pytest.raises(ValueError):
        lap.apply(b, b)  # in-place apply is not allowed


def test_canary_around_output(cuda):
    """Writes stay inside the output: guard values around it survive."""
    import torch
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    gd = GridDescriptor((13, 11, 17), (4.0, 3.5, 5.0), 0)
    lap = Laplace(gd, -0.5, 3)
    n = int(np.prod(gd.n_c))
    a = torch.randn((3, n), dtype=torch.float64, device=cuda).reshape(3, 13 - 1, 11 - 1, 17 - 1)
    buf = torch.full((3 * n + 2048,), 7.25, dtype=torch.float64, device=cuda)
    out = buf[1024:1024 + 3 * n].view(a.shape)
    lap.apply(a, out)
    torch.cuda.synchronize()
    assert bool((buf[:1024] == 7.25).all()) and bool((buf[1024 + 3 * n:] == 7.25).all())


@pytest.mark.parametrize('tag', ['np', 'p'])
def test_golden_jacobi_relax(golden, cuda, tag):
    from gpaw_b200.fd_operators import FDOperator
    from gpaw_b200.grid_descriptor import GridDescriptor
    d = golden
    gd = GridDescriptor(d['relax_%s_N' % tag], d['relax_%s_cell' % tag], d['relax_%s_pbc' % tag])
    op = FDOperator(d['relax_%s_coefs' % tag], d['relax_%s_offsets' % tag], gd)
    phi = dev(d['relax_%s_phi0' % tag], cuda)
    op.relax(2, phi, dev(d['relax_%s_rho' % tag], cuda), 3, 2.0 / 3.0)
    ref = d['relax_%s_jacobi3' % tag]
    assert rel_err(host(phi), ref) < TOL


def multicolour_gs_reference(c, o, pbc, phi, rho, nsweeps):
    """Multicolour Gauss-Seidel on the CPU with the oracle's stencil: colour
    (i0+i1+i2) mod (range+1); wrapped neighbours from the sweep-start copy."""
    phi = phi.copy()
    mp = int(np.abs(o).max())
    ncol = mp + 1
    idx = np.indices(phi.shape).sum(0) % ncol
    cn = c.copy()
    cn[0] = 0.0
    zero = np.zeros(3, bool)
    for _ in range(nsweeps):
        frozen = phi.copy()
        wrapped = K.fd_apply(cn, o, pbc, frozen) - K.fd_apply(cn, o, zero, frozen)
        for col in range(ncol):
            s = K.fd_apply(cn, o, zero, phi) + wrapped
            m = idx == col
            phi[m] = ((rho - s) * (1.0 / c[0]))[m]
    return phi


@pytest.mark.parametrize('tag', ['np', 'p'])
def test_multicolour_gauss_seidel(golden, cuda, tag):
    from gpaw_b200.fd_operators import FDOperator
    from gpaw_b200.grid_descriptor import GridDescriptor
    d = golden
    gd = GridDescriptor(d['relax_%s_N' % tag], d['relax_%s_cell' % tag], d['relax_%s_pbc' % tag])
    c, o = d['relax_%s_coefs' % tag], d['relax_%s_offsets' % tag]
    op = FDOperator(c, o, gd)
    phi = dev(d['relax_%s_phi0' % tag], cuda)
    op.relax(1, phi, dev(d['relax_%s_rho' % tag], cuda), 2)
    ref = multicolour_gs_reference(c, o, gd.pbc_c, d['relax_%s_phi0' % tag],
                                   d['relax_%s_rho' % tag], 2)
    assert rel_err(host(phi), ref) < TOL


BLOCKED_SHAPES = [((24, 16, 33), 1), ((40, 20, 36), 1), ((40, 20, 36), 0), ((17, 18, 40), (0, 1, 1)),
                  ((9, 33, 64), (1, 1, 0))]


@pytest.mark.parametrize('N,pbc', BLOCKED_SHAPES)
@pytest.mark.parametrize('n', [1, 2, 3])
def test_register_blocked_tiles(cuda, N, pbc, n):
    """Grids at least 16 x 32 in the plane (the register-blocked kernel for
    8- and 16-byte values): partial tiles, halos wrapping more than once on a
    narrow periodic axis, Bloch phases on every axis; float64, complex128 and
    complex64, and weighted-Jacobi sweeps."""
    import torch
    from gpaw_b200.fd_operators import FDOperator
    from gpaw_b200.grid_descriptor import GridDescriptor
    gd = G.Grid(N, np.array(N) * 0.3, pbc)
    c, o = G.laplace_stencil(gd, -0.5, n)
    rng = np.random.default_rng(10 + n)
    a = rng.standard_normal((3,) + tuple(gd.n_c))
    args = (gd.N_c, gd.cell_cv, gd.pbc_c)
    assert rel_err(gpu_apply(cuda, args, c, o, a), K.fd_apply(c, o, gd.pbc_c, a)) < TOL
    ac = a + 1j * rng.standard_normal(a.shape)
    ph = G.bloch_phases(gd, (0.3, -0.2, 0.15))
    ref = K.fd_apply(c, o, gd.pbc_c, ac, ph)
    assert rel_err(gpu_apply(cuda, args, c, o, ac, ph), ref) < TOL
    o64 = gpu_apply(cuda, args, c, o, ac, ph, dtype=torch.complex64)
    assert rel_err(o64.astype(complex), ref) < 2e-6
    # three weighted-Jacobi sweeps on one band
    op = FDOperator(c, o, GridDescriptor(*args))
    phi0, rho = a[0], a[1]
    phi = dev(phi0, cuda)
    op.relax(2, phi, dev(rho, cuda), 3, 2.0 / 3.0)
    p = phi0.copy()
    K.relax(2, c, o, gd.pbc_c, p, rho, 3, 2.0 / 3.0)
    assert rel_err(host(phi), p) < TOL


TMA_SHAPES = [((40, 32, 64), 1), ((24, 48, 96), (1, 1, 0)), ((20, 16, 32), (0, 1, 1)),
              ((18, 37, 70), 0), ((96, 96, 96), 1)]


@pytest.mark.parametrize('N,pbc', TMA_SHAPES)
@pytest.mark.parametrize('n', [1, 2, 3])
def test_complex128_tiles_all_boundaries(cuda, N, pbc, n):
    """complex128 bands on grids of whole 16 x 32 plane tiles along periodic
    axes (and ragged zero-boundary axes): Bloch phases on all three axes,
    Laplace and a gradient, then the device error flags stay clear."""
    import ctypes
    from gpaw_b200 import _lib
    gd = G.Grid(N, np.array(N) * 0.3, pbc)
    rng = np.random.default_rng(20 + n)
    nb = 2 if N[0] < 96 else 1
    a = rng.standard_normal((nb,) + tuple(gd.n_c)) + 1j * rng.standard_normal((nb,) + tuple(gd.n_c))
    args = (gd.N_c, gd.cell_cv, gd.pbc_c)
    for k in ((0.3, -0.2, 0.15), (0.25, 0.0, 0.0)):
        ph = G.bloch_phases(gd, k)
        for c, o in (G.laplace_stencil(gd, -0.5, n), G.gradient_stencil(gd, 2, 1.0, n)):
            ref = K.fd_apply(c, o, gd.pbc_c, a, ph, nthreads=8)
            assert rel_err(gpu_apply(cuda, args, c, o, a, ph), ref) < TOL, k
    flags = ctypes.c_int(-1)
    assert _lib.lib.gfd_device_errors(ctypes.byref(flags)) == 0
    assert flags.value == 0


def test_tma_fed_kernel_in_subprocess(cuda):
    """The TMA-fed complex128 kernel (opt-in with GFD_STAR_TMA=1, read once
    per process) against the oracle: the tile tests above in a child process
    with the switch on."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, GFD_STAR_TMA='1')
    r = subprocess.run([sys.executable, '-m', 'pytest', '-q', '-m', 'gpu', '-p', 'no:cacheprovider',
                        os.path.join(root, 'tests', 'test_gpu_stencil.py'),
                        '-k', 'complex128_tiles or bloch_complex_96'],
                       cwd=root, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert ' passed' in r.stdout


@pytest.mark.parametrize('case', ['bloch96', 'plain48', 'small', 'hex'])
def test_pseudo_hamiltonian_fused(cuda, case):
    """kin psit + vt psit in one pass against the oracle stencil plus the
    reference's numpy update Htpsit += psit * vt (gpaw/hamiltonian.py:
    395-398): complex128 Bloch bands on 96^3 (marching kernel), float64 on
    47^3 zero boundary, a small grid (one-thread-per-point kernel) and a
    hexagonal cell (cross terms: stencil, then the potential pass)."""
    import torch
    from gpaw_b200.fd_operators import FDOperator
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import apply_pseudo_hamiltonian
    rng = np.random.default_rng(31)
    if case == 'bloch96':
        gd = G.Grid((96,) * 3, (96 * 0.18 / BOHR,) * 3, 1)
        shape = (2,) + tuple(gd.n_c)
        a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        ph = G.bloch_phases(gd, (0.25, 0.0, 0.0))
    elif case == 'plain48':
        gd = G.Grid((48,) * 3, (48 * 0.2 / BOHR,) * 3, 0)
        a = rng.uniform(-1, 1, (3,) + tuple(gd.n_c))
        ph = None
    elif case == 'small':
        gd = G.Grid((12, 10, 14), (3.6, 3.0, 4.2), (1, 0, 1))
        a = rng.standard_normal((2,) + tuple(gd.n_c)) + 1j * rng.standard_normal((2,) + tuple(gd.n_c))
        ph = G.bloch_phases(gd, (0.1, 0.0, -0.3))
    else:
        gd = G.Grid((8, 8, 8), np.array([(1, 0, 0), (0.5, 3 ** 0.5 / 2, 0), (0, 0, 1.1)]) * 4.0, 1)
        a = rng.standard_normal((2,) + tuple(gd.n_c)) + 1j * rng.standard_normal((2,) + tuple(gd.n_c))
        ph = G.bloch_phases(gd, (0.1, -0.2, 0.3))
    c, o = G.laplace_stencil(gd, -0.5, 3 if case != 'hex' else 2)
    vt = rng.uniform(-2, 1, tuple(gd.n_c))
    ref = K.fd_apply(c, o, gd.pbc_c, a, ph, nthreads=8) + a * vt
    gdp = GridDescriptor(gd.N_c, gd.cell_cv, gd.pbc_c)
    t = dev(a, cuda)
    kin = FDOperator(c, o, gdp, t.dtype)
    out = torch.empty_like(t)
    apply_pseudo_hamiltonian(kin, t, out, dev(vt, cuda), ph)
    assert rel_err(host(out), ref) < TOL
    # FP32 variant against the FP64 oracle
    t32 = t.to(torch.complex64 if t.is_complex() else torch.float32)
    kin32 = FDOperator(c, o, gdp, t32.dtype)
    o32 = torch.empty_like(t32)
    kin32.apply_with_potential(t32, o32, dev(vt, cuda).float(), ph)
    assert rel_err(host(o32).astype(ref.dtype), ref) < 2e-6
    with pytest.raises(ValueError):
        kin.apply_with_potential(t, out, dev(vt, cuda).float(), ph)  # wrong potential dtype


def test_host_streamer_matches_device_apply(cuda):
    """Bands in pinned host memory through HostStreamer (copies and kernels
    overlapped in chunks, a ragged last chunk) give the device apply's
    result, with and without the local potential (to the stencil tolerance:
    an 8-band chunk of 32^3 takes the one-thread-per-point kernel, the
    37-band call the marching one)."""
    import torch
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.streaming import HostStreamer
    gd = GridDescriptor((32, 32, 32), (32 * 0.3,) * 3, 1)
    lap = Laplace(gd, -0.5, 3, complex)
    rng = np.random.default_rng(3)
    a = rng.standard_normal((37, 32, 32, 32)) + 1j * rng.standard_normal((37, 32, 32, 32))
    ph = np.exp(2j * np.pi * gd.sdisp_cd * np.array([0.25, 0, 0])[:, None])
    host_in = torch.from_numpy(a).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    ref = torch.empty((37, 32, 32, 32), dtype=torch.complex128, device=cuda)
    t = host_in.to(cuda)
    lap.apply(t, ref, ph)
    st = HostStreamer(lap, chunk_bands=8)
    st.apply(host_in, host_out, ph)
    torch.cuda.synchronize()
    assert rel_err(host_out.numpy(), host(ref)) < TOL
    vt = torch.rand((32, 32, 32), dtype=torch.float64, device=cuda)
    lap.apply_with_potential(t, ref, vt, ph)
    st.apply(host_in, host_out, ph, vt)
    torch.cuda.synchronize()
    assert rel_err(host_out.numpy(), host(ref)) < TOL
    with pytest.raises(ValueError):
        st.apply(t, ref, ph)  # device tensors


@pytest.mark.parametrize('switches', [{'GFD_TMASPLIT': '0'},
                                      {'GFD_TMASPLIT': '0', 'GFD_SPLIT': '0'}])
def test_other_complex_kernels_in_subprocess(cuda, switches):
    """complex128 bands up to radius 3 take the TMA-staged lane-pair kernel
    (star_tmasplit_kernel) where it applies; GFD_TMASPLIT=0 (read once per
    process) moves them to the cp.async lane-pair kernel (star_split_kernel,
    also the complex64 kernel), and GFD_SPLIT=0 as well to star_kernel.  The
    complex tests above, the pseudo-Hamiltonian and the preconditioner in a
    child process with the switches, so every kernel stays checked against
    the oracle."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, **switches)
    r = subprocess.run([sys.executable, '-m', 'pytest', '-q', '-m', 'gpu', '-p', 'no:cacheprovider',
                        os.path.join(root, 'tests', 'test_gpu_stencil.py'),
                        os.path.join(root, 'tests', 'test_gpu_preconditioner.py'),
                        '-k', 'complex128_tiles or bloch_complex_96 or register_blocked or '
                              'pseudo_hamiltonian or preconditioner'],
                       cwd=root, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert ' passed' in r.stdout


def test_bounded_wait_runs_out_and_reports(cuda):
    """The kernels' bounded mbarrier wait, made to run out: a probe kernel
    waits (limit 100000 SM cycles) on a barrier nothing completes, returns,
    and gfd_device_errors reports the flag once and then reads clear; the
    context stays usable (a stencil apply afterwards matches the oracle)."""
    import ctypes
    from gpaw_b200 import _lib
    flags = ctypes.c_int(-1)
    assert _lib.lib.gfd_device_errors(ctypes.byref(flags)) == 0  # clear any earlier flag
    assert _lib.lib.gfd_wait_selftest(100000) == _lib.GFD_OK, _lib.last_error()
    assert _lib.lib.gfd_device_errors(ctypes.byref(flags)) == 0
    assert flags.value == 1
    assert _lib.lib.gfd_device_errors(ctypes.byref(flags)) == 0
    assert flags.value == 0
    assert _lib.lib.gfd_wait_selftest(0) == _lib.GFD_EINVAL
    gd = G.Grid((20, 16, 40), np.array((20, 16, 40)) * 0.3, 1)
    c, o = G.laplace_stencil(gd, -0.5, 3)
    rng = np.random.default_rng(2)
    a = rng.standard_normal((1,) + tuple(gd.n_c)) + 1j * rng.standard_normal((1,) + tuple(gd.n_c))
    ph = G.bloch_phases(gd, (0.2, 0.1, -0.3))
    args = (gd.N_c, gd.cell_cv, gd.pbc_c)
    assert rel_err(gpu_apply(cuda, args, c, o, a, ph), K.fd_apply(c, o, gd.pbc_c, a, ph)) < TOL
