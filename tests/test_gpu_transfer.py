"""GPU parity of restriction and interpolation against the CPU oracle
(1e-13 relative in FP64) and the reference's conservation tests."""
import numpy as np
import pytest

from oracle import geometry as G
from oracle import kernels as K
from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-13


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def host(t):
    return t.detach().cpu().numpy()


def gpu_transform(cuda, gd, g2, nn, a, phases=None, dtype=None):
    import torch
    from gpaw_b200.transformers import Transformer
    t = dev(a, cuda)
    if dtype is not None:
        t = t.to(dtype)
    tr = Transformer(gd, g2, nn, t.dtype)
    out = torch.full(t.shape[:-3] + tuple(int(x) for x in g2.n_c), float('nan'),
                     dtype=t.dtype, device=cuda)
    tr.apply(t, out, phases)
    torch.cuda.synchronize()
    return host(out)


def product_grid(og):
    from gpaw_b200.grid_descriptor import GridDescriptor
    return GridDescriptor(og.N_c, og.cell_cv, og.pbc_c)


@pytest.mark.parametrize('tag', ['np', 'p'])
def test_golden_transformers(golden, cuda, tag):
    d = golden
    og = G.Grid(d['tr_%s_N' % tag], d['tr_%s_cell' % tag], d['tr_%s_pbc' % tag])
    gd = product_grid(og)
    for nn in (1, 2, 3, 4):
        for name, g2 in (('restrict', gd.coarsen()), ('interp', gd.refine())):
            out = gpu_transform(cuda, gd, g2, nn, d['tr_%s_in_r' % tag])
            assert rel_err(out, d['tr_%s_%s%d_r' % (tag, name, nn)]) < TOL, (name, nn)
            out = gpu_transform(cuda, gd, g2, nn, d['tr_%s_in_c' % tag], d['tr_%s_phase' % tag])
            assert rel_err(out, d['tr_%s_%s%d_c' % (tag, name, nn)]) < TOL, (name, nn)


@pytest.mark.parametrize('N,pbc', [((24, 16, 40), 1), ((24, 16, 40), 0), ((18, 22, 14), (1, 0, 1)),
                                   ((64, 48, 32), 0), ((10, 34, 70), 1)])
@pytest.mark.parametrize('nn', [1, 2, 3, 4])
def test_transform_shapes(cuda, N, pbc, nn):
    og = G.Grid(N, np.array(N) * 0.3, pbc)
    gd = product_grid(og)
    rng = np.random.default_rng(nn)
    a = rng.uniform(-1, 1, (2,) + tuple(og.n_c))
    ac = a + 1j * rng.uniform(-1, 1, a.shape)
    ph = G.bloch_phases(og, (0.25, -0.125, 0.3))
    for g2, o2 in ((gd.coarsen(), og.coarsen()), (gd.refine(), og.refine())):
        try:
            ref = K.transform(og, o2, nn, a)
        except AssertionError:
            continue  # the reference rejects this grid (coarse too small)
        assert rel_err(gpu_transform(cuda, gd, g2, nn, a), ref) < TOL
        assert rel_err(gpu_transform(cuda, gd, g2, nn, ac, ph), K.transform(og, o2, nn, ac, ph)) < TOL
        # FP32 variant against the FP64 oracle
        o32 = gpu_transform(cuda, gd, g2, nn, a, dtype=__import__('torch').float32)
        assert rel_err(o32.astype(float), ref) < 2e-6


def test_transformations_conserve_integral(cuda):
    """gpaw/test/transformations.py:9-48 on the GPU."""
    from gpaw_b200.grid_descriptor import GridDescriptor
    gd = GridDescriptor((20, 20, 20))
    rng = np.random.RandomState(8)
    a = rng.random_sample(tuple(gd.n_c))
    ac = rng.random_sample(tuple(gd.n_c)) + 1j * rng.random_sample(tuple(gd.n_c))
    for g2 in (gd.refine(), gd.coarsen()):
        for k in (2, 4, 6, 8):
            b = gpu_transform(cuda, gd, g2, k // 2, a)
            assert abs(a.sum() * gd.dv - b.sum() * g2.dv) < 1e-14
            b = gpu_transform(cuda, gd, g2, k // 2, ac, np.ones((3, 2), complex))
            assert abs(ac.sum() * gd.dv - b.sum() * g2.dv) < 1e-14


def test_batched_bands_112(cuda):
    """Band-batched restriction/interpolation at 112^3 <-> 224^3 (nn=3),
    periodic, on a few bands of the 256-band workload."""
    import torch
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.transformers import Transformer
    coarse = GridDescriptor((112,) * 3, (112 * 0.3,) * 3, 1)
    fine = coarse.refine()
    oc = G.Grid((112,) * 3, (112 * 0.3,) * 3, 1)
    of = oc.refine()
    rng = np.random.default_rng(4)
    a = rng.uniform(-1, 1, (2,) + tuple(coarse.n_c))
    ip = Transformer(coarse, fine, 3)
    t = dev(a, cuda)
    fine_t = torch.empty((2,) + tuple(int(x) for x in fine.n_c), dtype=torch.float64, device=cuda)
    ip.apply(t, fine_t)
    ref_f = K.transform(oc, of, 3, a, nthreads=8)
    assert rel_err(host(fine_t), ref_f) < TOL
    rs = Transformer(fine, coarse, 3)
    back = torch.empty_like(t)
    rs.apply(fine_t, back)
    assert rel_err(host(back), K.transform(of, oc, 3, ref_f, nthreads=8)) < TOL


@pytest.mark.parametrize('pbc', [0, (1, 0, 1), 1])
def test_pseudo_density_interpolation(cuda, pbc):
    """Density.interpolate (gpaw/density.py:217-235): two spins to the fine
    grid with nn = 3, renormalised to the pseudo charge unless every axis is
    periodic; against the oracle interpolation and the reference's formula."""
    import torch
    from gpaw_b200.density import interpolate_pseudo_density
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.transformers import Transformer
    og = G.Grid((24, 20, 28), (24 * 0.35, 20 * 0.35, 28 * 0.35), pbc)
    of = og.refine()
    gd = product_grid(og)
    fine = gd.refine()
    rng = np.random.default_rng(17)
    nt = rng.uniform(0, 1, (2,) + tuple(og.n_c))
    pseudo_charge = -3.75
    ref = K.transform(og, of, 3, nt, nthreads=8)
    if not og.pbc_c.all():
        ref = ref * (pseudo_charge / of.integrate(ref).sum())
    out = torch.empty((2,) + tuple(int(x) for x in fine.n_c), dtype=torch.float64, device=cuda)
    interpolate_pseudo_density(Transformer(gd, fine, 3), dev(nt, cuda), out, fine, pseudo_charge)
    torch.cuda.synchronize()
    assert rel_err(host(out), ref) < TOL
    if not og.pbc_c.all():
        assert abs(of.integrate(host(out)).sum() - pseudo_charge) < 1e-12


_RESTRICT_SCRIPT = r'''
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + '/tests')
import torch
from oracle import geometry as G
from oracle import kernels as K
from conftest import rel_err
from test_gpu_transfer import gpu_transform, product_grid
cuda = torch.device('cuda', 0)
out = []
for N, pbc in (((24, 16, 40), 1), ((24, 16, 40), 0), ((18, 22, 14), (1, 0, 1)),
               ((70, 36, 98), 1), ((66, 34, 40), 0)):
    og = G.Grid(N, np.array(N) * 0.3, pbc)
    gd = product_grid(og)
    g2, o2 = gd.coarsen(), og.coarsen()
    rng = np.random.default_rng(sum(N))
    a = rng.uniform(-1, 1, (3,) + tuple(og.n_c))
    ac = a + 1j * rng.uniform(-1, 1, a.shape)
    ph = G.bloch_phases(og, (0.25, -0.125, 0.3))
    for nn in (1, 2, 3, 4):
        try:
            ref = K.transform(og, o2, nn, a)
        except AssertionError:
            continue  # the reference rejects this grid (coarse too small)
        e64 = rel_err(gpu_transform(cuda, gd, g2, nn, a), ref)
        e32 = rel_err(gpu_transform(cuda, gd, g2, nn, a, dtype=torch.float32).astype(float), ref)
        refc = K.transform(og, o2, nn, ac, ph)
        ec = rel_err(gpu_transform(cuda, gd, g2, nn, ac, ph), refc)
        ec64 = rel_err(gpu_transform(cuda, gd, g2, nn, ac, ph, dtype=torch.complex64), refc)
        out.append([list(N), nn, e64, e32, ec, ec64])
print('RESULT ' + json.dumps(out))
'''


def test_marching_restriction(cuda):
    """With GFD_DIRECT_MAX=0 every restriction, however small, takes the
    marching kernel.  Against the oracle for k = 2..8, float64/complex128
    within 1e-13, float32/complex64 within 2e-6, periodic, zero and mixed
    boundaries, Bloch phases, tiles cut at every edge."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, GFD_DIRECT_MAX='0')
    r = subprocess.run([sys.executable, '-c', _RESTRICT_SCRIPT, root], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    line = [x for x in r.stdout.splitlines() if x.startswith('RESULT ')][-1]
    for N, nn, e64, e32, ec, ec64 in json.loads(line[len('RESULT '):]):
        assert e64 < TOL and ec < TOL, (N, nn, e64, ec)
        assert e32 < 2e-6 and ec64 < 2e-6, (N, nn, e32, ec64)
