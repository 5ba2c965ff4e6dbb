"""Host-side logic and the C ABI, without a GPU.

* libgpawfd.so loads and exports every function include/gpaw_fd.h declares;
* handle constructors validate their arguments (host-only calls);
* the product's coefficient builders, grid descriptor and transformer
  paddings agree with the oracle's restatement of the reference.
"""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import geometry as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, 'include', 'gpaw_fd.h')).read()
    return sorted(set(re.findall(r'GFD_API\s+[\w\s\*]+?\b(gfd_\w+)\s*\(', text)))


def test_library_exports_every_declared_symbol():
    from gpaw_b200 import _lib
    names = header_functions()
    assert len(names) >= 14
    raw = ctypes.CDLL(_lib.LIB_PATH)
    for name in names:
        assert hasattr(raw, name), name
    assert set(names) == set(_lib.SIGNATURES)
    assert _lib.lib.gfd_version().startswith(b'gpaw-fd-b200')


def _create_op(coefs, offsets, size, rng=None, nbr=None, real=1):
    from gpaw_b200 import _lib
    c, cp = _lib.f64(coefs)
    o, op = _lib.i64(offsets)
    s, sp = _lib.i64(size)
    n, np_ = _lib.i64(nbr if nbr is not None else [-1] * 6)
    h = _lib._vp()
    mp = int(np.abs(np.asarray(offsets)).max())
    st = _lib.lib.gfd_operator_create(len(c), cp, op, sp, mp if rng is None else rng, np_, real, 1,
                                      ctypes.byref(h))
    return st, h


def test_operator_create_validates_arguments():
    from gpaw_b200 import _lib
    st, h = _create_op([-6.0, 1, 1, 1, 1, 1, 1],
                       [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1),
                        (0, 0, -1)], (8, 8, 8))
    assert st == _lib.GFD_OK and h.value
    d = ctypes.c_double()
    assert _lib.lib.gfd_operator_get_diagonal_element(h, ctypes.byref(d)) == 0 and d.value == -6.0
    assert _lib.lib.gfd_operator_destroy(h) == 0
    # range smaller than the offsets
    st, _ = _create_op([1.0, 1.0], [(0, 0, 0), (2, 0, 0)], (8, 8, 8), rng=1)
    assert st == _lib.GFD_EINVAL and 'range' in _lib.last_error()
    # periodic axis shorter than the halo
    st, _ = _create_op([1.0, 1.0], [(0, 0, 0), (3, 0, 0)], (2, 8, 8), nbr=[0] * 6)
    assert st == _lib.GFD_EINVAL
    # another MPI rank as neighbour: no domain decomposition
    st, _ = _create_op([1.0], [(0, 0, 0)], (8, 8, 8), nbr=[1, 1, -1, -1, -1, -1])
    assert st == _lib.GFD_EUNSUPPORTED
    # zero-size grid
    st, _ = _create_op([1.0], [(0, 0, 0)], (0, 8, 8))
    assert st == _lib.GFD_EINVAL


def test_transformer_create_checks_sizes():
    from gpaw_b200 import _lib
    gd = G.Grid((16, 12, 20), (8.0, 6.0, 10.0), 0)
    for g2 in (gd.coarsen(), gd.refine()):
        for nn in (1, 2, 3):
            pad, npad, skip, interp = G.transformer_layout(gd, g2, nn)
            args = [_lib.i64(x) for x in (gd.n_c, g2.n_c, pad, npad, skip, gd.neighbor_cd)]
            h = _lib._vp()
            st = _lib.lib.gfd_transformer_create(args[0][1], args[1][1], 2 * nn, args[2][1],
                                                 args[3][1], args[4][1], args[5][1], 1,
                                                 int(interp), ctypes.byref(h))
            assert st == 0, _lib.last_error()
            _lib.lib.gfd_transformer_destroy(h)
            # a wrong output size is rejected
            bad = [_lib.i64(x) for x in (np.array(g2.n_c) + 1,)]
            st = _lib.lib.gfd_transformer_create(args[0][1], bad[0][1], 2 * nn, args[2][1],
                                                 args[3][1], args[4][1], args[5][1], 1,
                                                 int(interp), ctypes.byref(h))
            assert st == _lib.GFD_EINVAL


CELLS = [((12, 12, 12), (3.6, 3.6, 3.6)),
         ((8, 10, 12), (2.4, 3.0, 3.9)),
         ((8, 8, 8), [(1, 0, 0), (0.5, 3 ** 0.5 / 2, 0), (0, 0, 1.1)]),
         ((6, 6, 6), [(0, 1, 1), (1, 0, 1), (1, 1, 0)]),
         ((6, 6, 6), [(-1, 1, 1), (1, -1, 1), (1, 1, -1)])]


@pytest.mark.parametrize('N,cell', CELLS)
def test_coefficients_match_oracle(N, cell):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Gradient, Laplace
    gd = GridDescriptor(N, cell, True)
    og = G.Grid(N, cell, True)
    for n in range(1, 7):
        op = Laplace(gd, -0.5, n, allocate=False)
        c, o = G.laplace_stencil(og, -0.5, n)
        assert np.array_equal(op.offset_pc, o)
        assert np.abs(op.coef_p - c).max() <= 1e-14 * np.abs(c).max()
    for v in range(3):
        for n in (1, 3, 5):
            op = Gradient(gd, v, 1.0, n, allocate=False)
            c, o = G.gradient_stencil(og, v, 1.0, n)
            assert np.array_equal(op.offset_pc, o)
            assert np.abs(op.coef_p - c).max() <= 1e-14 * np.abs(c).max()


@pytest.mark.parametrize('pbc', [0, 1, (1, 0, 1)])
def test_grid_descriptor_and_transformer_layout(pbc):
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.transformers import Transformer
    gd = GridDescriptor((16, 12, 20), (8.0, 6.0, 10.0), pbc)
    og = G.Grid((16, 12, 20), (8.0, 6.0, 10.0), pbc)
    for attr in ('n_c', 'beg_c', 'end_c', 'h_cv', 'neighbor_cd', 'sdisp_cd', 'xxxiucell_cv'):
        assert np.allclose(getattr(gd, attr), getattr(og, attr), rtol=0, atol=0), attr
    assert gd.dv == og.dv
    assert np.array_equal(gd.get_size_of_global_array(), og.global_size())
    for g2, o2 in ((gd.coarsen(), og.coarsen()), (gd.refine(), og.refine())):
        for nn in (1, 2, 3, 4):
            t = Transformer(gd, g2, nn, allocate=False)
            pad, npad, skip, interp = G.transformer_layout(og, o2, nn)
            assert np.array_equal(t.pad_cd, pad) and np.array_equal(t.neighborpad_cd, npad)
            assert np.array_equal(t.skip_cd, skip) and t.interpolate == interp


def test_poisson_hierarchy_matches_reference_rules():
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.poisson import PoissonSolver
    from oracle.poisson import PoissonSolver as OraclePS
    for N, pbc in ((128, 0), (48, 0), (20, 1), (6, 0)):
        gd = GridDescriptor((N,) * 3, (N * 0.38,) * 3, pbc)
        ps = PoissonSolver(nn=3)
        ps.set_grid_descriptor(gd)
        ops = OraclePS(3)
        ops.set_grid_descriptor(G.Grid((N,) * 3, (N * 0.38,) * 3, pbc))
        assert ps.levels == ops.levels
        assert ps.presmooths == ops.presmooths and ps.postsmooths == ops.postsmooths
        assert ps.weights == ops.weights
        for a, (c, o) in zip(ps.operators, ops.stencils):
            assert np.array_equal(a.offset_pc, o)
            assert np.abs(a.coef_p - c).max() <= 1e-14 * np.abs(c).max()


def test_no_cpu_path_for_host_tensors():
    """Product calls reject host tensors instead of computing on the CPU."""
    import torch
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.fd_operators import Laplace
    gd = GridDescriptor((8, 8, 8), (2.0, 2.0, 2.0), 1, device='cpu')
    op = Laplace(gd, -0.5, 2)
    a = torch.zeros((8, 8, 8), dtype=torch.float64)
    with pytest.raises(ValueError, match='CUDA'):
        op.apply(a, torch.zeros_like(a))


def test_tune_cache_file_roundtrip(tmp_path):
    """The launch-plan cache loads, counts, saves, rejects malformed files and
    clears without touching a GPU; plans are looked up by operator key."""
    from gpaw_b200 import _lib
    lib = _lib.lib
    n = ctypes.c_int(-1)
    assert lib.gfd_autotune_clear() == 0
    good = tmp_path / 'plans.txt'
    good.write_text('gfd-tune 1\n# comment\n'
                    '0 1 0 96 96 96 3 7 9 1 0 2 1234.5\n'
                    '1 0 0 224 224 224 3 7 8 0 0 4 99.0\n')
    assert lib.gfd_autotune_load(str(good).encode()) == 0
    assert lib.gfd_autotune_count(ctypes.byref(n)) == 0 and n.value == 2
    st, h = _create_op([-3.0, 1, 1, 0.5, 0.5, 0.25, 0.25, 0.1, 0.1, 0.05, 0.05, 0.02, 0.02,
                        0.01, 0.01, 0.005, 0.005, 0.001, 0.001],
                       [(0, 0, 0)] + [tuple(s * k * e for e in np.eye(3, dtype=int)[a])
                                      for k in (1, 2, 3) for a in range(3) for s in (1, -1)],
                       (96, 96, 96), nbr=[0] * 6, real=0)
    assert st == 0
    plan = _lib.TunePlan()
    found = ctypes.c_int(0)
    assert lib.gfd_autotune_operator_plan(h, _lib.GFD_COMPLEX128, _lib.GFD_TUNE_APPLY, 512,
                                          ctypes.byref(plan), ctypes.byref(found)) == 0
    assert found.value == 1 and plan.as_dict() == {'form': 'march', 'tile': 32,
                                                   'ctas_per_sm': 2, 'us': 1234.5}
    assert lib.gfd_autotune_operator_plan(h, _lib.GFD_COMPLEX128, _lib.GFD_TUNE_APPLY, 256,
                                          ctypes.byref(plan), ctypes.byref(found)) == 0
    assert found.value == 0   # another band-count class
    lib.gfd_operator_destroy(h)
    out = tmp_path / 'saved.txt'
    assert lib.gfd_autotune_save(str(out).encode()) == 0
    lines = [ln.split() for ln in out.read_text().splitlines()[1:] if not ln.startswith('#')]
    assert sorted(tuple(map(float, ln)) for ln in lines) == sorted([
        (0, 1, 0, 96, 96, 96, 3, 7, 9, 1, 0, 2, 1234.5), (1, 0, 0, 224, 224, 224, 3, 7, 8, 0, 0, 4, 99.0)])
    for bad in ('not a cache\n', 'gfd-tune 1\n0 1 0 96 96 96 3 7 9 5 0 2 1.0\n',
                'gfd-tune 1\n0 1 0 96\n'):
        p = tmp_path / 'bad.txt'
        p.write_text(bad)
        assert lib.gfd_autotune_load(str(p).encode()) == _lib.GFD_EINVAL
    assert lib.gfd_autotune_load(str(tmp_path / 'missing.txt').encode()) == _lib.GFD_EINVAL
    assert lib.gfd_autotune_count(ctypes.byref(n)) == 0 and n.value == 2
    assert lib.gfd_autotune_clear() == 0
    assert lib.gfd_autotune_count(ctypes.byref(n)) == 0 and n.value == 0


def test_madelung_matches_oracle():
    """gfd_madelung (host code of the library) against the oracle's
    restatement of gpaw/utilities/ewald.py:148, and the simple cubic
    lattice's known value in a neutralising background, 2.837297 / L."""
    from gpaw_b200.poisson import madelung
    from oracle import poisson as OP
    for cell in (np.diag([10.0, 10.0, 10.0]), np.diag([9.0, 12.0, 15.5]),
                 np.array([[8.0, 0.0, 0.0], [2.0, 9.0, 0.0], [0.5, 1.0, 11.0]])):
        m = madelung(cell)
        assert abs(m - OP.madelung(cell)) < 1e-12 * abs(m), cell
    assert abs(madelung(np.diag([7.3] * 3)) * 7.3 - 2.837297) < 1e-6


def test_timer_nesting_and_metrics_log(tmp_path):
    """Timer keeps the reference's rules (gpaw/utilities/timing.py:86-166):
    regions nest by name, stop must follow stack order, inclusive and
    exclusive times add up; MetricsLog writes one JSON object per line."""
    import json
    import time
    from gpaw_b200.timing import MetricsLog, Timer
    t = Timer()
    t.start('SCF')
    t.start('Poisson')
    time.sleep(0.02)
    with pytest.raises(RuntimeError, match='stack order'):
        t.stop('SCF')
    t.stop('Poisson')
    t.start('Poisson')
    time.sleep(0.01)
    t.stop()
    t.stop('SCF')
    with pytest.raises(RuntimeError):
        t.stop()
    scf, poisson = t.get_time('SCF'), t.get_time('SCF', 'Poisson')
    assert 0.03 <= poisson <= scf
    rows, tot = t.table()
    excl = {names: te for names, _, te in rows}
    assert abs(excl[('SCF',)] - (scf - poisson)) < 1e-12
    assert abs(sum(excl.values()) - tot) < 1e-9
    u = Timer()
    u.add(t)
    u.add(t)
    assert abs(u.get_time('SCF', 'Poisson') - 2 * poisson) < 1e-12
    path = str(tmp_path / 'm.jsonl')
    with MetricsLog(path) as m:
        m.log('request', rid=1, N=np.int64(32), residual=np.float64(1e-11), status='ok')
        m.timer(t)
    recs = [json.loads(line) for line in open(path)]
    assert recs[0]['kind'] == 'request' and recs[0]['N'] == 32 and recs[0]['residual'] == 1e-11
    assert [r['region'] for r in recs[1:]] == ['SCF', 'SCF.Poisson', 'Other', 'Total']
