"""ctypes bindings to the CPU oracle libraries -- TEST INFRASTRUCTURE ONLY.

impl='port' calls liboracle.so, the C restatement in gfd_oracle.c.
impl='ref'  calls _ref/libgpawref.so: GPAW's own c/bmgs/bmgs.c and c/bc.c
            compiled unmodified, driven by ref_driver.c.  It exists only
            where the reference tree was available at build time.
"""
import ctypes
import os
import subprocess

import numpy as np

from . import geometry

_HERE = os.path.dirname(os.path.abspath(__file__))


def _host_has_avx512():
    """True when the CPU offers the x86-64-v4 feature set (AVX-512 F, BW,
    CD, DQ, VL)."""
    try:
        with open('/proc/cpuinfo') as f:
            for line in f:
                if line.startswith('flags'):
                    flags = set(line.split(':', 1)[1].split())
                    return {'avx512f', 'avx512bw', 'avx512cd', 'avx512dq',
                            'avx512vl'} <= flags
    except OSError:
        pass
    return False


def _variant(path):
    """The x86-64-v4 build of a library where the host supports it and it
    was built, else the x86-64-v3 one."""
    v4 = path[:-3] + '_v4.so'
    if _host_has_avx512() and os.path.exists(v4):
        return v4
    return path


PORT_PATH = _variant(os.path.join(_HERE, 'liboracle.so'))
REF_PATH = _variant(os.path.join(_HERE, '_ref', 'libgpawref.so'))
ISA = 'x86-64-v4' if PORT_PATH.endswith('_v4.so') else 'x86-64-v3'

_libs = {}

_i64p = ctypes.POINTER(ctypes.c_int64)
_lp = ctypes.POINTER(ctypes.c_long)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(ref=True):
    """Compile the oracle libraries (make -C oracle)."""
    target = 'all' if ref else 'port'
    subprocess.run(['make', '-s', '-C', _HERE, target], check=True)


def have_ref():
    return os.path.exists(REF_PATH)


def _lib(impl):
    if impl in _libs:
        return _libs[impl]
    path = PORT_PATH if impl == 'port' else REF_PATH
    if not os.path.exists(path):
        if impl == 'port':
            build(ref=False)
        else:
            raise FileNotFoundError('reference oracle library not built: %s' % path)
    lib = ctypes.CDLL(path)
    if impl == 'port':
        lib.orc_fd_apply.argtypes = [ctypes.c_int, _dp, _i64p, _i64p, _ip, ctypes.c_int,
                                     ctypes.c_int64, _dp, _dp, _dp, ctypes.c_int]
        lib.orc_relax.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _i64p, _i64p, _ip,
                                  _dp, _dp, ctypes.c_int, ctypes.c_double]
        lib.orc_transform.argtypes = [ctypes.c_int, ctypes.c_int, _i64p, _i64p, _i64p, _ip,
                                      ctypes.c_int, ctypes.c_int64, _dp, _dp, _dp, ctypes.c_int]
        lib.orc_transform_shape.argtypes = [ctypes.c_int, ctypes.c_int, _i64p, _i64p, _i64p,
                                            _i64p]
    else:
        lib.ref_fd_apply.argtypes = [ctypes.c_int, _dp, _lp, _lp, ctypes.c_int, _lp,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
                                     ctypes.c_int]
        lib.ref_relax.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _lp, _lp, ctypes.c_int, _lp,
                                  ctypes.c_int, _dp, _dp, ctypes.c_int, ctypes.c_double]
        lib.ref_transform.argtypes = [_lp, _lp, ctypes.c_int, _lp, _lp, _lp, _lp, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int]
    _libs[impl] = lib
    return lib


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def _i64(x):
    return np.ascontiguousarray(np.asarray(x, np.int64).ravel())


def _cl(x):
    return np.ascontiguousarray(np.asarray(x, np.int_).ravel())


def _phases(phase_cd):
    if phase_cd is None:
        return np.ones((3, 2), complex)
    return np.ascontiguousarray(np.asarray(phase_cd, complex).reshape(3, 2))


def _nbands(a):
    return int(np.prod(a.shape[:-3])) if a.ndim > 3 else 1


def _check(st, what):
    if st != 0:
        raise ValueError('oracle %s failed with status %d' % (what, st))


def fd_apply(coefs, offsets_pc, pbc_c, a, phase_cd=None, nthreads=1, impl='port'):
    """out[x, g] = sum_p coefs[p] * a[x, g + offsets_pc[p]] with zero or
    (Bloch-)periodic halos.  `a` is float64 or complex128, shape (..., n0, n1, n2)."""
    a = np.ascontiguousarray(a)
    assert a.dtype in (np.float64, np.complex128)
    real = a.dtype == np.float64
    coefs = np.ascontiguousarray(coefs, float)
    offsets_pc = np.asarray(offsets_pc, np.int64).reshape(-1, 3)
    n_c = a.shape[-3:]
    out = np.empty_like(a)
    nb = _nbands(a)
    ph = _phases(phase_cd)
    lib = _lib(impl)
    if impl == 'port':
        per = np.ascontiguousarray(np.asarray(pbc_c, np.int32).ravel() * np.ones(3, np.int32))
        st = lib.orc_fd_apply(len(coefs), _ptr(coefs), _ptr(_i64(offsets_pc), _i64p),
                              _ptr(_i64(n_c), _i64p), _ptr(per, _ip), 1 if real else 2, nb,
                              _ptr(a.view(np.float64)), _ptr(out.view(np.float64)),
                              _ptr(ph.view(np.float64)), nthreads)
    else:
        mp, flat, cfd = geometry.fd_layout(offsets_pc, n_c)
        nbr = np.where(np.asarray(pbc_c, bool).ravel()[:, None] * np.ones((3, 2), bool), 0, -1)
        st = lib.ref_fd_apply(len(coefs), _ptr(coefs), _ptr(_cl(flat), _lp),
                              _ptr(_cl(n_c), _lp), mp, _ptr(_cl(nbr), _lp), int(real),
                              int(cfd), nb, _ptr(a.view(np.float64)),
                              _ptr(out.view(np.float64)), _ptr(ph.view(np.float64)), nthreads)
    _check(st, 'fd_apply')
    return out


def relax(method, coefs, offsets_pc, pbc_c, phi, rho, nsweeps, w, impl='port'):
    """In-place relaxation of phi (float64, 3-D) for L phi = rho.
    method 1: lexicographic Gauss-Seidel; otherwise weighted Jacobi."""
    assert phi.dtype == np.float64 and phi.flags.c_contiguous
    rho = np.ascontiguousarray(rho, float)
    coefs = np.ascontiguousarray(coefs, float)
    offsets_pc = np.asarray(offsets_pc, np.int64).reshape(-1, 3)
    n_c = phi.shape
    lib = _lib(impl)
    if w is None:
        w = 1.0
    if impl == 'port':
        per = np.ascontiguousarray(np.asarray(pbc_c, np.int32).ravel() * np.ones(3, np.int32))
        st = lib.orc_relax(int(method), len(coefs), _ptr(coefs), _ptr(_i64(offsets_pc), _i64p),
                           _ptr(_i64(n_c), _i64p), _ptr(per, _ip), _ptr(phi), _ptr(rho),
                           int(nsweeps), float(w))
    else:
        mp, flat, cfd = geometry.fd_layout(offsets_pc, n_c)
        nbr = np.where(np.asarray(pbc_c, bool).ravel()[:, None] * np.ones((3, 2), bool), 0, -1)
        st = lib.ref_relax(int(method), len(coefs), _ptr(coefs), _ptr(_cl(flat), _lp),
                           _ptr(_cl(n_c), _lp), mp, _ptr(_cl(nbr), _lp), int(cfd), _ptr(phi),
                           _ptr(rho), int(nsweeps), float(w))
    _check(st, 'relax')


def transform(gdin, gdout, nn, a, phases=None, nthreads=1, impl='port'):
    """Restriction (gdin twice as fine as gdout) or interpolation of a."""
    a = np.ascontiguousarray(a)
    assert a.dtype in (np.float64, np.complex128)
    real = a.dtype == np.float64
    pad, npad, skip, interp = geometry.transformer_layout(gdin, gdout, nn)
    nb = _nbands(a)
    out = np.zeros(a.shape[:-3] + tuple(gdout.n_c), a.dtype)
    ph = _phases(phases)
    lib = _lib(impl)
    if impl == 'port':
        per = np.ascontiguousarray(gdin.pbc_c.astype(np.int32))
        st = lib.orc_transform(int(interp), 2 * nn, _ptr(_i64(gdin.n_c), _i64p),
                               _ptr(_i64(pad), _i64p), _ptr(_i64(skip), _i64p), _ptr(per, _ip),
                               1 if real else 2, nb, _ptr(a.view(np.float64)),
                               _ptr(out.view(np.float64)), _ptr(ph.view(np.float64)), nthreads)
    else:
        st = lib.ref_transform(_ptr(_cl(gdin.n_c), _lp), _ptr(_cl(gdout.n_c), _lp), 2 * nn,
                               _ptr(_cl(pad), _lp), _ptr(_cl(npad), _lp), _ptr(_cl(skip), _lp),
                               _ptr(_cl(gdin.neighbor_cd), _lp), int(real), int(interp), nb,
                               _ptr(a.view(np.float64)), _ptr(out.view(np.float64)),
                               _ptr(ph.view(np.float64)), nthreads)
    _check(st, 'transform')
    return out
