"""ctypes binding of libgpawfd.so (declared in include/gpaw_fd.h).

The library is the only compute path: if it is missing or cannot be loaded,
importing this module raises ImportError.  There is no CPU fallback.
"""
import ctypes
import math
import os

import numpy as np

from .errors import PoissonConvergenceError

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libgpawfd.so')

GFD_OK = 0
GFD_EINVAL = 1
GFD_ENOMEM = 2
GFD_ENOCONV = 3
GFD_ETIMEOUT = 4
GFD_ECUDA = 5
GFD_EUNSUPPORTED = 6
GFD_ENEEDGAUSS = 7

GFD_SOLVE_ZERO_INITIAL_PHI = 1

GFD_FLOAT64 = 0
GFD_COMPLEX128 = 1
GFD_FLOAT32 = 2
GFD_COMPLEX64 = 3

GFD_RELAX_GS = 1
GFD_RELAX_JACOBI = 2

GFD_POISSON_FP64 = 0
GFD_POISSON_MIXED = 1

GFD_BATCH_NO_GROUPS = 1

GFD_TUNE_APPLY = 0
GFD_TUNE_JACOBI = 1
GFD_TUNE_POTENTIAL = 3


class TunePlan(ctypes.Structure):
    """gfd_tune_plan: form 0 one thread per point / 1 marching kernel, the
    marching tile (0: 32 columns, 1: 16, 2: 8, 3: 32 columns by 8 rows, 4: complex
    bands with the real and imaginary parts on lane pairs, 5: the same for
    complex128 on full rows staged by TMA, 6: complex128, 48 columns by 8
    rows), the
    axis-0 split target in CTAs per SM and the measured microseconds per
    launch."""
    _fields_ = [('form', ctypes.c_int), ('tile', ctypes.c_int), ('ctas_per_sm', ctypes.c_int),
                ('us', ctypes.c_double)]

    def as_dict(self):
        return {'form': ('direct', 'march')[self.form],
                'tile': (32, 16, 8, '32x8', 'split', 'tma-split', '48x8')[self.tile],
                'ctas_per_sm': self.ctas_per_sm, 'us': self.us}

# Every function the header declares: name -> (restype, argtypes).
_vp = ctypes.c_void_p
_i64p = ctypes.POINTER(ctypes.c_int64)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
SIGNATURES = {
    'gfd_last_error': (ctypes.c_size_t, [ctypes.c_char_p, ctypes.c_size_t]),
    'gfd_version': (ctypes.c_char_p, []),
    'gfd_operator_create': (ctypes.c_int, [ctypes.c_int, _dp, _i64p, _i64p, ctypes.c_int, _i64p,
                                           ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]),
    'gfd_operator_destroy': (ctypes.c_int, [_vp]),
    'gfd_operator_apply': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int64, _dp, _vp]),
    'gfd_operator_relax': (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int,
                                          ctypes.c_double, _vp]),
    'gfd_operator_relax_noalloc': (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                                  ctypes.c_int, ctypes.c_double, _vp]),
    'gfd_operator_get_diagonal_element': (ctypes.c_int, [_vp, _dp]),
    'gfd_device_errors': (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    'gfd_wait_selftest': (ctypes.c_int, [ctypes.c_longlong]),
    'gfd_test_fail_alloc': (ctypes.c_int, [ctypes.c_longlong]),
    'gfd_density_interpolate': (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_int, _vp]),
    'gfd_poisson_set_rhs_operator': (ctypes.c_int, [_vp, _vp]),
    'gfd_preconditioner_create': (ctypes.c_int, [_vp] * 7 + [ctypes.c_int, ctypes.c_int64,
                                                             ctypes.POINTER(_vp)]),
    'gfd_preconditioner_destroy': (ctypes.c_int, [_vp]),
    'gfd_preconditioner_apply': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int64, _dp,
                                                _vp]),
    'gfd_operator_apply_potential': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int64, _dp, _vp, _vp]),
    'gfd_transformer_create': (ctypes.c_int, [_i64p, _i64p, ctypes.c_int, _i64p, _i64p, _i64p,
                                              _i64p, ctypes.c_int, ctypes.c_int,
                                              ctypes.POINTER(_vp)]),
    'gfd_transformer_destroy': (ctypes.c_int, [_vp]),
    'gfd_transformer_apply': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int64, _dp,
                                             _vp]),
    'gfd_poisson_create': (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                          ctypes.POINTER(_vp), _ip, _ip, _dp, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(_vp)]),
    'gfd_poisson_destroy': (ctypes.c_int, [_vp]),
    'gfd_poisson_solve': (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, _ip, _dp, _vp]),
    'gfd_poisson_solve_ex': (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_int, _ip, _dp,
                                            _vp]),
    'gfd_poisson_load_gauss': (ctypes.c_int, [_vp, _dp, _i64p, _dp, ctypes.c_double, _vp]),
    'gfd_poisson_set_madelung': (ctypes.c_int, [_vp, ctypes.c_double]),
    'gfd_madelung': (ctypes.c_int, [_dp, _dp]),
    'gfd_poisson_solve_async': (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_int, _vp]),
    'gfd_poisson_result': (ctypes.c_int, [_vp, _ip, _dp]),
    'gfd_poisson_batch_create': (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp),
                                                ctypes.POINTER(_vp)]),
    'gfd_poisson_batch_destroy': (ctypes.c_int, [_vp]),
    'gfd_poisson_batch_create_ex': (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp), ctypes.c_int,
                                                   ctypes.POINTER(_vp)]),
    'gfd_poisson_batch_grouped': (ctypes.c_int, [_vp, _ip]),
    'gfd_poisson_batch_solve_async': (ctypes.c_int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                                     ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                     _vp]),
    'gfd_grid_sum': (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_double, _dp, _vp]),
    'gfd_autotune_operator': (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp,
                                             ctypes.c_int64, _dp, ctypes.c_double, ctypes.c_int,
                                             _vp, ctypes.POINTER(TunePlan)]),
    'gfd_autotune_transformer': (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int64,
                                                ctypes.c_int, _vp, ctypes.POINTER(TunePlan)]),
    'gfd_autotune_operator_plan': (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                                  ctypes.POINTER(TunePlan), _ip]),
    'gfd_autotune_transformer_plan': (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int64,
                                                     ctypes.POINTER(TunePlan), _ip]),
    'gfd_autotune_count': (ctypes.c_int, [_ip]),
    'gfd_autotune_clear': (ctypes.c_int, []),
    'gfd_autotune_save': (ctypes.c_int, [ctypes.c_char_p]),
    'gfd_autotune_load': (ctypes.c_int, [ctypes.c_char_p]),
    'gfd_poisson_autotune': (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError('libgpawfd.so is not built (run python -m gpaw_b200.build): %s'
                          % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def last_error():
    buf = ctypes.create_string_buffer(1024)
    lib.gfd_last_error(buf, 1024)
    return buf.value.decode(errors='replace')


def check(status, what=''):
    """Map a status code to the exception the reference would raise."""
    if status == GFD_OK:
        return
    msg = last_error()
    if what:
        msg = '%s: %s' % (what, msg)
    if status == GFD_EINVAL:
        raise ValueError(msg)
    if status == GFD_ENOMEM:
        raise MemoryError(msg)
    if status == GFD_ENOCONV:
        raise PoissonConvergenceError(msg)
    if status in (GFD_EUNSUPPORTED, GFD_ENEEDGAUSS):
        raise NotImplementedError(msg)
    raise RuntimeError('%s (status %d)' % (msg, status))


def i64(a):
    a = np.ascontiguousarray(np.asarray(a, np.int64).ravel())
    return a, a.ctypes.data_as(_i64p)


def f64(a):
    a = np.ascontiguousarray(np.asarray(a, np.float64).ravel())
    return a, a.ctypes.data_as(_dp)


def phases_arg(phase_cd):
    """12 host doubles (phase_cd[c][d] as re, im) or None."""
    if phase_cd is None:
        return None, None
    if hasattr(phase_cd, 'detach'):
        phase_cd = phase_cd.detach().cpu().numpy()
    ph = np.ascontiguousarray(np.asarray(phase_cd, np.complex128).reshape(3, 2))
    flat = ph.view(np.float64).ravel().copy()
    return flat, flat.ctypes.data_as(_dp)


def nan():
    return math.nan
