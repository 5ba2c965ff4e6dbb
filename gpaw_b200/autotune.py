"""Launch-plan autotuning of the stencil and transfer kernels.

The library picks, per (operation, dtype, mode, grid, radius or transfer
order, boundary conditions, band-count class), the kernel form (one thread
per point or the marching kernel), the marching tile and the axis-0 split.
Without a tuned plan it uses built-in rules; tune_operator / tune_transformer
time every candidate on the GPU and cache the fastest in the library, where
every later launch with the same key finds it.  Plans change times; the
results of the marching candidates are bit-identical, the one-thread-per-point
form sums a stencil's terms in another order (rounding-level differences).

    from gpaw_b200 import autotune
    autotune.tune_operator(lap, nbands=512, phase_cd=phase_cd)
    autotune.tune_transformer(restrictor, nbands=256)
    autotune.save('plans.txt')        # GFD_TUNE_CACHE=plans.txt reloads it
"""
import torch

from . import _lib
from .tensors import dtype_code, is_complex, stream_of, torch_dtype

_MODES = {'apply': _lib.GFD_TUNE_APPLY, 'jacobi': _lib.GFD_TUNE_JACOBI,
          'potential': _lib.GFD_TUNE_POTENTIAL}


def _scratch(shape, dtype, device, seed=0):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    if torch_dtype(dtype) in (torch.complex128, torch.complex64):
        return torch.randn(shape, dtype=torch_dtype(dtype), device=device, generator=g)
    return torch.rand(shape, dtype=torch_dtype(dtype), device=device, generator=g) - 0.5


def tune_operator(op, nbands=1, mode='apply', dtype=None, phase_cd=None, w=2.0 / 3.0,
                  reps=5, device='cuda'):
    """Tune op (an FDOperator) for launches of nbands bands in mode 'apply',
    'jacobi' (relaxation sweeps; real dtypes) or 'potential'
    (apply_with_potential).  Allocates its own scratch bands.  Returns the
    chosen plan as a dict."""
    if mode not in _MODES:
        raise ValueError('mode must be one of %s' % sorted(_MODES))
    dtype = torch_dtype(dtype if dtype is not None else op.dtype)
    shape = (int(nbands),) + tuple(op.shape)
    a = _scratch(shape, dtype, device, 1)
    b = torch.empty_like(a)
    src = None
    if mode == 'jacobi':
        src = _scratch(shape, dtype, device, 2)
    elif mode == 'potential':
        real = torch.float32 if dtype in (torch.float32, torch.complex64) else torch.float64
        src = _scratch(tuple(op.shape), real, device, 3)
    _, pp = _lib.phases_arg(phase_cd if is_complex(dtype) else None)
    plan = _lib.TunePlan()
    _lib.check(_lib.lib.gfd_autotune_operator(
        op.operator, dtype_code(a), _MODES[mode], a.data_ptr(), b.data_ptr(),
        None if src is None else src.data_ptr(), int(nbands), pp, float(w), int(reps),
        stream_of(a), _lib.ctypes.byref(plan)), 'autotune')
    torch.cuda.current_stream(a.device).synchronize()
    return plan.as_dict()


def tune_transformer(tr, nbands=1, dtype=None, reps=5, device='cuda'):
    """Tune a Transformer (restriction or interpolation) for nbands bands."""
    t = getattr(tr, 'transformer', None)
    if t is None:
        return None  # identity transformer: nothing runs
    dtype = torch_dtype(dtype if dtype is not None else tr.dtype)
    a = _scratch((int(nbands),) + tuple(tr.ngpin), dtype, device, 4)
    b = torch.empty((int(nbands),) + tuple(tr.ngpout), dtype=a.dtype, device=a.device)
    plan = _lib.TunePlan()
    _lib.check(_lib.lib.gfd_autotune_transformer(
        t, dtype_code(a), a.data_ptr(), b.data_ptr(), int(nbands), int(reps), stream_of(a),
        _lib.ctypes.byref(plan)), 'autotune')
    torch.cuda.current_stream(a.device).synchronize()
    return plan.as_dict()


def operator_plan(op, nbands=1, mode='apply', dtype=None):
    """The cached plan for these launches, or None (built-in rules)."""
    dtype = torch_dtype(dtype if dtype is not None else op.dtype)
    plan = _lib.TunePlan()
    found = _lib.ctypes.c_int(0)
    _lib.check(_lib.lib.gfd_autotune_operator_plan(
        op.operator, _lib_dtype(dtype), _MODES[mode], int(nbands), _lib.ctypes.byref(plan),
        _lib.ctypes.byref(found)))
    return plan.as_dict() if found.value else None


def transformer_plan(tr, nbands=1, dtype=None):
    dtype = torch_dtype(dtype if dtype is not None else tr.dtype)
    plan = _lib.TunePlan()
    found = _lib.ctypes.c_int(0)
    _lib.check(_lib.lib.gfd_autotune_transformer_plan(
        tr.transformer, _lib_dtype(dtype), int(nbands), _lib.ctypes.byref(plan),
        _lib.ctypes.byref(found)))
    return plan.as_dict() if found.value else None


def _lib_dtype(dtype):
    return {torch.float64: _lib.GFD_FLOAT64, torch.complex128: _lib.GFD_COMPLEX128,
            torch.float32: _lib.GFD_FLOAT32, torch.complex64: _lib.GFD_COMPLEX64}[dtype]


def count():
    n = _lib.ctypes.c_int(0)
    _lib.check(_lib.lib.gfd_autotune_count(_lib.ctypes.byref(n)))
    return n.value


def clear():
    _lib.check(_lib.lib.gfd_autotune_clear())


def save(path):
    _lib.check(_lib.lib.gfd_autotune_save(str(path).encode()), 'autotune.save')


def load(path):
    _lib.check(_lib.lib.gfd_autotune_load(str(path).encode()), 'autotune.load')
