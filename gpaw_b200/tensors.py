"""Device-array helpers: dtype codes, contiguity checks, current stream."""
import numpy as np
import torch

from . import _lib

_DTYPE_CODE = {
    torch.float64: _lib.GFD_FLOAT64,
    torch.complex128: _lib.GFD_COMPLEX128,
    torch.float32: _lib.GFD_FLOAT32,
    torch.complex64: _lib.GFD_COMPLEX64,
}

_FROM_NUMPY = {
    float: torch.float64, np.float64: torch.float64, complex: torch.complex128,
    np.complex128: torch.complex128, np.float32: torch.float32, np.complex64: torch.complex64,
}


def torch_dtype(dtype):
    """float / complex / numpy / torch dtype -> torch dtype."""
    if isinstance(dtype, torch.dtype):
        return dtype
    if dtype in _FROM_NUMPY:
        return _FROM_NUMPY[dtype]
    return _FROM_NUMPY[np.dtype(dtype).type]


def dtype_code(t):
    try:
        return _DTYPE_CODE[t.dtype]
    except KeyError:
        raise ValueError('unsupported dtype %s' % t.dtype)


def is_complex(dtype):
    return torch_dtype(dtype) in (torch.complex128, torch.complex64)


def real_of(dtype):
    """The real dtype an operator of this dtype is built for."""
    return not is_complex(dtype)


def require_device(t, name='array'):
    if not isinstance(t, torch.Tensor):
        raise TypeError('%s must be a torch tensor on a CUDA device' % name)
    if not t.is_cuda:
        raise ValueError('%s must live on a CUDA device (no CPU path)' % name)
    if not t.is_contiguous():
        raise ValueError('%s must be C-contiguous' % name)


def stream_of(t):
    return torch.cuda.current_stream(t.device).cuda_stream


def stream_of_device(device):
    """The current stream of a CUDA device (torch.device or index)."""
    return torch.cuda.current_stream(device).cuda_stream


def nbands(t):
    """Number of 3-D arrays in a (..., n0, n1, n2) tensor."""
    n = 1
    for s in t.shape[:-3]:
        n *= s
    return n
