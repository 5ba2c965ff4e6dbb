"""Grid transformers on the GPU (drop-in for gpaw.transformers).

Transformer(gdin, gdout, nn, dtype).apply(input, output, phases) restricts
(gdin twice as fine as gdout) or interpolates (gdout twice as fine) with
K = 2 nn Lagrange taps per axis.  The halo widths and skips follow
_Transformer.__init__ (gpaw/transformers.py:19-62):

  restriction     pad = (2nn-1-2 beg_out+beg_in, 2nn-2+2 end_out-end_in)
  interpolation   pad = (nn-1-beg_out//2+beg_in, nn+end_out//2-end_in),
                  skip = (beg_out % 2, end_out % 2)

which for one domain is (2nn-1, 2nn-2) periodic / (2nn-2, 2nn-2) zero
boundary for restriction and (nn-1, nn) / (nn, nn) with skip (1, 0) on a
zero-boundary axis for interpolation.
"""
import numpy as np

from . import _lib
from .tensors import dtype_code, is_complex, nbands, require_device, stream_of, torch_dtype


class _Transformer:
    def __init__(self, gdin, gdout, nn=1, dtype=float, allocate=True):
        if not 1 <= nn <= 4:
            raise ValueError('nn must be 1..4')
        self.gdin = gdin
        self.gdout = gdout
        self.nn = nn
        self.dtype = torch_dtype(dtype)
        pad_cd = np.zeros((3, 2), int)
        npad_cd = np.zeros((3, 2), int)
        skip_cd = np.zeros((3, 2), int)
        if (gdin.N_c == 2 * gdout.N_c).all():
            pad_cd[:, 0] = 2 * nn - 1 - 2 * gdout.beg_c + gdin.beg_c
            pad_cd[:, 1] = 2 * nn - 2 + 2 * gdout.end_c - gdin.end_c
            npad_cd[:, 0] = 2 * nn - 2 + 2 * gdout.beg_c - gdin.beg_c
            npad_cd[:, 1] = 2 * nn - 1 - 2 * gdout.end_c + gdin.end_c
            self.interpolate = False
        elif (gdout.N_c == 2 * gdin.N_c).all():
            pad_cd[:, 0] = nn - 1 - gdout.beg_c // 2 + gdin.beg_c
            pad_cd[:, 1] = nn + gdout.end_c // 2 - gdin.end_c
            npad_cd[:, 0] = nn + gdout.beg_c // 2 - gdin.beg_c
            npad_cd[:, 1] = nn - 1 - gdout.end_c // 2 + gdin.end_c
            skip_cd[:, 0] = gdout.beg_c % 2
            skip_cd[:, 1] = gdout.end_c % 2
            self.interpolate = True
            # Same size guard as the reference (gpaw/transformers.py:50-51),
            # kept so that both accept exactly the same grids.
            if ((gdin.n_c[0] + 2 * nn - 1) * (gdin.n_c[1] + 2 * nn - 1) >
                    gdout.n_c[0] * gdout.n_c[1]):
                raise AssertionError('coarse grid too small for nn=%d interpolation' % nn)
        else:
            raise ValueError('grids must differ by a factor of two on every axis')
        if (pad_cd < 0).any():
            raise ValueError('negative transformer padding')
        self.pad_cd = pad_cd
        self.neighborpad_cd = npad_cd
        self.skip_cd = skip_cd
        self.ngpin = tuple(int(x) for x in gdin.n_c)
        self.ngpout = tuple(int(x) for x in gdout.n_c)
        self.transformer = None
        self.allocated = False
        if allocate:
            self.allocate()

    def allocate(self):
        if self.allocated:
            raise RuntimeError('already allocated')
        a = [_lib.i64(x) for x in (self.gdin.n_c, self.gdout.n_c, self.pad_cd,
                                   self.neighborpad_cd, self.skip_cd, self.gdin.neighbor_cd)]
        handle = _lib._vp()
        _lib.check(_lib.lib.gfd_transformer_create(
            a[0][1], a[1][1], 2 * self.nn, a[2][1], a[3][1], a[4][1], a[5][1],
            int(not is_complex(self.dtype)), int(self.interpolate), _lib.ctypes.byref(handle)),
            'Transformer')
        self.transformer = handle
        self.allocated = True

    def __del__(self):
        h = getattr(self, 'transformer', None)
        lib = getattr(_lib, 'lib', None) if _lib is not None else None
        if h and lib is not None:  # at interpreter exit the module may be gone
            lib.gfd_transformer_destroy(h)
            self.transformer = None

    def apply(self, input, output, phases=None):
        require_device(input, 'input')
        require_device(output, 'output')
        if tuple(input.shape[-3:]) != self.ngpin or tuple(output.shape[-3:]) != self.ngpout:
            raise ValueError('array shapes %s -> %s do not match the transformer %s -> %s'
                             % (tuple(input.shape), tuple(output.shape), self.ngpin, self.ngpout))
        if tuple(input.shape[:-3]) != tuple(output.shape[:-3]):
            raise ValueError('leading (band) dimensions differ')
        if input.dtype != output.dtype:
            raise ValueError('input and output dtypes differ')
        if is_complex(input.dtype) != is_complex(self.dtype):
            raise ValueError('transformer built for %s arrays, got %s' % (self.dtype, input.dtype))
        _, pp = _lib.phases_arg(phases if is_complex(input.dtype) else None)
        _lib.check(_lib.lib.gfd_transformer_apply(
            self.transformer, dtype_code(input), input.data_ptr(), output.data_ptr(),
            nbands(input), pp, stream_of(input)), 'Transformer.apply')

    def estimate_memory(self, mem):
        mem.subnode('buf', 0)


class _Identity:
    """nn=9: identity copy (gpaw/transformers.py:147-155)."""

    allocated = True

    def allocate(self):
        pass

    def apply(self, input, output, phases=None):
        output.copy_(input)


def Transformer(gdin, gdout, nn=1, dtype=float, allocate=True):
    if nn == 9:
        return _Identity()
    return _Transformer(gdin, gdout, nn, dtype, allocate)
