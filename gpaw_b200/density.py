"""Pseudo density on the fine grid: Density.interpolate (gpaw/density.py:
217-235) on the GPU.

The reference interpolates every spin channel to the fine grid and, when
some axis has a zero boundary (where interpolation does not conserve the
number of electrons), scales the result so that it integrates to the pseudo
charge -(charge + comp_charge).  Here that is one call: the interpolation of
all spins, a deterministic device reduction and the scaling, with no
host-device round trip.
"""
import torch

from . import _lib
from .tensors import require_device, stream_of


def interpolate_pseudo_density(interpolator, nt_sG, nt_sg, finegd, pseudo_charge):
    """nt_sg = interpolator(nt_sG) spin by spin, renormalised to
    pseudo_charge = -(charge + comp_charge) unless finegd is periodic on
    every axis (gpaw/density.py:226-235).  interpolator: a coarse-to-fine
    Transformer (nn = 3 in GPAW); nt_sG, nt_sg: float64 CUDA tensors of
    shape (nspins,) + grid."""
    require_device(nt_sG, 'nt_sG')
    require_device(nt_sg, 'nt_sg')
    if nt_sG.dtype != torch.float64 or nt_sg.dtype != torch.float64:
        raise ValueError('densities are float64')
    if not (nt_sG.is_contiguous() and nt_sg.is_contiguous()):
        raise ValueError('densities must be contiguous')
    nspins = nt_sG.shape[0] if nt_sG.dim() == 4 else 1
    if tuple(nt_sg.shape[-3:]) != tuple(int(x) for x in finegd.n_c) or nt_sg.numel() != \
            nspins * int(finegd.n_c.prod()):
        raise ValueError('nt_sg must have shape (nspins,) + the fine grid')
    if not interpolator.allocated:
        interpolator.allocate()
    _lib.check(_lib.lib.gfd_density_interpolate(
        interpolator.transformer, nt_sG.data_ptr(), nt_sg.data_ptr(), nspins,
        float(pseudo_charge), float(finegd.dv), int(not finegd.pbc_c.all()), stream_of(nt_sG)),
        'interpolate_pseudo_density')
    return nt_sg
