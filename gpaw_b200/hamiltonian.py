"""The finite-difference pseudo-Hamiltonian on wave-function bands.

GPAW applies it as two passes over every band
(gpaw/wavefunctions/fd.py:50-52, FDWaveFunctions.apply_pseudo_hamiltonian):

    self.kin.apply(psit_xG, Htpsit_xG, kpt.phase_cd)        # -1/2 nabla^2
    hamiltonian.apply_local_potential(psit_xG, Htpsit_xG, s)  # += psit * vt

(gpaw/hamiltonian.py:371-398).  Here the two are one kernel pass: the
potential joins the stencil's centre weight, so each band is read once and
written once.
"""
from .fd_operators import FDOperator


def apply_pseudo_hamiltonian(kin, psit_xG, Htpsit_xG, vt_G, phase_cd=None):
    """Htpsit_xG = kin psit_xG + vt_G psit_xG (band-batched, CUDA tensors).

    kin: the kinetic FDOperator (Laplace(gd, -0.5, nn, dtype)); vt_G: the
    spin channel's local potential on the same grid (float64 for
    float64/complex128 bands, float32 for float32/complex64); phase_cd: the
    k-point's Bloch phases for complex bands."""
    if not isinstance(kin, FDOperator):
        raise TypeError('kin must be an FDOperator')
    kin.apply_with_potential(psit_xG, Htpsit_xG, vt_G, phase_cd)
