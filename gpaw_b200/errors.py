"""Exceptions of the finite-difference path (gpaw/__init__.py:46-53)."""


class ConvergenceError(Exception):
    pass


class PoissonConvergenceError(ConvergenceError):
    pass
