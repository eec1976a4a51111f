"""ptychotomo_b200 — B200-native ptycho-tomography ADMM engine.

Drop-in for the hot path of nikitinvv/ptychotomo: the native operator
classes :class:`radonusfft` and :class:`ptychofft` (same constructor and
method signatures as the reference's SWIG classes) and the ADMM
:class:`Solver` (same methods as src/ptychotomo/solver.py) on torch CUDA
tensors.  All arithmetic runs in the sm_100a library
``libptychotomo_b200.so``; there is no CPU fallback.  The reference's host
helpers :func:`probe` and :func:`scanner3` (NumPy) are provided too, and
:func:`read_tiff`/:func:`write_tiff` in place of the dxchange calls of the
reference's driver script.
"""
from ._lib import PtychotomoArgError, PtychotomoError, lib  # noqa: F401
from .objects import probe, scanner3  # noqa: F401
from .operators import ptychofft, radonusfft  # noqa: F401
from .volumes import read_tiff, read_volume, write_tiff, write_volume  # noqa: F401

__version__ = "0.1.0"


def __getattr__(name):
    # the Solver needs torch; import it lazily so the operator classes do not
    if name == "Solver":
        from .solver import Solver
        return Solver
    raise AttributeError(name)
