"""ferrox_b200 -- FerroX's coupled time step (TDGL + semiconductor Newton +
variable-permittivity Poisson + E = -grad phi) on one NVIDIA B200.

The compute path is the native library libferrox_b200.so (hand-written
sm_100a CUDA behind the C ABI in include/ferrox_b200.h); ``api.FerroX`` is the
Python view of that ABI.  ``decks`` builds synthetic inputs files for the named
device stacks; ``plotfile`` reads the AMReX plotfiles the library writes.
"""
from . import decks  # noqa: F401

__all__ = ["decks", "api", "plotfile"]
