"""cufcm_fil_b200 -- B200-native mobility engine for racksa/CUFCM_FIL's hot path.

The engine is ``libcufil.so`` (hand-written CUDA for sm_100a behind the C ABI
in ``include/cufil.h``); this package holds its ctypes bindings and the host
mirror of the reference's mobility-solver interface.
"""
from ._lib import CufilError, load as load_library, LIB_PATH  # noqa: F401
from .mobility import RpyMobilitySolver  # noqa: F401

__all__ = ["RpyMobilitySolver", "CufilError", "load_library", "LIB_PATH"]
