"""falm_b200: B200-native (sm_100a) implementation of FALM's LES time step.

The compute path is the CUDA library ``libfalm_b200.so`` behind the C ABI in
``include/falm_b200.h``; this package holds its ctypes binding, a Python
handle with the reference's method names, and the synthetic case builders.
"""
from . import _lib, cases
from ._lib import load, FalmError, BC_CHANNEL, BC_CAVITY

__all__ = ["_lib", "cases", "load", "FalmError", "BC_CHANNEL", "BC_CAVITY", "Context"]


def __getattr__(name):
    if name == "Context":
        from .api import Context
        return Context
    raise AttributeError(name)
