"""B200-native (sm_100a) EmSART reconstruction hot path.

The CUDA library ``libesb.so`` (C ABI in ``include/esb.h``) holds every
kernel; this package is the host layer over it. Importing the package loads
the library and raises ImportError when it has not been built.
"""
from . import _lib  # noqa: F401  (loads libesb.so or raises)
from .emsart import *  # noqa: F401,F403

__all__ = [n for n in dir() if not n.startswith("_")]
