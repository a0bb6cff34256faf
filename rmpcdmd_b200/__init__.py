"""B200-native RMPCDMD solvent hot path.

The package is a thin host layer over the CUDA library built from
``rmpcdmd_b200/csrc`` (C ABI in ``include/rmpcd.h``).  Importing it loads the
library; if the library has not been built the import fails -- there is no
CPU implementation behind this API.
"""
from ._capi import lib as _lib

_lib()  # load now: a missing library is an import error, not a silent fallback

from .api import *  # noqa: E402,F401,F403
from .api import __all__  # noqa: E402,F401

__version__ = "0.1.0"
