"""thrustrtc_b200 -- a B200-native implementation of ThrustRTC's data-parallel core.

``import thrustrtc_b200 as trtc`` offers the reference package's interface for the hot path
(sort, scans, reductions, the compaction family, the object model and the JIT launchers),
backed by nvcc-built sm_100a kernels and NVRTC instantiations for user Functors.  Importing
fails if the CUDA library has not been built; there is no CPU fallback.
"""
from . import _native  # noqa: F401  (raises ImportError when libPyThrustRTC.so is missing)
from .api import *  # noqa: F401,F403
from .api import check_i as _check_i, lib as _lib

__version__ = "0.1.0"


def init():
    """Initialises the CUDA context (the reference does this at import: __init__.py:3)."""
    _check_i(_lib.n_trtc_try_init())
