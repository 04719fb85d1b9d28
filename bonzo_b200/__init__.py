"""bonzo_b200: B200-native VL2 + HLLD + CT MHD step with the bonzo interface.

Host-side modules are importable without a GPU; the compute path lives in
libbnzgpu.so (built by bonzo_b200/build.py) and has no CPU fallback.
"""
__version__ = "0.1.0"

from ._lib import Batch, BnzError, Context  # noqa: E402,F401
from .simulation import Simulation  # noqa: E402,F401
