"""vship_b200 -- a B200-native SSIMULACRA2 and Butteraugli engine behind Vship's C ABI.

The product is libvship.so (built from csrc/ by build.py); this package is its Python
binding (api.py), the ctypes mirror of the ABI (abi.py) and the seeded synthetic frame
generator used by the benchmark and tests (synth.py).
"""
from .api import SSIMU2, SSIMU2Batch, Surrogate, Butteraugli, CVVDP, VshipError, PinnedBuffer, load, load_library  # noqa: F401
from . import abi  # noqa: F401
