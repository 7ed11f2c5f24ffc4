"""cansfz -- host side of the B200-native CaNS-Fizzy per-step hot path.

The compute runs in the CUDA library ``libcansfz.so`` (sm_100a) behind the C
ABI declared in ``include/cansfz.h``; this package reads the reference's
input files, builds the run parameters and drives that ABI through ctypes.
"""
from . import namelist  # noqa: F401
from .params import Params, from_file, from_namelist, from_text  # noqa: F401
