"""uegccd_b200 -- B200 (sm_100a) coupled-cluster hot path of the uniform-electron-gas code uegCCD.

The compute lives in libuegccd.so (C ABI: include/uegccd.h); this package is
its Python face and the host-side mirror of the reference's drivers.
"""
from . import _capi
from .solver import Batch, Context

__all__ = ["Batch", "Context", "_capi"]
__version__ = "0.1"
