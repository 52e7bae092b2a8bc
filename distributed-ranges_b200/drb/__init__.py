"""drb: the B200-native gemv hot path of Distributed Ranges.

``drb.mp`` mirrors the reference's dr::mp gemv interface; ``drb.gen`` builds
seeded synthetic workloads; ``drb._capi`` is the ctypes binding of
include/drb.h.  Importing the package requires the in-tree CUDA library
(``make -C distributed-ranges_b200``): there is no CPU fallback.
"""
from . import _capi, gen, mp  # noqa: F401
from ._capi import DrbError  # noqa: F401

__version__ = "0.1"
