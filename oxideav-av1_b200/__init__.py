"""B200-native AV1 reconstruction and post-filter engine.

The hot path of the reference decoder's frame driver — everything after the
tile walk has parsed a frame's symbols — runs here as hand-written sm_100a
CUDA kernels behind the C ABI declared in ``include/av1g.h``.  This package is
the Python host layer over that ABI: ctypes bindings (``abi``), device-resident
frames and batched launches (``postfilter``), and the seeded synthetic
workload generator (``synth``).
"""
from . import abi  # noqa: F401
from .build import build_library  # noqa: F401

__all__ = ["abi", "build_library"]
