"""B200-native GRAPE-6 force engine for Starlab's kira integrator.

The product is the C-ABI library ``lib/libg6b200.so`` (built from ``csrc/``
by ``starlab_b200.build``); this package adds a Python binding of that ABI
(``g6``), seeded initial-condition generators (``ics``) and the multi-cluster
drivers built on the same library.
"""
from .g6 import G6Engine, G6Error, load_library, LIB_PATH, FP64, MIXED  # noqa: F401

__all__ = ["G6Engine", "G6Error", "load_library", "LIB_PATH", "FP64", "MIXED"]
