"""B200-native multislice engine with the reference's simulation API.

The compute path is ``libmslice_b200.so`` (hand-written sm_100a CUDA behind the
C ABI in ``include/mslice.h``); this package is its Python mirror.  Importing
it does not touch the GPU; creating a ``ManagedMultisliceSimulation`` does.
"""
from ._lib import LIB_PATH, MultisliceError, lib
from .simulation import ManagedMultisliceSimulation, stem_raster_concurrent, write_tiff

DATA_DIR = __import__("os").path.join(__import__("os").path.dirname(__file__), "data")
FPARAMS = __import__("os").path.join(DATA_DIR, "fparams.dat")

__all__ = ["ManagedMultisliceSimulation", "stem_raster_concurrent", "write_tiff", "MultisliceError", "lib", "LIB_PATH", "FPARAMS", "DATA_DIR"]
