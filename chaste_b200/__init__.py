"""B200-native monodomain tissue for Chaste's operator-split step.

The compute path is libchastegpu.so (include/chaste_gpu.h); this package holds
its ctypes binding (_native), the Chaste-API mirror (heart), the build step
(build) and the CellML emitter (codegen).
"""
from ._native import ChasteGpuError, Tissue  # noqa: F401

__all__ = ["ChasteGpuError", "Tissue"]
