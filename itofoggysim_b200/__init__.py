"""B200-native multi-sphere Mie solve (ItoFoggySim's T-matrix GMRES path) on sm_100a.

The compute path is libfoggy_b200.so (CUDA, C ABI in include/foggy_gpu.h); this package holds
its ctypes binding, the host-side mirror of the reference's solver interface and the seeded
synthetic scenes.
"""
from . import scene  # noqa: F401

__all__ = ["scene", "solver", "build"]
