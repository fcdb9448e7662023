"""flowgpu - B200 implementation of the shedsaw/flow-solver nonlinear iteration.

Python side of the package: mesh generation (meshgen), the ctypes binding of
the CUDA library (capi) and the host preprocessing (prep).
"""
from . import meshgen  # noqa: F401

__all__ = ["meshgen", "capi"]
