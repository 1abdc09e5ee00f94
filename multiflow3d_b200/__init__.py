"""B200-native MultiFlow3D pressure-Poisson multigrid (newsolv_mg) library.

The product is the native library ``libmf3d.so`` (hand-written CUDA for
sm_100a plus a C++ host driver) behind the C ABI in ``include/mf3d.h``.
This package holds its ctypes binding (``abi``), the host-side mirror of the
reference's projection interface (``solver``), input generators
(``problems``) and the build recipe (``build``).
"""
from . import abi  # noqa: F401

__all__ = ["abi"]
