"""B200-native implicit 2D (and 1D) DG / condensed-HDG Euler solver.

The compute path is lib/libdgh_gpu.so: hand-written sm_100a CUDA kernels behind the C ABI in
include/dgh_gpu.h, plus the C++ host integrator.  This package only loads that library
(`_lib`), offers a Python mirror of the reference's solver surface (`solver`), and builds the
library in-tree (`build`).
"""
from ._lib import BIN1D_PATH, BIN_PATH, LIB_PATH, build, load  # noqa: F401

__all__ = ["build", "load", "LIB_PATH", "BIN_PATH", "BIN1D_PATH"]
