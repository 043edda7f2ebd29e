"""bigwham_dev_b200: a B200-native (sm_100a) H-matrix x vector backend for BigWham.

The reference (BigWham) builds the H-matrix on the host; this package applies
it on one GPU with hand-written CUDA kernels behind a C ABI
(include/bigwham_b200.h).

* ``HmatGpu``      -- device H-matrix (upload once, matvec / rmatvec / matmat).
* ``meshes``       -- synthetic crack meshes for the benchmark and the tests.
"""
from .hmat import HmatGpu  # noqa: F401
from ._capi import BigWhamError, LIB_PATH  # noqa: F401

__all__ = ["HmatGpu", "BigWhamError", "LIB_PATH"]
