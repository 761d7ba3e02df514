"""drifter_b200: B200-native (sm_100a) matrix-free operator path of DRIFTER.

The compute lives in libdrifter_b200.so (hand-written CUDA kernels behind the C ABI of
include/drifter_b200.h); this package is the host-side mirror of the reference's operator
and solver interfaces. Importing the package does not touch the GPU.
"""
from ._abi import DrfError, launch_count, lib  # noqa: F401

__version__ = "0.1.0"


def load():
    """Loads the CUDA library (raises ImportError if it was not built)."""
    return lib()
