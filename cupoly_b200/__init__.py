"""cupoly_b200: a B200-native (sm_100a) engine for exact arithmetic in Z_q[x]/(x^nphi + 1).

It covers cuPoly's hot path (hierarchical DGT, RNS pointwise arithmetic, HPS
basis extension and t/Q scaling, sampling) behind cuPoly's own API:

* ``cupoly_b200.cupoly``  -- CUDAEngine / Context / poly_t / poly_* / DGTEngine / Sampler;
* ``cupoly_b200.engine``  -- per-instance engines over device tensors;
* ``cupoly_b200.batch``   -- fused, batched BFV multiplication under CUDA graphs;
* ``include/cupoly_b200.h`` -- the C ABI every call goes through.
"""
from . import _lib  # noqa: F401
from ._lib import CupolyError, LIB_PATH  # noqa: F401

__version__ = "0.1.0"


def native_library():
    """Load and return the native library (raises if it is not built)."""
    return _lib.lib()
