"""plamatrix_b200: B200 (sm_100a) implementation of PlaMatrix's Levenberg-Marquardt
normal-equation hot path behind the reference's API.

Native code lives in libplamatrix_b200.so (C ABI: include/plamatrix_b200.h); this
package is the Python mirror of the reference's interface for that path.
"""
from . import _native  # noqa: F401

__all__ = ["_native"]
