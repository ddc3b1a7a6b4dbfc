"""rtlib_b200 -- B200-native (sm_100a) path-guiding hot path of RTLib.

The product is the native library librtpg.so (CUDA kernels + C ABI, include/rtpg.h); this
package is its thin Python host layer.
"""
from ._lib import RtpgError, lib  # noqa: F401

__all__ = ["RtpgError", "lib"]
