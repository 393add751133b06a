"""B200-native backend for XPRecon's iterative cone-beam reconstruction path.

The hot path (forward projector, error, multiplicative back-projection,
-log/normalise preprocessing) runs as sm_100a CUDA kernels in
``lib/libxpr.so`` behind the C ABI of ``include/xpr.h``; the ``xprecon`` tool in
``lib/`` is the drop-in for the reference's ``XPRecon`` command line.  This
package is the Python binding of that library; it has no fallback path.
"""
from ._lib import LIB_PATH, XprError, check, lib  # noqa: F401

__all__ = ["LIB_PATH", "XprError", "check", "lib"]
