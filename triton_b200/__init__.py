"""triton_b200: B200-native (sm_100a) time-stepping hot path of the TRITON
2-D shallow-water model behind a C ABI (include/triton_b200.h).

The compute runs in triton_b200/lib/libtriton_b200.so (hand-written CUDA);
this package is the Python side of that ABI: ``Domain`` (one simulation on
the GPU) and ``scenarios`` (seeded synthetic workloads in the reference's
data model).  There is no CPU implementation of the step in the product.
"""
from ._abi import EV_END, EV_LOG, EV_OBS, EV_PRINT, TriError, lib  # noqa: F401
from .domain import Domain  # noqa: F401

__all__ = ["Domain", "TriError", "lib", "EV_END", "EV_PRINT", "EV_OBS", "EV_LOG"]
