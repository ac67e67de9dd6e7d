"""gray_b200: B200-native geodesic hot path of GRay2 (luxsrc/gray).

The compute path is libgray_cuda.so (hand-written sm_100a kernels behind
the C ABI of include/gray_cuda.h).  There is no CPU fallback: importing
the API without the built library raises.
"""
from . import api, configs  # noqa: F401
from .api import Context, GrayError, make_desc, make_grid  # noqa: F401

__all__ = ["api", "configs", "Context", "GrayError", "make_desc", "make_grid"]
