"""grapher_b200: gviz's force-directed layout step on NVIDIA B200 (sm_100a).

The product is the C ABI library ``lib/libgvizcuda.so`` (include/gvizcuda.h)
and the gviz adapter (include/gvizCudaForceEmbedder.h). This package holds
its CUDA sources (csrc/), the build recipe (build.py) and a thin Python
binding used by tests and the benchmark.
"""
from ._native import FP32, FP64, MODEL_FR, MODEL_LINLOG, GvizCudaError  # noqa: F401
from .layout import ForceLayout  # noqa: F401
from . import graphs  # noqa: F401

__all__ = ["ForceLayout", "graphs", "MODEL_FR", "MODEL_LINLOG", "FP32", "FP64",
           "GvizCudaError"]
