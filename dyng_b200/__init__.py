"""dyng_b200: dynG's batch-dynamic single-source shortest-path update, built for NVIDIA B200.

The device path is the CUDA library dyng_b200/libdyngb200.so (C ABI: include/dyngb200.h); this
package binds it with ctypes and mirrors the reference's Python names (dyng.Graph, dyng.EdgeBatch,
dyng.sssp.compute / update, dyng.mosp.compute / update).  There is no CPU fallback.
"""
from . import mosp, sssp
from .graph import (ApplySummary, CapacityError, CSR, CudaError, DyngError, EdgeBatch, Graph,
                    GraphProperties, InternalError, InvalidArgumentError, NotSupportedError,
                    OutOfMemoryError, Resources, StaleResultError, default_resources)

__all__ = ["sssp", "mosp", "ApplySummary", "CSR", "EdgeBatch", "Graph", "GraphProperties", "Resources",
           "default_resources", "DyngError", "InvalidArgumentError", "NotSupportedError",
           "StaleResultError", "OutOfMemoryError", "CudaError", "CapacityError", "InternalError"]
