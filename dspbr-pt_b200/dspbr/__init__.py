"""B200 path-tracing hot path of dspbr-pt behind the reference's embedding API.

Public surface: PathtracingViewport (viewport.py, mirror of
packages/lib/pathtracing_viewport.ts), the lower-level Context / DeviceScene /
DeviceIbl / Bvh wrappers of the C ABI (include/dspbr.h), the render Server
(server.py, continuous batching of viewport requests), and the seeded
synthetic workloads (synth.py).
"""
from .viewport import (Bvh, Context, DeviceIbl, DeviceScene, PathtracingCamera, PathtracingViewport,
                       createPathtracingViewport, look_at_matrix)
from .server import Server
from . import synth

__all__ = ["Bvh", "Context", "DeviceIbl", "DeviceScene", "PathtracingCamera", "PathtracingViewport", "Server",
           "createPathtracingViewport", "look_at_matrix", "synth"]
