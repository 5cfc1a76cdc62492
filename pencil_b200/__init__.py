"""pencil_b200 - B200 path-tracing core for the Pencil ray tracer.

The product is libpencil_gpu.so (include/pencil_gpu.h): hand-written sm_100a
CUDA kernels behind a C-ABI that replaces pencil::Renderer::render. This
package builds it in-tree and mirrors Pencil's host interface in Python.
"""
from . import _abi
from ._abi import GpuError
from .renderer import GpuContext, Renderer, RenderSettings, RenderStats, default_context
from .scene import CameraArgs, Light, Material, Scene

__all__ = ["GpuContext", "GpuError", "Renderer", "RenderSettings", "RenderStats",
           "default_context", "CameraArgs", "Light", "Material", "Scene"]
