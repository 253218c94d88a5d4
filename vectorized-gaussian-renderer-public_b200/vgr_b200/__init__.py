"""B200-native batched Gaussian-splat sensor renderer.

Drop-in for the camera path of the reference ``isaacsim_gaussian_renderer``
package: the same service (``RendererService``), backend seam
(``GaussianRendererBackend``, ``CustomCudaBackend``), contracts and native
module surface (``native_module``), implemented over the C ABI of
libvgr_b200.so (include/vgr_b200.h).
"""

from .backend import GaussianRendererBackend, RenderRequest, RenderStats
from .contracts import OUTPUT_SPECS, ensure_tensor
from .cuda_backend import (
    COUNTER_NAMES,
    DEFAULT_GAUSSIAN_SUPPORT_SIGMA,
    CustomCudaBackend,
    RendererCapacityError,
)
from .native_module import NativeRendererModule, load_native_extension
from .renderer_service import RendererService
from .scene import GaussianScene, SceneRegistry

__all__ = [
    "COUNTER_NAMES",
    "DEFAULT_GAUSSIAN_SUPPORT_SIGMA",
    "CustomCudaBackend",
    "GaussianRendererBackend",
    "GaussianScene",
    "NativeRendererModule",
    "OUTPUT_SPECS",
    "RenderRequest",
    "RenderStats",
    "RendererCapacityError",
    "RendererService",
    "SceneRegistry",
    "ensure_tensor",
    "load_native_extension",
]
