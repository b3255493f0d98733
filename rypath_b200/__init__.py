"""rypath_b200: the B200 (sm_100a) backend for rypath's spectral path-tracing hot path.

The compute path is librypath_cuda.so (hand-written CUDA + C ABI, include/rypath_cuda.h);
this package holds the ctypes binding and the host-side mirror of the reference's renderer
interface (``build_renderer`` / ``RenderScene.sample`` / ``render_progressive``).
"""

from . import abi  # noqa: F401
