"""tileink_b200: B200-native (sm_100a) tile rasterization path of tileink.

Scene recording mirrors the reference's Canvas API (tileink_b200.canvas);
rendering goes through the C ABI in include/tileink.h (tileink_b200.renderer).
The CUDA library must be built in-tree first (python -m tileink_b200.build);
there is no CPU fallback.
"""
from .canvas import BezPath, Brush, Canvas, RetainedScene, generate, plan_line_tile_count, FILL_NONZERO, FILL_EVEN_ODD
from .renderer import NativeRenderer, TileinkError
from . import _native as native

__all__ = ["BezPath", "Brush", "Canvas", "RetainedScene", "generate", "plan_line_tile_count", "NativeRenderer", "TileinkError",
           "native", "FILL_NONZERO", "FILL_EVEN_ODD"]
