"""B200-native Hopkins/SOCS aerial-image engine (drop-in for highuvlith-core's
imaging call).  Build the CUDA library with ``python -m highuvlith_b200.build``."""
from .api import (AerialImageResult, GridConfig, MaskConfig, OpticsConfig, SimulationEngine, SourceConfig,  # noqa: F401
                  UnevenPlan, rasterize_rects)
from ._lib import HuvError  # noqa: F401

__version__ = "0.1.0"
