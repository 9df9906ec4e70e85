"""B200-native strand software-raster path (Fiber / bevy_strand_rasterizer).

The compute path lives in libfiber.so (CUDA, sm_100a) behind include/fiber.h;
this package holds the host-side mirror of the reference's plugin API
(plugin.py), the ctypes ABI (abi.py), the `.strands` loader (strand_cache.py)
and seeded synthetic scenes (scene.py).
"""
from .plugin import (FineBinningBackend, FroxelConfig, PackedStrandBuffers, PrepassTelemetrySettings,
                     StochasticCullSettings, StrandList, StrandMaterial, StrandRasterizerPlugin, pack_indexed_strands,
                     pack_strand_set, pack_strands)

__all__ = [
    "FineBinningBackend", "FroxelConfig", "PackedStrandBuffers", "PrepassTelemetrySettings",
    "StochasticCullSettings", "StrandList", "StrandMaterial", "StrandRasterizerPlugin", "pack_indexed_strands",
    "pack_strand_set", "pack_strands",
]
