"""voxelrt_b200: VoxelRT's plain per-frame GI path (brick->voxel DDA, 1-spp
path tracing, temporal reprojection, a-trous denoise, present) as
hand-written sm_100a CUDA kernels behind the C ABI in include/vrt.h.
"""
from ._lib import (HIT_DTYPE, VRT_SCENE_FULL, VRT_SCENE_RANDOM, VRT_SCENE_SMALL, VRT_SCENE_VOXELRT,
                   VRT_SCENE_VOXELRT_LAMPS, VrtError,
                   VrtFrameStats, VrtUniforms, lib)
from .api import (BRICK, FLAG_DENOISE, FLAG_TEMPORAL, VOXEL_SIZE, Batch, CameraPose, Context, Lighting,
                  RadianceCache, Scene, Server, Session,
                  camera_matrices, camera_spline, generate_scene, make_uniforms, uniforms_bytes)

__all__ = [
    "HIT_DTYPE", "VRT_SCENE_FULL", "VRT_SCENE_RANDOM", "VRT_SCENE_SMALL", "VRT_SCENE_VOXELRT",
    "VRT_SCENE_VOXELRT_LAMPS", "VrtError",
    "VrtFrameStats", "VrtUniforms", "lib", "BRICK", "FLAG_DENOISE", "FLAG_TEMPORAL", "VOXEL_SIZE", "CameraPose",
    "Batch", "Context", "Lighting", "RadianceCache", "Scene", "Server", "Session", "camera_matrices", "camera_spline", "generate_scene",
    "make_uniforms", "uniforms_bytes",
]
