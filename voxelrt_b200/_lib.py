"""ctypes view of include/vrt.h (libvrt.so).

The library is the product: this module only loads it and mirrors the C
structs.  A missing library is an ImportError -- there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "libvrt.so"

VRT_OK = 0
ERR_NAMES = {1: "INVALID", 2: "CUDA", 3: "OOM", 4: "NO_DEVICE", 5: "BUDGET", 6: "TIMEOUT", 7: "STATE"}

VRT_SCENE_VOXELRT = 0
VRT_SCENE_SMALL = 1
VRT_SCENE_FULL = 2
VRT_SCENE_RANDOM = 3
VRT_SCENE_VOXELRT_LAMPS = 4


class VrtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"VRT_ERR_{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class VrtUniforms(C.Structure):
    _fields_ = [
        ("invViewProj", C.c_float * 16),
        ("prevViewProj", C.c_float * 16),
        ("camPos", C.c_float * 4),
        ("prevCamPos", C.c_float * 4),
        ("sunDir", C.c_float * 4),
        ("sunRadiance", C.c_float * 4),
        ("params0", C.c_uint32 * 4),
        ("params1", C.c_float * 4),
        ("params2", C.c_uint32 * 4),
        ("params3", C.c_float * 4),
        ("params4", C.c_float * 4),
        ("params5", C.c_float * 4),
        ("params6", C.c_float * 4),
    ]


class VrtDeviceConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget_bytes", C.c_uint64)]


class VrtSessionConfig(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("firefly_clamp", C.c_float),
                ("accum_f32", C.c_int), ("keep_radiance_f32", C.c_int), ("path_kernel", C.c_int)]


class VrtTuning(C.Structure):
    _fields_ = [("refill_min", C.c_int), ("trace_blocks_per_sm", C.c_int), ("shade_blocks_per_sm", C.c_int),
                ("trace_variant", C.c_int), ("atrous_tile_rows", C.c_int), ("tail_wave", C.c_int)]


PATH_WAVEFRONT = 0
PATH_MEGAKERNEL = 1
PATH_BATCH_ONLY = 2


class VrtEditBox(C.Structure):
    _fields_ = [("x0", C.c_int), ("y0", C.c_int), ("z0", C.c_int), ("x1", C.c_int), ("y1", C.c_int),
                ("z1", C.c_int), ("value", C.c_uint32), ("pad", C.c_int)]


class VrtCompletion(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("session", C.c_int), ("pad", C.c_int), ("t_arrival", C.c_double),
                ("t_done", C.c_double)]


class VrtHit(C.Structure):
    _fields_ = [("t", C.c_float), ("n", C.c_float * 3), ("mat", C.c_uint32), ("voxel", C.c_int32 * 3),
                ("face", C.c_int32), ("steps", C.c_uint32), ("bytes", C.c_uint32), ("pad", C.c_uint32)]


HIT_DTYPE = np.dtype([("t", "<f4"), ("n", "<f4", 3), ("mat", "<u4"), ("voxel", "<i4", 3), ("face", "<i4"),
                      ("steps", "<u4"), ("bytes", "<u4"), ("pad", "<u4")])


class VrtFrameStats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("dda_outer", C.c_uint64), ("dda_inner", C.c_uint64),
                ("voxel_reads", C.c_uint64), ("pixels", C.c_uint64), ("ms_pathtrace", C.c_float),
                ("ms_temporal", C.c_float), ("ms_atrous", C.c_float), ("ms_present", C.c_float),
                ("ms_total", C.c_float), ("launches", C.c_uint32), ("trace_launches", C.c_uint32),
                ("ms_trace", C.c_float), ("cache_on", C.c_uint32), ("cache_queries", C.c_uint64),
                ("cache_samples", C.c_uint64), ("ms_cache", C.c_float), ("ms_reuse", C.c_float),
                ("trace_step_slots", C.c_uint64)]


class VrtLightStats(C.Structure):
    _fields_ = [("count", C.c_uint32), ("pad", C.c_uint32), ("total_weight", C.c_double), ("ms_list", C.c_float),
                ("ms_alias", C.c_float), ("ms_grid", C.c_float), ("pad2", C.c_float)]


class VrtCacheConfig(C.Structure):
    _fields_ = [("enabled", C.c_int), ("train_bounces", C.c_int), ("train_vertices", C.c_int),
                ("train_batch", C.c_int), ("train_steps", C.c_int), ("learning_rate", C.c_float),
                ("seed", C.c_uint32), ("pad", C.c_int)]


class VrtCameraPose(C.Structure):
    _fields_ = [("pos", C.c_double * 3), ("yaw", C.c_double), ("pitch", C.c_double), ("fov_y", C.c_double),
                ("near_z", C.c_double), ("far_z", C.c_double)]


class VrtLighting(C.Structure):
    _fields_ = [("sun_dir", C.c_float * 3), ("sun_cos_radius", C.c_float), ("sun_irradiance", C.c_float * 3),
                ("sky_intensity", C.c_float)]


assert C.sizeof(VrtUniforms) == 304
assert C.sizeof(VrtHit) == 48 == HIT_DTYPE.itemsize

P = C.c_void_p
I = C.c_int
U32 = C.c_uint32
SZ = C.c_size_t

# name -> (restype, argtypes)
SIGNATURES = {
    "vrt_abi_version": (I, []),
    "vrt_last_error_string": (C.c_char_p, []),
    "vrt_create": (I, [C.POINTER(VrtDeviceConfig), C.POINTER(P)]),
    "vrt_destroy": (I, [P]),
    "vrt_ctx_synchronize": (I, [P]),
    "vrt_ctx_bytes_in_use": (C.c_uint64, [P]),
    "vrt_scene_upload": (I, [P, P, I, C.POINTER(P)]),
    "vrt_scene_upload_prebuilt": (I, [P, P, P, P, I, C.POINTER(P)]),
    "vrt_scene_edit_box": (I, [P, I, I, I, I, I, I, U32]),
    "vrt_scene_read": (I, [P, P, P, P]),
    "vrt_scene_destroy": (I, [P]),
    "vrt_trace_rays": (I, [P, P, P, P, I, P]),
    "vrt_trace_rays_device": (I, [P, P, P, P, I, P]),
    "vrt_session_create": (I, [P, P, C.POINTER(VrtSessionConfig), C.POINTER(P)]),
    "vrt_session_destroy": (I, [P]),
    "vrt_session_set_scene": (I, [P, P]),
    "vrt_session_reset": (I, [P]),
    "vrt_frame": (I, [P, C.POINTER(VrtUniforms)]),
    "vrt_pass_pathtrace": (I, [P, C.POINTER(VrtUniforms)]),
    "vrt_pass_reuse_temporal": (I, [P, C.POINTER(VrtUniforms)]),
    "vrt_pass_reuse_spatial": (I, [P, C.POINTER(VrtUniforms)]),
    "vrt_pass_dupmap": (I, [P, C.POINTER(VrtUniforms)]),
    "vrt_session_set_pairing_sigma": (I, [P, C.c_float]),
    "vrt_make_pairing": (I, [P, P, SZ]),
    "vrt_pass_temporal": (I, [P, C.POINTER(VrtUniforms)]),
    "vrt_pass_atrous": (I, [P, C.POINTER(VrtUniforms), I]),
    "vrt_pass_present": (I, [P, C.POINTER(VrtUniforms)]),
    "vrt_end_frame": (I, [P]),
    "vrt_session_set_timing": (I, [P, I]),
    "vrt_session_set_tuning": (I, [P, C.POINTER(VrtTuning)]),
    "vrt_session_get_tuning": (I, [P, C.POINTER(VrtTuning)]),
    "vrt_session_autotune": (I, [P, C.POINTER(VrtUniforms), I, C.POINTER(VrtTuning), C.POINTER(C.c_float)]),
    "vrt_session_last_stats": (I, [P, C.POINTER(VrtFrameStats)]),
    "vrt_read_radiance": (I, [P, P, SZ]),
    "vrt_read_radiance_f32": (I, [P, P, SZ]),
    "vrt_read_albedo": (I, [P, P, SZ]),
    "vrt_read_gbuffer": (I, [P, P, SZ]),
    "vrt_read_accum": (I, [P, P, SZ]),
    "vrt_read_denoise": (I, [P, I, P, SZ]),
    "vrt_read_final": (I, [P, P, SZ]),
    "vrt_read_ldr": (I, [P, P, SZ]),
    "vrt_read_reservoirs": (I, [P, I, P, SZ]),
    "vrt_read_direct": (I, [P, P, SZ]),
    "vrt_read_dupmap": (I, [P, P, SZ]),
    "vrt_read_hdr": (I, [P, P, SZ]),
    "vrt_write_history": (I, [P, P, P]),
    "vrt_denoise_atrous_noalloc": (I, [P, I, P, P, I, I, P]),
    "vrt_session_checkpoint_size": (I, [P, C.POINTER(C.c_uint64)]),
    "vrt_session_checkpoint": (I, [P, P, C.c_uint64]),
    "vrt_session_restore": (I, [P, P, C.c_uint64]),
    "vrt_mlp_selftest_gemm": (I, [I, I, I, P, P, P]),
    "vrt_mlp_create": (I, [P, U32, C.POINTER(P)]),
    "vrt_mlp_destroy": (I, [P]),
    "vrt_mlp_num_params": (I, []),
    "vrt_mlp_get_params": (I, [P, P]),
    "vrt_mlp_set_params": (I, [P, P]),
    "vrt_mlp_encode_device": (I, [P, P, I, C.c_float, P]),
    "vrt_mlp_infer_device": (I, [P, P, I, C.c_float, P]),
    "vrt_mlp_gradient_device": (I, [P, P, P, I, C.c_float, P, C.POINTER(C.c_float)]),
    "vrt_mlp_train_device": (I, [P, P, P, I, C.c_float, C.c_float, I, C.POINTER(C.c_float)]),
    "vrt_mlp_check": (I, [P]),
    "vrt_selftest_bounded_wait": (I, [C.c_uint]),
    "vrt_selftest_present": (I, [P, P, P]),
    "vrt_scene_build_lights": (I, [P, P]),
    "vrt_scene_read_lights": (I, [P, P, C.c_size_t, P, C.c_size_t, P, C.c_size_t]),
    "vrt_hdr_accum_reset": (I, [P]),
    "vrt_hdr_accum_add": (I, [P]),
    "vrt_hdr_accumulate": (I, [P, P, U32, I]),
    "vrt_hdr_accum_read": (I, [P, P, C.c_size_t, C.POINTER(U32)]),
    "vrt_hdr_set_reference": (I, [P, P, C.c_size_t]),
    "vrt_hdr_frame_error": (I, [P, C.POINTER(C.c_double)]),
    "vrt_hdr_accum_error": (I, [P, C.POINTER(C.c_double)]),
    "vrt_session_set_cache": (I, [P, P]),
    "vrt_session_cache_mlp": (I, [P, C.POINTER(P)]),
    "vrt_session_read_cache_samples": (I, [P, P, P, I, C.POINTER(I)]),
    "vrt_server_create": (I, [P, C.POINTER(P), I, I, C.POINTER(P)]),
    "vrt_server_destroy": (I, [P]),
    "vrt_server_now": (C.c_double, [P]),
    "vrt_server_submit": (I, [P, I, C.POINTER(VrtUniforms), C.POINTER(VrtEditBox), I, C.c_double, P,
                              C.POINTER(C.c_uint64)]),
    "vrt_server_poll": (I, [P, C.POINTER(VrtCompletion), I, C.POINTER(I)]),
    "vrt_server_drain": (I, [P, C.POINTER(VrtCompletion), I, C.POINTER(I)]),
    "vrt_server_pending": (I, [P, C.POINTER(I), C.POINTER(I)]),
    "vrt_server_create_dynamic": (I, [P, I, C.c_longlong, I, C.POINTER(P)]),
    "vrt_server_open_session": (I, [P, P, C.POINTER(VrtSessionConfig), C.POINTER(C.c_uint64)]),
    "vrt_server_session_of": (I, [P, C.c_uint64, C.POINTER(I)]),
    "vrt_server_close_session": (I, [P, I]),
    "vrt_server_sessions": (I, [P, C.POINTER(I), C.POINTER(I)]),
    "vrt_server_set_sequential": (I, [P, I]),
    "vrt_server_set_solo_pixels": (I, [P, C.c_longlong]),
    "vrt_server_set_min_batch": (I, [P, I]),
    "vrt_batch_create": (I, [P, C.POINTER(P), I, C.POINTER(P)]),
    "vrt_batch_destroy": (I, [P]),
    "vrt_batch_frame": (I, [P, C.POINTER(VrtUniforms)]),
    "vrt_batch_frame_subset": (I, [P, P, I, C.POINTER(VrtUniforms)]),
    "vrt_batch_set_graph": (I, [P, I]),
    "vrt_batch_set_tuning": (I, [P, C.POINTER(VrtTuning)]),
    "vrt_batch_autotune": (I, [P, C.POINTER(VrtUniforms), I, C.POINTER(VrtTuning), C.POINTER(C.c_float)]),
    "vrt_batch_last_stats": (I, [P, C.POINTER(VrtFrameStats)]),
    "vrt_make_uniforms": (I, [C.POINTER(VrtCameraPose), C.POINTER(VrtCameraPose), C.POINTER(VrtLighting), U32, U32,
                              U32, I, I, C.c_float, C.c_float, C.POINTER(VrtUniforms)]),
    "vrt_camera_matrices": (I, [C.POINTER(VrtCameraPose), C.c_double, P, P]),
    "vrt_camera_spline": (I, [C.POINTER(VrtCameraPose), I, C.POINTER(VrtCameraPose)]),
    "vrt_scene_generate": (I, [I, I, U32, P, C.POINTER(VrtCameraPose)]),
}


def _load() -> C.CDLL:
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH} is missing: build it with `python -m voxelrt_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(str(_LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class _Lib:
    """Loads libvrt.so on first use (so the build step can import this
    package before the library exists); any use without the library raises."""

    _cdll = None

    def __getattr__(self, name):
        if _Lib._cdll is None:
            _Lib._cdll = _load()
        return getattr(_Lib._cdll, name)


lib = _Lib()


def check(code: int) -> None:
    if code != VRT_OK:
        raise VrtError(code, lib.vrt_last_error_string().decode(errors="replace"))


def ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)
