"""Pythonic host interface over the C ABI, mirroring the reference renderer's
operator surface: a device context, a device-resident voxel scene
(generateScene + brick build, scene.js), per-view sessions holding the render
targets (main.js:335-360), and frame()/pass calls in the reference pass order
(main.js:680-772).
"""
from __future__ import annotations

import atexit
import ctypes as C
import math
import weakref
from dataclasses import dataclass

import numpy as np

from ._lib import (HIT_DTYPE, PATH_BATCH_ONLY, PATH_MEGAKERNEL, PATH_WAVEFRONT, VrtCameraPose, VrtCompletion,
                   VrtCacheConfig, VrtDeviceConfig, VrtEditBox, VrtLightStats, VrtFrameStats, VrtLighting, VrtSessionConfig, VrtTuning, VrtUniforms,
                   check, lib, ptr)

# Live handles, closed in dependency order when the interpreter exits (objects
# still alive at exit would otherwise be finalized in arbitrary order, after
# parts of the runtime they need are gone).
_LIVE = {k: weakref.WeakSet() for k in ("server", "batch", "cache", "session", "scene", "context")}


def _track(kind: str, obj) -> None:
    _LIVE[kind].add(obj)


def _ctx_alive(obj) -> bool:
    """False once the object's context was destroyed: destroying the object
    would go through the freed context, so its device memory is left to the
    process exit instead.  The garbage collector can finalize a context
    before the objects that refer to it when both sit in one unreachable
    cycle (a failed call's traceback, for one), after it has cleared the weak
    references through which the context would have closed them first."""
    c = getattr(obj, "ctx", None)
    return c is None or bool(getattr(c, "h", None))


@atexit.register
def _close_all() -> None:
    for kind in ("server", "batch", "cache", "session", "scene", "context"):
        for obj in list(_LIVE[kind]):
            try:
                obj.close()
            except Exception:
                pass


# Reference constants (scene.js:5-6, common.wgsl:11)
VOXEL_SIZE = 1.0 / 16.0
BRICK = 8
FLAG_TEMPORAL = 1
FLAG_DENOISE = 2


@dataclass
class Lighting:
    """Sun and sky (uniform slots sunDir / sunRadiance)."""
    sun_dir: tuple = (0.3, 0.8, 0.5)
    sun_cos_radius: float = math.cos(math.radians(0.27))
    sun_irradiance: tuple = (3.0, 3.0, 3.0)
    sky_intensity: float = 1.0

    def c(self) -> VrtLighting:
        l = VrtLighting()
        l.sun_dir[:] = [float(v) for v in self.sun_dir]
        l.sun_cos_radius = float(self.sun_cos_radius)
        l.sun_irradiance[:] = [float(v) for v in self.sun_irradiance]
        l.sky_intensity = float(self.sky_intensity)
        return l

    @staticmethod
    def reference_default() -> "Lighting":
        """main.js:402-412: azimuth 0.9, elevation 0.85, radius 0.03 rad, E=(5,4.5,3.8)."""
        el, az = 0.85, 0.9
        return Lighting((math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az)),
                        math.cos(0.03), (5.0, 4.5, 3.8), 1.0)


@dataclass
class CameraPose:
    pos: tuple
    yaw: float = 0.0
    pitch: float = 0.0
    fov_y: float = math.radians(70.0)
    near_z: float = 0.05
    far_z: float = 400.0

    def c(self) -> VrtCameraPose:
        p = VrtCameraPose()
        p.pos[:] = [float(v) for v in self.pos]
        p.yaw, p.pitch, p.fov_y, p.near_z, p.far_z = self.yaw, self.pitch, self.fov_y, self.near_z, self.far_z
        return p

    @staticmethod
    def from_c(p: VrtCameraPose) -> "CameraPose":
        return CameraPose(tuple(p.pos), p.yaw, p.pitch, p.fov_y, p.near_z, p.far_z)


def generate_scene(kind: int, n: int, seed: int):
    """Procedural voxel world (packed u32, N^3) and its default camera pose."""
    vox = np.empty(n * n * n, np.uint32)
    spawn = VrtCameraPose()
    check(lib.vrt_scene_generate(int(kind), int(n), int(seed) & 0xFFFFFFFF, ptr(vox), C.byref(spawn)))
    return vox, CameraPose.from_c(spawn)


def camera_spline(spawn: CameraPose, frame: int) -> CameraPose:
    out = VrtCameraPose()
    check(lib.vrt_camera_spline(C.byref(spawn.c()), int(frame), C.byref(out)))
    return CameraPose.from_c(out)


def camera_matrices(pose: CameraPose, aspect: float):
    vp = np.empty(16, np.float32)
    ivp = np.empty(16, np.float32)
    check(lib.vrt_camera_matrices(C.byref(pose.c()), float(aspect), ptr(vp), ptr(ivp)))
    return vp, ivp


# ReSTIR flag bits of params2.x (common.wgsl:40-59) and the presets built from
# them (main.js:34-62).  The library implements every flag of these presets,
# plus footprint, mixed sigma, adaptive candidate counts and the light grid;
# frames with confdenoise, mutate or worldgi set are rejected.
RF = {"restir": 1, "treuse": 2, "sreuse": 4, "paired": 8, "dupmap": 16, "footprint": 32, "vector": 64,
      "unified": 128, "plane": 256, "rescue": 512, "fullv": 1024, "rclamp": 2048, "lightpower": 4096,
      "mixsigma": 8192, "adaptcand": 16384, "confdenoise": 32768, "lightgrid": 65536, "mutate": 131072,
      "histisolate": 262144, "worldgi": 524288}
PRESETS = {
    "base": [],
    "gi": ["restir", "treuse", "sreuse"],
    "lin": ["restir", "treuse", "sreuse", "paired", "dupmap", "vector", "unified"],
    "ours": ["restir", "treuse", "sreuse", "paired", "dupmap", "vector", "unified", "plane", "rescue", "fullv",
             "rclamp", "lightpower"],
    "ours_motion": ["restir", "treuse", "sreuse", "paired", "dupmap", "vector", "unified", "plane", "rescue", "fullv",
                    "rclamp", "lightpower", "histisolate"],
}


def make_pairing(sigmas) -> np.ndarray:
    """The pairing textures of paired spatial reuse (pairing.js:80-89)."""
    sg = np.ascontiguousarray(sigmas, np.float64)
    out = np.zeros(254 * 254 + 230 * 230 + 210 * 210, np.uint32)
    check(lib.vrt_make_pairing(ptr(sg), ptr(out), out.size))
    return out


def preset_flags(preset: str) -> int:
    flags = 0
    for k in PRESETS[preset]:
        flags |= RF[k]
    return flags


def make_uniforms(cur: CameraPose, prev: CameraPose | None, light: Lighting, frame: int, bounces: int, flags: int,
                  width: int, height: int, exposure: float = 1.0, max_history: float = 64.0, preset: str = "base",
                  taps: int = 3, ccap: float = 20.0, radius: float = 30.0, light_count: int = 0) -> VrtUniforms:
    """The 304-byte uniform block (main.js:399-426).  preset selects the
    reservoir flags of params2.x; taps, ccap and radius are the reference's
    tuning defaults (main.js:72-76) in params2.z, params3.x, params4.x;
    light_count is the scene's emissive-face count (params2.y, read by
    unified NEE)."""
    u = VrtUniforms()
    check(lib.vrt_make_uniforms(C.byref(cur.c()), C.byref(prev.c()) if prev is not None else None,
                                C.byref(light.c()), int(frame) & 0xFFFFFFFF, int(bounces), int(flags), int(width),
                                int(height), float(exposure), float(max_history), C.byref(u)))
    u.params2[0] = preset_flags(preset)
    u.params2[1] = int(light_count)
    u.params2[2] = int(taps)
    u.params3[0] = float(ccap)
    u.params4[0] = float(radius)
    return u


def uniforms_bytes(u: VrtUniforms) -> bytes:
    return C.string_at(C.addressof(u), C.sizeof(u))


class Context:
    """A CUDA device with its own stream and an HBM admission budget."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        cfg = VrtDeviceConfig(int(device), int(hbm_budget_bytes))
        h = C.c_void_p()
        check(lib.vrt_create(C.byref(cfg), C.byref(h)))
        self.h = h
        _track("context", self)

    def synchronize(self) -> None:
        check(lib.vrt_ctx_synchronize(self.h))

    @property
    def bytes_in_use(self) -> int:
        return int(lib.vrt_ctx_bytes_in_use(self.h))

    def selftest_present(self) -> tuple[int, int]:
        """(mismatches, smallest differing bit pattern or 0xffffffff) of the
        present pass's threshold table against the exact arithmetic over every
        float of [0, 8) (vrt_selftest_present)."""
        n = C.c_uint64()
        f = C.c_uint32()
        check(lib.vrt_selftest_present(self.h, C.byref(n), C.byref(f)))
        return int(n.value), int(f.value)

    def close(self) -> None:
        if self.h:
            # objects of this context still open (a test that failed midway, a
            # caller that forgot one) go first: they need the context to close
            for kind in ("server", "batch", "cache", "session", "scene"):
                for obj in list(_LIVE[kind]):
                    if getattr(obj, "ctx", None) is self:
                        try:
                            obj.close()
                        except Exception:
                            pass
            lib.vrt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """Device-resident voxel grid + bricks + masks (+ occupancy bitmap)."""

    def __init__(self, ctx: Context, voxels: np.ndarray, n: int, bricks=None, masks=None):
        voxels = np.ascontiguousarray(voxels, np.uint32)
        assert voxels.size == n ** 3
        h = C.c_void_p()
        if bricks is None:
            check(lib.vrt_scene_upload(ctx.h, ptr(voxels), int(n), C.byref(h)))
        else:
            b = np.ascontiguousarray(bricks, np.uint32)
            m = np.ascontiguousarray(masks, np.uint32)
            check(lib.vrt_scene_upload_prebuilt(ctx.h, ptr(voxels), ptr(b), ptr(m), int(n), C.byref(h)))
        self.h, self.ctx, self.n = h, ctx, n
        _track("scene", self)

    def edit_box(self, x0, y0, z0, x1, y1, z1, value: int) -> None:
        check(lib.vrt_scene_edit_box(self.h, x0, y0, z0, x1, y1, z1, int(value) & 0xFFFFFFFF))

    def read(self):
        n, bg = self.n, self.n // BRICK
        v = np.empty(n ** 3, np.uint32)
        b = np.empty(bg ** 3, np.uint32)
        m = np.empty(16 * bg ** 3, np.uint32)
        check(lib.vrt_scene_read(self.h, ptr(v), ptr(b), ptr(m)))
        return v, b, m

    def trace_rays(self, origins: np.ndarray, dirs: np.ndarray, tmax: np.ndarray) -> np.ndarray:
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(tmax, np.float32).reshape(-1)
        n = o.shape[0]
        out = np.zeros(n, HIT_DTYPE)
        check(lib.vrt_trace_rays(self.h, ptr(o), ptr(d), ptr(t), n, ptr(out)))
        return out

    def build_lights(self):
        """Rebuild the light list, alias table and light grid from the current
        voxels (vrt_scene_build_lights); returns the build statistics."""
        st = VrtLightStats()
        check(lib.vrt_scene_build_lights(self.h, C.byref(st)))
        self._lights_n = int(st.count)
        return st

    def lights(self):
        """(words [n x 2] uint32, alias [max(n,1) x 4] float32, grid [cells x 34]
        uint32) of the last build_lights()."""
        n = getattr(self, "_lights_n", None)
        if n is None:
            raise RuntimeError("call build_lights() first")
        bg = self.n // BRICK
        words = np.zeros((n, 2), np.uint32)
        alias = np.zeros((max(n, 1), 4), np.float32)
        grid = np.zeros((bg ** 3, 34), np.uint32)
        check(lib.vrt_scene_read_lights(self.h, ptr(words), words.nbytes, ptr(alias), alias.nbytes, ptr(grid),
                                        grid.nbytes))
        return words, alias, grid

    def close(self) -> None:
        if self.h:
            if _ctx_alive(self):
                lib.vrt_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Session:
    """Render targets of one view (radiance, albedo, G-buffer x2, history x2,
    denoise x2, LDR) and the frame loop over them."""

    def __init__(self, ctx: Context, scene: Scene, width: int, height: int, firefly_clamp: float = 48.0,
                 accum_f32: bool = False, keep_radiance_f32: bool = False, path_kernel: str = "wavefront"):
        pk = {"wavefront": PATH_WAVEFRONT, "megakernel": PATH_MEGAKERNEL, "batch_only": PATH_BATCH_ONLY}[path_kernel]
        cfg = VrtSessionConfig(int(width), int(height), float(firefly_clamp), int(bool(accum_f32)),
                               int(bool(keep_radiance_f32)), pk)
        h = C.c_void_p()
        check(lib.vrt_session_create(ctx.h, scene.h, C.byref(cfg), C.byref(h)))
        self.h, self.ctx, self.scene = h, ctx, scene
        self.w, self.h_px = int(width), int(height)
        self.accum_f32 = bool(accum_f32)
        _track("session", self)

    # frame + passes --------------------------------------------------------
    def frame(self, u: VrtUniforms) -> None:
        check(lib.vrt_frame(self.h, C.byref(u)))

    def pathtrace(self, u): check(lib.vrt_pass_pathtrace(self.h, C.byref(u)))
    def reuse_temporal(self, u): check(lib.vrt_pass_reuse_temporal(self.h, C.byref(u)))
    def reuse_spatial(self, u): check(lib.vrt_pass_reuse_spatial(self.h, C.byref(u)))
    def dupmap(self, u): check(lib.vrt_pass_dupmap(self.h, C.byref(u)))
    def set_pairing_sigma(self, sigma: float): check(lib.vrt_session_set_pairing_sigma(self.h, float(sigma)))
    def temporal(self, u): check(lib.vrt_pass_temporal(self.h, C.byref(u)))
    def atrous(self, u, it): check(lib.vrt_pass_atrous(self.h, C.byref(u), int(it)))
    def present(self, u): check(lib.vrt_pass_present(self.h, C.byref(u)))
    def end_frame(self): check(lib.vrt_end_frame(self.h))
    def reset(self): check(lib.vrt_session_reset(self.h))

    def set_scene(self, scene: Scene) -> None:
        check(lib.vrt_session_set_scene(self.h, scene.h))
        self.scene = scene

    def set_tuning(self, refill_min: int = 0, trace_blocks_per_sm: int = 0, shade_blocks_per_sm: int = 0,
                   trace_variant: int = 0, atrous_tile_rows: int = 0, tail_wave: int = -1) -> None:
        t = VrtTuning(int(refill_min), int(trace_blocks_per_sm), int(shade_blocks_per_sm), int(trace_variant),
                      int(atrous_tile_rows), int(tail_wave))
        check(lib.vrt_session_set_tuning(self.h, C.byref(t)))

    def autotune(self, u: VrtUniforms, frames: int = 3):
        """Picks the fastest wavefront launch shape and a-trous tile shape for
        frames like `u`; resets history."""
        t = VrtTuning()
        ms = C.c_float()
        check(lib.vrt_session_autotune(self.h, C.byref(u), int(frames), C.byref(t), C.byref(ms)))
        return (t.refill_min, t.trace_blocks_per_sm, t.shade_blocks_per_sm, t.trace_variant,
                t.atrous_tile_rows, t.tail_wave), float(ms.value)

    def get_tuning(self) -> tuple:
        t = VrtTuning()
        check(lib.vrt_session_get_tuning(self.h, C.byref(t)))
        return (t.refill_min, t.trace_blocks_per_sm, t.shade_blocks_per_sm, t.trace_variant, t.atrous_tile_rows,
                t.tail_wave)

    def set_cache(self, enabled: bool = True, train_bounces: int = 6, train_vertices: int = 3,
                  train_batch: int = 65536, train_steps: int = 1, learning_rate: float = 1e-2, seed: int = 1) -> None:
        """Cache-assisted path tracing (vrt_session_set_cache)."""
        cfg = VrtCacheConfig(int(bool(enabled)), int(train_bounces), int(train_vertices), int(train_batch),
                             int(train_steps), float(learning_rate), int(seed) & 0xFFFFFFFF, 0)
        check(lib.vrt_session_set_cache(self.h, C.byref(cfg)))

    def cache_params(self) -> np.ndarray:
        """FP32 master weights of the session's cache network."""
        m = C.c_void_p()
        check(lib.vrt_session_cache_mlp(self.h, C.byref(m)))
        if not m.value:
            raise RuntimeError("the cache was never enabled on this session")
        out = np.zeros(RadianceCache.N_PARAMS, np.float32)
        check(lib.vrt_mlp_get_params(m, ptr(out)))
        return out

    def set_cache_params(self, p: np.ndarray) -> None:
        m = C.c_void_p()
        check(lib.vrt_session_cache_mlp(self.h, C.byref(m)))
        if not m.value:
            raise RuntimeError("the cache was never enabled on this session")
        p = np.ascontiguousarray(p, np.float32)
        check(lib.vrt_mlp_set_params(m, ptr(p)))

    def cache_samples(self, cap: int | None = None):
        """(q9 [n x 9], y3 [n x 3], produced) of the last cache-assisted frame."""
        if cap is None:
            cap = ((self.w + 3) // 4) * ((self.h_px + 3) // 4) * 8
        q = np.zeros((cap, 9), np.float32)
        y = np.zeros((cap, 3), np.float32)
        n = C.c_int()
        check(lib.vrt_session_read_cache_samples(self.h, ptr(q), ptr(y), int(cap), C.byref(n)))
        k = min(n.value, cap)
        return q[:k], y[:k], n.value

    # HDR reference pipeline ------------------------------------------------
    def hdr_accum_reset(self) -> None:
        check(lib.vrt_hdr_accum_reset(self.h))

    def hdr_accum_add(self) -> None:
        check(lib.vrt_hdr_accum_add(self.h))

    def hdr_accumulate(self, u: VrtUniforms, frame0: int, spp: int) -> None:
        """spp path-trace passes (frames frame0..), their HDR radiance summed in FP64."""
        check(lib.vrt_hdr_accumulate(self.h, C.byref(u), C.c_uint32(frame0), int(spp)))

    def hdr_accum_sums(self):
        """(FP64 sums H x W x 3, frames added)."""
        out = np.zeros((self.h_px, self.w, 3), np.float64)
        n = C.c_uint32()
        check(lib.vrt_hdr_accum_read(self.h, ptr(out), out.nbytes, C.byref(n)))
        return out, int(n.value)

    def hdr_accum(self):
        """(mean HDR image H x W x 3 float64, frames added)."""
        sums, n = self.hdr_accum_sums()
        return sums / max(n, 1), n

    def set_hdr_reference(self, img: np.ndarray) -> None:
        ref = np.ascontiguousarray(img, np.float32)
        if ref.shape != (self.h_px, self.w, 3):
            raise ValueError("reference must be H x W x 3")
        check(lib.vrt_hdr_set_reference(self.h, ptr(ref), ref.nbytes))

    def hdr_frame_mse(self) -> float:
        """MSE of the last frame's HDR radiance against the reference (on the device)."""
        v = C.c_double()
        check(lib.vrt_hdr_frame_error(self.h, C.byref(v)))
        return v.value / (self.w * self.h_px * 3)

    def hdr_accum_mse(self) -> float:
        """MSE of the accumulated mean against the reference (on the device)."""
        v = C.c_double()
        check(lib.vrt_hdr_accum_error(self.h, C.byref(v)))
        return v.value / (self.w * self.h_px * 3)

    def set_timing(self, on: bool) -> None:
        check(lib.vrt_session_set_timing(self.h, int(bool(on))))

    def stats(self) -> VrtFrameStats:
        s = VrtFrameStats()
        check(lib.vrt_session_last_stats(self.h, C.byref(s)))
        return s

    # readbacks -------------------------------------------------------------
    def _read(self, fn, dtype, comps, *extra):
        a = np.empty((self.h_px, self.w, comps), dtype)
        check(fn(self.h, *extra, ptr(a), a.nbytes))
        return a

    def radiance(self): return self._read(lib.vrt_read_radiance, np.uint16, 4)
    def radiance_f32(self): return self._read(lib.vrt_read_radiance_f32, np.float32, 4)
    def albedo(self): return self._read(lib.vrt_read_albedo, np.uint8, 4)
    def gbuffer(self): return self._read(lib.vrt_read_gbuffer, np.float32, 4)
    def ldr(self): return self._read(lib.vrt_read_ldr, np.uint8, 4)
    def denoise(self, i): return self._read(lib.vrt_read_denoise, np.uint16, 4, int(i))
    def reservoirs(self, which: int): return self._read(lib.vrt_read_reservoirs, np.uint32, 8, int(which))
    def direct(self): return self._read(lib.vrt_read_direct, np.uint16, 4)
    def dupmap_image(self): return self._read(lib.vrt_read_dupmap, np.float32, 1)[..., 0]

    def accum(self):
        return self._read(lib.vrt_read_accum, np.float32 if self.accum_f32 else np.uint16, 4)

    def final(self, denoised: bool):
        f32 = self.accum_f32 and not denoised
        return self._read(lib.vrt_read_final, np.float32 if f32 else np.uint16, 4)

    def hdr(self):
        a = np.empty((self.h_px, self.w, 3), np.float32)
        check(lib.vrt_read_hdr(self.h, ptr(a), a.nbytes))
        return a

    def checkpoint(self) -> bytes:
        """The session's state as bytes (vrt_session_checkpoint)."""
        n = C.c_uint64()
        check(lib.vrt_session_checkpoint_size(self.h, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        check(lib.vrt_session_checkpoint(self.h, ptr(buf), n.value))
        return buf.tobytes()

    def restore(self, state: bytes) -> None:
        """Loads a checkpoint of a session of the same size (vrt_session_restore)."""
        buf = np.frombuffer(state, np.uint8)
        check(lib.vrt_session_restore(self.h, ptr(buf), buf.size))

    def write_history(self, accum_prev: np.ndarray | None, gbuf_prev: np.ndarray | None) -> None:
        a = None if accum_prev is None else np.ascontiguousarray(accum_prev)
        g = None if gbuf_prev is None else np.ascontiguousarray(gbuf_prev, np.float32)
        check(lib.vrt_write_history(self.h, ptr(a) if a is not None else None, ptr(g) if g is not None else None))

    def close(self) -> None:
        if self.h:
            if _ctx_alive(self):
                lib.vrt_session_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """One frame for each of several sessions in a single launch sequence
    (replayed as a CUDA graph); images equal each session rendered alone."""

    def __init__(self, ctx: Context, sessions: list):
        arr = (C.c_void_p * len(sessions))(*[s.h for s in sessions])
        h = C.c_void_p()
        check(lib.vrt_batch_create(ctx.h, arr, len(sessions), C.byref(h)))
        self.h, self.ctx, self.sessions = h, ctx, list(sessions)
        _track("batch", self)

    def frame(self, uniforms: list) -> None:
        arr = (VrtUniforms * len(uniforms))(*uniforms)
        check(lib.vrt_batch_frame(self.h, arr))

    def set_graph(self, on: bool) -> None:
        check(lib.vrt_batch_set_graph(self.h, int(bool(on))))

    def set_tuning(self, refill_min=0, trace_blocks_per_sm=0, shade_blocks_per_sm=0, trace_variant=0,
                   atrous_tile_rows=0, tail_wave=-1) -> None:
        t = VrtTuning(int(refill_min), int(trace_blocks_per_sm), int(shade_blocks_per_sm), int(trace_variant),
                      int(atrous_tile_rows), int(tail_wave))
        check(lib.vrt_batch_set_tuning(self.h, C.byref(t)))

    def autotune(self, uniforms: list, frames: int = 2):
        arr = (VrtUniforms * len(uniforms))(*uniforms)
        t = VrtTuning()
        ms = C.c_float()
        check(lib.vrt_batch_autotune(self.h, arr, int(frames), C.byref(t), C.byref(ms)))
        return (t.refill_min, t.trace_blocks_per_sm, t.shade_blocks_per_sm, t.trace_variant, t.atrous_tile_rows,
                t.tail_wave), float(ms.value)

    def stats(self) -> VrtFrameStats:
        s = VrtFrameStats()
        check(lib.vrt_batch_last_stats(self.h, C.byref(s)))
        return s

    def close(self) -> None:
        if self.h:
            if _ctx_alive(self):
                lib.vrt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous batching over device-resident sessions (vrt_server_*)."""

    def __init__(self, ctx: Context, sessions: list | None, max_in_flight: int = 2, max_sessions: int = 0,
                 max_pixels: int = 0):
        """sessions: the fixed set of served sessions; or None for a server whose
        sessions come and go through open_session / close_session, with
        `max_sessions` slots and a launch pool of `max_pixels` pixels."""
        h = C.c_void_p()
        if sessions is None:
            check(lib.vrt_server_create_dynamic(ctx.h, int(max_sessions), int(max_pixels), int(max_in_flight),
                                                C.byref(h)))
        else:
            arr = (C.c_void_p * len(sessions))(*[s.h for s in sessions])
            check(lib.vrt_server_create(ctx.h, arr, len(sessions), int(max_in_flight), C.byref(h)))
        self.h, self.ctx, self.sessions = h, ctx, list(sessions or [])
        self._buf = (VrtCompletion * 4096)()
        _track("server", self)

    def open_session(self, scene: Scene, width: int, height: int, firefly_clamp: float = 48.0,
                     accum_f32: bool = False, path_kernel: str = "batch_only") -> int:
        """Queues a session for admission by the HBM budget; returns its ticket."""
        pk = {"wavefront": PATH_WAVEFRONT, "megakernel": PATH_MEGAKERNEL, "batch_only": PATH_BATCH_ONLY}[path_kernel]
        cfg = VrtSessionConfig(int(width), int(height), float(firefly_clamp), int(bool(accum_f32)), 0, pk)
        t = C.c_uint64()
        check(lib.vrt_server_open_session(self.h, scene.h, C.byref(cfg), C.byref(t)))
        return int(t.value)

    def session_of(self, ticket: int):
        """The slot of an admitted session, or None while it waits for admission."""
        k = C.c_int()
        code = lib.vrt_server_session_of(self.h, C.c_uint64(ticket), C.byref(k))
        if code == 7:      # VRT_ERR_STATE: still waiting
            return None
        check(code)
        return int(k.value)

    def close_session(self, slot: int) -> None:
        check(lib.vrt_server_close_session(self.h, int(slot)))

    def session_counts(self) -> tuple:
        """(open sessions, sessions waiting for admission)."""
        o, w = C.c_int(), C.c_int()
        check(lib.vrt_server_sessions(self.h, C.byref(o), C.byref(w)))
        return int(o.value), int(w.value)

    def set_sequential(self, on: bool) -> None:
        check(lib.vrt_server_set_sequential(self.h, int(bool(on))))

    def set_solo_pixels(self, pixels: int) -> None:
        """Sessions of at least `pixels` pixels (with their own path scratch)
        render alone; smaller ones are batched (0: batch everything)."""
        check(lib.vrt_server_set_solo_pixels(self.h, int(pixels)))

    def set_min_batch(self, sessions: int) -> None:
        """While fewer than `sessions` sessions have pending requests, requests
        render alone through their own frame path (1: always batch)."""
        check(lib.vrt_server_set_min_batch(self.h, int(sessions)))

    def now(self) -> float:
        return float(lib.vrt_server_now(self.h))

    def submit(self, session: int, u: VrtUniforms, edits=(), t_arrival: float = -1.0, ldr_out=None) -> int:
        """edits: iterable of (x0, y0, z0, x1, y1, z1, value); ldr_out: uint8 array of W*H*4 or None."""
        eds = (VrtEditBox * max(1, len(edits)))(*[VrtEditBox(*e, 0) for e in edits]) if edits else None
        t = C.c_uint64()
        check(lib.vrt_server_submit(self.h, int(session), C.byref(u), eds, len(edits), float(t_arrival),
                                    ptr(ldr_out) if ldr_out is not None else None, C.byref(t)))
        return int(t.value)

    def _collect(self, fn):
        n = C.c_int()
        check(fn(self.h, self._buf, len(self._buf), C.byref(n)))
        return [(c.ticket, c.session, c.t_arrival, c.t_done) for c in self._buf[:n.value]]

    def poll(self):
        return self._collect(lib.vrt_server_poll)

    def drain(self):
        out = []
        while True:
            got = self._collect(lib.vrt_server_drain)
            out += got
            q, f = C.c_int(), C.c_int()
            check(lib.vrt_server_pending(self.h, C.byref(q), C.byref(f)))
            if q.value == 0 and f.value == 0:
                return out

    def close(self) -> None:
        if self.h:
            if _ctx_alive(self):
                lib.vrt_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RadianceCache:
    """The radiance-cache MLP (vrt_mlp_*): BF16 tensor-core inference and
    training on device buffers.  Device arrays are torch CUDA tensors
    (contiguous float32; encoded features uint16/int16); each call orders
    itself after the caller's CUDA work and finishes before it returns."""

    N_PARAMS = 14336

    def __init__(self, ctx: Context, seed: int = 1, extent: float = 16.0):
        h = C.c_void_p()
        check(lib.vrt_mlp_create(ctx.h, C.c_uint32(seed & 0xFFFFFFFF), C.byref(h)))
        self.h, self.ctx, self.extent = h, ctx, float(extent)
        _track("cache", self)

    @staticmethod
    def _dp(t):
        import torch
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()):
            raise ValueError("expected a contiguous CUDA tensor")
        return C.c_void_p(t.data_ptr())

    @staticmethod
    def _sync():
        import torch
        torch.cuda.synchronize()

    def params(self) -> np.ndarray:
        out = np.zeros(self.N_PARAMS, np.float32)
        check(lib.vrt_mlp_get_params(self.h, ptr(out)))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.N_PARAMS:
            raise ValueError("wrong parameter count")
        check(lib.vrt_mlp_set_params(self.h, ptr(p)))

    def encode(self, q9, out) -> None:
        self._sync()
        check(lib.vrt_mlp_encode_device(self.h, self._dp(q9), q9.numel() // 9, C.c_float(self.extent), self._dp(out)))
        self.ctx.synchronize()

    def infer(self, q9, out3) -> None:
        self._sync()
        check(lib.vrt_mlp_infer_device(self.h, self._dp(q9), q9.numel() // 9, C.c_float(self.extent), self._dp(out3)))
        self.ctx.synchronize()
        check(lib.vrt_mlp_check(self.h))

    def gradient(self, q9, y3, grad_out=None) -> float:
        self._sync()
        loss = C.c_float()
        check(lib.vrt_mlp_gradient_device(self.h, self._dp(q9), self._dp(y3), q9.numel() // 9,
                                          C.c_float(self.extent),
                                          self._dp(grad_out) if grad_out is not None else None, C.byref(loss)))
        self.ctx.synchronize()
        return float(loss.value)

    def train(self, q9, y3, lr: float = 1e-3, steps: int = 1) -> float:
        """`steps` Adam steps; returns the loss before the first one."""
        self._sync()
        loss = C.c_float()
        check(lib.vrt_mlp_train_device(self.h, self._dp(q9), self._dp(y3), q9.numel() // 9, C.c_float(self.extent),
                                       C.c_float(lr), int(steps), C.byref(loss)))
        self.ctx.synchronize()
        check(lib.vrt_mlp_check(self.h))
        return float(loss.value)

    def close(self) -> None:
        if getattr(self, "h", None):
            if _ctx_alive(self):
                check(lib.vrt_mlp_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
