"""C-ABI library checks that need no GPU: the library loads, exports every
function include/vrt.h declares, and its host-only helpers behave."""
import ctypes as C
import math
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    src = (ROOT / "include" / "vrt.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vrt_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol(vrt):
    names = declared_functions()
    assert len(names) >= 39
    for n in names:
        assert hasattr(vrt.lib, n), f"libvrt.so does not export {n}"


def test_abi_version(vrt):
    assert vrt.lib.vrt_abi_version() == 1


def test_no_device_is_reported_without_gpu(vrt):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(vrt.VrtError) as e:
        vrt.Context(0)
    assert e.value.code == 4  # VRT_ERR_NO_DEVICE


def test_scene_generate_deterministic(vrt):
    for kind, n, seed in [(0, 64, 1337), (1, 64, 1), (2, 64, 2), (3, 64, 3)]:
        a, sa = vrt.generate_scene(kind, n, seed)
        b, sb = vrt.generate_scene(kind, n, seed)
        assert np.array_equal(a, b)
        assert sa == sb
        solid = (a != 0).mean()
        assert 0.05 < solid < 0.6
        if kind != 0:   # scene.js places its spawn in metres; it leaves small grids
            assert all(0 < p < n / 16 for p in sa.pos), sa


def test_small_scene_contents(vrt):
    vox, spawn = vrt.generate_scene(1, 64, 1)
    g = vox.reshape(64, 64, 64)
    e = (g >> 24) & 0xFF
    assert (e == round(10 * 255 / 24)).sum() == 36          # 6x6 emissive panel, intensity 10
    assert e[e != 0].size == 36
    terrain_cols = (g[:, :21, :] != 0).any(1)
    assert terrain_cols.all()
    assert math.isclose(spawn.fov_y, math.radians(60))


def test_full_scene_contents(vrt):
    vox, spawn = vrt.generate_scene(2, 256, 2)
    e = (vox >> 24) & 0xFF
    assert (e == round(15 * 255 / 24)).sum() == 3 * 27      # three 3x3x3 RGB lanterns of intensity 15
    assert (vox == 0x2a445f).sum() > 40 * 20                 # trunks of 40 trees


def test_random_scene_emissive_fraction(vrt):
    vox, _ = vrt.generate_scene(3, 128, 11)
    solid = vox != 0
    em = ((vox >> 24) & 0xFF) != 0
    frac = em.sum() / solid.sum()
    assert 0.0006 < frac < 0.0014


def test_camera_matrices_match_oracle(vrt, orc):
    pose = vrt.CameraPose((8.0, 5.2125, 2.5), -0.5236, -0.05, math.radians(60))
    for aspect in (16 / 9, 1.0, 256 / 144):
        vp, ivp = vrt.camera_matrices(pose, aspect)
        ovp, oivp = orc.camera_matrices(pose.pos, pose.yaw, pose.pitch, pose.fov_y, aspect)
        assert np.array_equal(vp.view(np.uint32), ovp.view(np.uint32))
        assert np.array_equal(ivp.view(np.uint32), oivp.view(np.uint32))


def test_uniform_block_layout(vrt):
    cur = vrt.CameraPose((1.0, 2.0, 3.0), 0.1, -0.2, math.radians(60))
    prev = vrt.CameraPose((1.5, 2.0, 3.0), 0.0, -0.2, math.radians(60))
    light = vrt.Lighting()
    u = vrt.make_uniforms(cur, prev, light, 7, 2, 3, 320, 180, 1.5, 64.0)
    raw = np.frombuffer(vrt.uniforms_bytes(u), np.uint8)
    f = raw.view(np.float32)
    i = raw.view(np.uint32)
    assert raw.size == 304
    assert tuple(f[32:35]) == pytest.approx((1.0, 2.0, 3.0))
    assert tuple(f[36:39]) == pytest.approx((1.5, 2.0, 3.0))
    sd = f[40:43].astype(np.float64)
    assert np.linalg.norm(sd) == pytest.approx(1.0, abs=1e-6)
    assert f[43] == np.float32(math.cos(math.radians(0.27)))
    assert tuple(i[48:51]) == (7, 2, 3)
    assert tuple(f[52:55]) == (320.0, 180.0, 1.5)
    assert i[56] == 0                                     # plain path: no ReSTIR flags
    assert f[65] == 64.0                                  # params4.y = max history
    vp, _ = vrt.camera_matrices(prev, 320 / 180)
    assert np.array_equal(f[16:32], vp)                   # prevViewProj from the previous pose


def test_spline_advances(vrt):
    _, spawn = vrt.generate_scene(2, 256, 2)
    p1 = vrt.camera_spline(spawn, 1)
    p120 = vrt.camera_spline(spawn, 120)
    step = math.dist(spawn.pos, p1.pos)
    assert step == pytest.approx(0.05)
    assert p120.yaw - spawn.yaw == pytest.approx(math.radians(60))


def test_invalid_arguments(vrt):
    vox = np.zeros(8 ** 3, np.uint32)
    code = vrt.lib.vrt_scene_generate(0, 12, 0, C.c_void_p(vox.ctypes.data), None)
    assert code == 1
    assert vrt.lib.vrt_scene_generate(9, 8, 0, C.c_void_p(vox.ctypes.data), None) == 1
    assert vrt.lib.vrt_trace_rays(None, None, None, None, 1, None) == 1
    assert "bad argument" in vrt.lib.vrt_last_error_string().decode()
