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


def test_scene_lamps_variant(vrt):
    """scene.js generateScene(N, 'lamps') (scene.js:303-409): the default world
    with the room's ceiling strip replaced by dim strips, coloured panels,
    occluders and small bright lamps, dimmed exterior lanterns and no corner
    lamp -- every other voxel as in the default world."""
    n = 256
    d, sd = vrt.generate_scene(vrt.VRT_SCENE_VOXELRT, n, 1337)
    a, sa = vrt.generate_scene(vrt.VRT_SCENE_VOXELRT_LAMPS, n, 1337)
    b, _ = vrt.generate_scene(vrt.VRT_SCENE_VOXELRT_LAMPS, n, 1337)
    assert np.array_equal(a, b) and sa == sd
    # differences only in the room (walls 2 voxels thick) and at the three lanterns
    room_w = min(80, n * 45 // 100)
    cx, cz = n // 2, int(n * 0.55)
    x0, x1, z0, z1 = cx - room_w // 2, cx + room_w // 2, cz - room_w // 2, cz + room_w // 2
    z, y, x = np.unravel_index(np.nonzero(a != d)[0], (n, n, n))
    in_room = (x >= x0 - 2) & (x <= x1 + 2) & (z >= z0 - 2) & (z <= z1 + 2)
    lanterns = [(int(n * 0.35), int(n * 0.25)), (int(n * 0.68), int(n * 0.30)), (int(n * 0.25), int(n * 0.65))]
    at_lantern = np.zeros_like(in_room)
    for lx, lz in lanterns:
        at_lantern |= (np.abs(x - lx) <= 1) & (np.abs(z - lz) <= 1)
    assert x.size > 0 and np.all(in_room | at_lantern)
    # the variant's emitters: hot lamps (E 255), four panels, dim strips (E 45), dimmed lanterns (E 64)
    emis = {int(v) for v in np.unique(a[(a >> 24) != 0])}
    def m(r, g, bl, e):
        return r | g << 8 | bl << 16 | e << 24
    for want in (m(255, 214, 150, 255), m(255, 140, 40, 200), m(40, 220, 200, 165), m(190, 80, 255, 245),
                 m(150, 255, 60, 125), m(140, 180, 255, 45), m(255, 190, 110, 64), m(90, 220, 255, 64),
                 m(255, 90, 200, 64)):
        assert want in emis, hex(want)
    assert m(255, 240, 220, 210) not in emis          # no ceiling strip
    assert m(255, 190, 110, 255) not in emis          # no full-power warm lantern or corner lamp


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


def test_noalloc_denoise_rejects_overlapping_output(vrt):
    """vrt_denoise_atrous_noalloc checks its buffers before it touches a
    device: an output that overlaps the history or the G-buffer (an in-place
    denoise, whose first iteration would read neighbours other threads are
    overwriting) is rejected with VRT_ERR_INVALID.  The pointers here are
    never dereferenced."""
    lib = vrt.lib
    W, H = 64, 32
    px = W * H
    base = 1 << 20
    acc, gb = base, base + px * 16 * 4
    for acc_f32, out in [(0, acc), (0, acc + px * 8 - 8), (1, acc + px * 16 - 8), (0, gb), (0, gb + px * 16 - 8),
                         (0, acc - px * 8 + 8)]:
        code = lib.vrt_denoise_atrous_noalloc(C.c_void_p(acc), acc_f32, C.c_void_p(gb), C.c_void_p(out), W, H, None)
        assert code == 1, (acc_f32, out - base)
        assert "overlaps" in lib.vrt_last_error_string().decode()
