"""Batched frames (vrt_batch_*): several sessions rendered in one launch
sequence must produce exactly the images each session produces alone."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (scene kind, N, seed, W, H, bounces, clamp, accum_f32, flags)
JOBS = [
    (1, 64, 1, 256, 144, 2, 10.0, False, 3),
    (2, 256, 2, 320, 180, 3, 10.0, False, 3),
    (3, 128, 7, 257, 131, 1, 48.0, True, 3),
    (0, 256, 1337, 200, 120, 6, 0.0, False, 1),
    (3, 64, 9, 96, 54, 4, 10.0, True, 0),
    (2, 128, 5, 333, 77, 2, 10.0, False, 3),
]


@pytest.fixture(scope="module")
def ctx(vrt):
    c = vrt.Context(0)
    yield c
    c.close()


def _poses(vrt, spawn, f):
    pose = vrt.camera_spline(spawn, f)
    prev = vrt.camera_spline(spawn, f - 1) if f else None
    return pose, prev


def _outputs(s):
    out = {"rad": s.radiance(), "alb": s.albedo(), "gbuf": s.gbuffer(), "acc": s.accum(), "ldr": s.ldr()}
    out["den0"] = s.denoise(0)
    return out


def _check_same(a, b, what):
    for k in a:
        assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), f"{what}: {k} differs"


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_equals_sessions_alone(ctx, vrt, use_graph):
    scenes, spawns, alone, inbatch = [], [], [], []
    for kind, n, seed, W, H, nb, fc, f32, flags in JOBS:
        vox, spawn = vrt.generate_scene(kind, n, seed)
        if kind == 0:
            spawn = vrt.CameraPose((n / 32.0, n / 40.0, n / 64.0), 0.2, -0.1, math.radians(70))
        sc = vrt.Scene(ctx, vox, n)
        scenes.append(sc)
        spawns.append(spawn)
        alone.append(vrt.Session(ctx, sc, W, H, firefly_clamp=fc, accum_f32=f32, keep_radiance_f32=True))
        inbatch.append(vrt.Session(ctx, sc, W, H, firefly_clamp=fc, accum_f32=f32, keep_radiance_f32=True,
                                   path_kernel="batch_only"))
    batch = vrt.Batch(ctx, inbatch)
    batch.set_graph(use_graph)
    light = vrt.Lighting()
    for f in range(3):
        us = []
        for i, (kind, n, seed, W, H, nb, fc, f32, flags) in enumerate(JOBS):
            pose, prev = _poses(vrt, spawns[i], f)
            bounces = nb if f != 2 else max(1, nb - 1)      # bounce change forces a new graph
            us.append(vrt.make_uniforms(pose, prev, light, 100 + f, bounces, flags, W, H))
        batch.frame(us)
        st = batch.stats()
        rays = 0
        for i in range(len(JOBS)):
            alone[i].set_timing(True)
            alone[i].frame(us[i])
            rays += alone[i].stats().rays
            _check_same(_outputs(alone[i]), _outputs(inbatch[i]), f"frame {f} job {i}")
            assert np.array_equal(alone[i].radiance_f32().view(np.uint32), inbatch[i].radiance_f32().view(np.uint32))
        assert st.rays == rays
        assert st.pixels == sum(W * H for _, _, _, W, H, *_ in JOBS)
    batch.close()
    for s in alone + inbatch:
        s.close()
    for sc in scenes:
        sc.close()


@pytest.mark.parametrize("acc_f32", [False, True])
def test_large_and_small_jobs_without_graph_match_alone(ctx, vrt, acc_f32):
    """Frames launched without a graph, jobs of half a megapixel beside small
    ones and one with the denoiser off, both history formats: every job's
    a-trous tiles and outputs equal the session alone."""
    specs = [(2, 128, 3, 1024, 512, 3), (1, 64, 1, 200, 120, 3), (2, 128, 4, 1100, 480, 1),
             (3, 64, 9, 96, 54, 3)]
    scenes, alone, inbatch, spawns = [], [], [], []
    for kind, n, seed, W, H, flags in specs:
        vox, spawn = vrt.generate_scene(kind, n, seed)
        sc = vrt.Scene(ctx, vox, n)
        scenes.append(sc)
        spawns.append(spawn)
        alone.append(vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, accum_f32=acc_f32))
        inbatch.append(vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, accum_f32=acc_f32, path_kernel="batch_only"))
    batch = vrt.Batch(ctx, inbatch)
    batch.set_graph(False)
    for f in range(3):
        us = []
        for i, (kind, n, seed, W, H, flags) in enumerate(specs):
            pose, prev = _poses(vrt, spawns[i], f)
            us.append(vrt.make_uniforms(pose, prev, vrt.Lighting(), 40 + f, 2, flags, W, H))
        batch.frame(us)
        for i in range(len(specs)):
            alone[i].frame(us[i])
            _check_same(_outputs(alone[i]), _outputs(inbatch[i]), f"frame {f} job {i}")
    batch.close()
    for s in alone + inbatch:
        s.close()
    for sc in scenes:
        sc.close()


def test_batch_only_session_refuses_single_frames(ctx, vrt):
    vox, spawn = vrt.generate_scene(1, 64, 1)
    sc = vrt.Scene(ctx, vox, 64)
    s = vrt.Session(ctx, sc, 64, 36, path_kernel="batch_only")
    with pytest.raises(vrt.VrtError) as e:
        s.frame(vrt.make_uniforms(spawn, None, vrt.Lighting(), 0, 2, 3, 64, 36))
    assert e.value.code == 7
    s.close(); sc.close()


def test_batch_autotune(ctx, vrt):
    vox, spawn = vrt.generate_scene(2, 128, 3)
    sc = vrt.Scene(ctx, vox, 128)
    ss = [vrt.Session(ctx, sc, 160 + 32 * i, 90, firefly_clamp=10.0, path_kernel="batch_only") for i in range(3)]
    b = vrt.Batch(ctx, ss)
    us = [vrt.make_uniforms(spawn, None, vrt.Lighting(), 0, 2, 3, 160 + 32 * i, 90) for i in range(3)]
    tune, ms = b.autotune(us, frames=1)
    assert ms > 0 and tune[0] in (4, 8, 12, 16, 24)
    b.frame(us)
    b.close()
    for s in ss:
        s.close()
    sc.close()
