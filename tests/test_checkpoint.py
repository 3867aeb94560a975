"""Session checkpoint / resume (vrt_session_checkpoint, vrt_session_restore).

A session checkpointed after some frames and restored into a fresh session
(on a scene object holding other voxels) must render the following frames
exactly as the original session does: history and G-buffer, frame parity,
the edited voxels, the radiance cache's network and Adam state, and the FP64
HDR accumulation all come back.  VoxelBench resumes its reference
accumulations the same way (VoxelBench/pipeline/harness.cpp:241-256).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H, N = 256, 144, 64


@pytest.fixture(scope="module")
def ctx(vrt):
    c = vrt.Context(0)
    yield c
    c.close()


def _u(vrt, spawn, f, flags=3):
    pose = vrt.camera_spline(spawn, f)
    prev = vrt.camera_spline(spawn, f - 1) if f else None
    return vrt.make_uniforms(pose, prev, vrt.Lighting(), f, 2, flags, W, H)


def _frames(vrt, s, spawn, f0, f1):
    out = []
    for f in range(f0, f1):
        s.frame(_u(vrt, spawn, f))
        out.append((s.ldr().copy(), s.accum().copy(), s.gbuffer().copy()))
    return out


def _fresh(vrt, ctx, seed, **kw):
    vox, _ = vrt.generate_scene(vrt.VRT_SCENE_SMALL, N, seed)
    sc = vrt.Scene(ctx, vox, N)
    return sc, vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, **kw)


@pytest.mark.parametrize("acc_f32", [False, True])
def test_restored_session_renders_the_same_frames(ctx, vrt, acc_f32):
    vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_SMALL, N, 1)
    sc = vrt.Scene(ctx, vox, N)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, accum_f32=acc_f32)
    _frames(vrt, s, spawn, 0, 5)
    sc.edit_box(20, 10, 20, 30, 14, 26, 0)           # an edit before the checkpoint
    state = s.checkpoint()
    want = _frames(vrt, s, spawn, 5, 9)
    sc2, s2 = _fresh(vrt, ctx, 7, accum_f32=acc_f32)  # other voxels until restored
    s2.restore(state)
    got = _frames(vrt, s2, spawn, 5, 9)
    for (a, b, c), (x, y, z) in zip(got, want):
        assert np.array_equal(a, x) and np.array_equal(b, y) and np.array_equal(c.view(np.uint32), z.view(np.uint32))
    assert np.array_equal(sc2.read()[0], sc.read()[0])
    for o in (s, s2, sc, sc2):
        o.close()


def test_restored_cache_session_continues_training(ctx, vrt):
    """The network comes back exactly; the frames after it agree within the
    denoised-output tolerance.  They are not bitwise reproducible: training
    samples are appended by many blocks in whatever order they finish, and the
    order of a step's gradient sums follows it (in the original session too)."""
    vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_SMALL, N, 1)
    sc = vrt.Scene(ctx, vox, N)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0)
    s.set_cache(seed=5)
    _frames(vrt, s, spawn, 0, 6)
    state = s.checkpoint()
    p0 = s.cache_params()
    want = _frames(vrt, s, spawn, 6, 9)
    sc2, s2 = _fresh(vrt, ctx, 3)
    s2.restore(state)                                 # enables the cache with the saved network
    assert np.array_equal(s2.cache_params(), p0)
    got = _frames(vrt, s2, spawn, 6, 9)
    for (a, b, _), (x, y, _) in zip(got, want):
        g = b.view(np.float16).astype(np.float64)
        w = y.view(np.float16).astype(np.float64)
        assert (np.abs(g - w) / np.maximum(np.abs(w), 1e-3)).max() <= 2e-3
        assert np.abs(a.astype(np.int32) - x.astype(np.int32)).max() <= 1
    for o in (s, s2, sc, sc2):
        o.close()


def test_hdr_accumulation_resumes(ctx, vrt):
    vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_SMALL, N, 1)
    sc = vrt.Scene(ctx, vox, N)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, keep_radiance_f32=True)
    u = _u(vrt, spawn, 0, 0)
    s.hdr_accum_reset()
    s.hdr_accumulate(u, 100, 8)
    state = s.checkpoint()
    s.hdr_accumulate(u, 108, 8)
    want, n = s.hdr_accum_sums()
    sc2, s2 = _fresh(vrt, ctx, 3, keep_radiance_f32=True)
    s2.restore(state)
    s2.hdr_accumulate(u, 108, 8)
    got, n2 = s2.hdr_accum_sums()
    assert n == n2 == 16 and np.array_equal(got, want)
    for o in (s, s2, sc, sc2):
        o.close()


def test_restore_rejects_foreign_checkpoints(ctx, vrt):
    vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_SMALL, N, 1)
    sc = vrt.Scene(ctx, vox, N)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0)
    s.frame(_u(vrt, spawn, 0))
    state = s.checkpoint()
    other = vrt.Session(ctx, sc, W // 2, H, firefly_clamp=10.0)
    with pytest.raises(vrt.VrtError) as e:
        other.restore(state)                          # another render size
    assert e.value.code == 1
    bad = bytearray(state)
    bad[0:8] = b"NOTACKPT"
    with pytest.raises(vrt.VrtError) as e:
        s.restore(bytes(bad))
    assert e.value.code == 1
    with pytest.raises(vrt.VrtError) as e:
        s.restore(state[:-4])                          # truncated
    assert e.value.code == 1
    for o in (s, other, sc):
        o.close()
