"""HDR reference pipeline: FP64 accumulation of the capture's HDR radiance on
the device (bit-identical to the CPU oracle's FP64 accumulation over the same
frames), device-side squared errors, and the .rgbf32 reference files."""
import numpy as np
import pytest


def test_rgbf32_round_trip(tmp_path):
    from voxelrt_b200.quality import read_rgbf32, write_rgbf32
    img = np.random.default_rng(1).random((5, 7, 3)).astype(np.float32)
    write_rgbf32(tmp_path / "ref", img, {"frames": 4096})
    np.testing.assert_array_equal(read_rgbf32(tmp_path / "ref"), img)
    import json
    assert json.loads((tmp_path / "ref.json").read_text())["frames"] == 4096


@pytest.mark.gpu
@pytest.mark.parametrize("bounces,spp", [(2, 5), (6, 8)])
def test_hdr_accumulation_bit_exact_vs_oracle(vrt, orc, bounces, spp):
    W, H, n = 64, 36, 64
    vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_SMALL, n, 1)
    ctx = vrt.Context(0)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, keep_radiance_f32=True)
    u = vrt.make_uniforms(spawn, None, vrt.Lighting(), 0, bounces, 0, W, H)
    s.hdr_accum_reset()
    s.hdr_accumulate(u, 1000, spp)
    sums, count = s.hdr_accum_sums()
    assert count == spp
    b, m = orc.build_bricks(vox, n)
    acc = orc.accumulate_f64(vox, b, m, n, vrt.uniforms_bytes(u), 10.0, W, H, 1000, spp)
    np.testing.assert_array_equal(sums, acc)


@pytest.mark.gpu
def test_hdr_errors_match_numpy(vrt):
    from voxelrt_b200.quality import hdr_image, mse
    W, H, n = 96, 54, 64
    vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_SMALL, n, 1)
    ctx = vrt.Context(0)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, keep_radiance_f32=True)
    ref = np.random.default_rng(3).random((H, W, 3)).astype(np.float32)
    s.set_hdr_reference(ref)
    s.hdr_accum_reset()
    frames = []
    for f in range(3):
        s.pathtrace(vrt.make_uniforms(spawn, None, vrt.Lighting(), f, 2, 0, W, H))
        s.end_frame()
        s.hdr_accum_add()
        img = hdr_image(s)
        frames.append(img)
        assert s.hdr_frame_mse() == pytest.approx(mse(img, ref), rel=1e-12)
    assert s.hdr_accum_mse() == pytest.approx(mse(np.mean(frames, axis=0), ref), rel=1e-12)
