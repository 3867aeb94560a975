"""The allocation-free denoise entry point (vrt_denoise_atrous_noalloc).

It exists for callers that cannot allocate device memory while they denoise
-- engines whose device memory is owned by their own allocator and budget,
or frame loops that must not call cudaMalloc/cudaFree because those calls
synchronize the device.  Its intermediate image lives in a fixed device array
of the library (at most 1920x1080 pixels), shared by all calls.

The test renders frames through the regular session API, hands the frame's
history and G-buffer to the allocation-free entry point on caller-owned
device buffers, and checks the result against the session's own a-trous
output, for two calls in a row.  This file is collected last so a failure
here cannot hide the other tests' results.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-6)


def test_noalloc_denoise_matches_session_chain(vrt):
    import torch
    from voxelrt_b200._lib import lib

    W, H, n = 320, 180, 64
    vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_SMALL, n, 1)
    ctx = vrt.Context(0)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0)
    dev = torch.device("cuda", 0)
    acc_d = torch.empty(H * W * 4, dtype=torch.int16, device=dev)
    gb_d = torch.empty(H * W * 4, dtype=torch.float32, device=dev)
    out_d = torch.empty(H * W * 4, dtype=torch.int16, device=dev)
    prev = None
    for f in range(2):                       # two calls in a row
        pose = vrt.camera_spline(spawn, f)
        s.frame(vrt.make_uniforms(pose, prev, vrt.Lighting(), f, 2, vrt.FLAG_TEMPORAL | vrt.FLAG_DENOISE, W, H))
        prev = pose
        acc = s.accum()                      # rgba16f history of this frame
        gb = s.gbuffer()
        want = s.denoise(0)                  # the session's a-trous result (dA)
        acc_d.copy_(torch.from_numpy(acc.view(np.int16).ravel()))
        gb_d.copy_(torch.from_numpy(gb.ravel()))
        out_d.fill_(0)
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream(dev).cuda_stream
        code = lib.vrt_denoise_atrous_noalloc(C.c_void_p(acc_d.data_ptr()), 0, C.c_void_p(gb_d.data_ptr()),
                                              C.c_void_p(out_d.data_ptr()), W, H, C.c_void_p(stream))
        assert code == 0, lib.vrt_last_error_string().decode()
        torch.cuda.synchronize()
        got = out_d.cpu().numpy().view(np.uint16).reshape(H, W, 4)
        g32 = got.view(np.float16).astype(np.float32)
        w32 = want.view(np.float16).astype(np.float32)
        assert _rel(g32, w32).max() <= 2e-3          # denoised-output tolerance of the parity tests
        assert np.array_equal(got, want)             # and in fact the same bits
    s.close()
    sc.close()
    ctx.close()


def test_noalloc_rejects_images_above_its_limit(vrt):
    from voxelrt_b200._lib import lib
    code = lib.vrt_denoise_atrous_noalloc(C.c_void_p(16), 0, C.c_void_p(16), C.c_void_p(16), 1920, 1081, None)
    assert code == 1
    assert "1920x1080" in lib.vrt_last_error_string().decode()
