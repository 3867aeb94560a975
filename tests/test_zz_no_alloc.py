"""The allocation-free denoise entry point (vrt_denoise_atrous_noalloc).

It exists for callers that cannot allocate device memory while they denoise
-- engines whose device memory is owned by their own allocator and budget,
or frame loops that must not call cudaMalloc/cudaFree because those calls
synchronize the device.  Its intermediate image lives in a fixed device array
of the library (at most 1920x1080 pixels), shared by all calls.

The tests render frames through the regular session API, hand each frame's
history and G-buffer to the allocation-free entry point on caller-owned
device buffers, and check the result against the session's own a-trous
output and against the CPU oracle's a-trous chain, for two calls in a row:
with an rgba16f and an rgba32f history, and at the size limit itself.  They
also check that the device's free memory does not change across calls.  This
file is collected last so a failure here cannot hide the other tests' results.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-6)


def _oracle_chain(orc, acc, acc_f32, gb, W, H):
    """accum -> dA (step 1) -> dB (step 2) -> dA (step 4) on the CPU."""
    a = orc.atrous(W, H, acc, acc_f32, gb, 1)
    b = orc.atrous(W, H, a, False, gb, 2)
    return orc.atrous(W, H, b, False, gb, 4)


def _run_noalloc(lib, torch, dev, acc, acc_f32, gb, W, H):
    acc_d = torch.from_numpy(np.ascontiguousarray(acc).view(np.uint8).ravel().copy()).to(dev)
    gb_d = torch.from_numpy(np.ascontiguousarray(gb).view(np.uint8).ravel().copy()).to(dev)
    out_d = torch.zeros(H * W * 8, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev).cuda_stream
    free0 = torch.cuda.mem_get_info(dev)[0]
    code = lib.vrt_denoise_atrous_noalloc(C.c_void_p(acc_d.data_ptr()), 1 if acc_f32 else 0,
                                          C.c_void_p(gb_d.data_ptr()), C.c_void_p(out_d.data_ptr()), W, H,
                                          C.c_void_p(stream))
    assert code == 0, lib.vrt_last_error_string().decode()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(dev)[0]
    return out_d.cpu().numpy().view(np.uint16).reshape(H, W, 4), free0, free1


@pytest.mark.parametrize("W,H,acc_f32", [(320, 180, False), (320, 180, True), (1920, 1080, False)])
def test_noalloc_denoise_matches_session_chain_and_oracle(vrt, orc, W, H, acc_f32):
    import torch
    from voxelrt_b200._lib import lib

    n = 64 if W < 1000 else 256
    kind = vrt.VRT_SCENE_SMALL if n == 64 else vrt.VRT_SCENE_FULL
    vox, spawn = vrt.generate_scene(kind, n, 1 if n == 64 else 2)
    ctx = vrt.Context(0)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, accum_f32=acc_f32)
    dev = torch.device("cuda", 0)
    prev = None
    frees = []
    for f in range(2):                       # two calls in a row
        pose = vrt.camera_spline(spawn, f)
        s.frame(vrt.make_uniforms(pose, prev, vrt.Lighting(), f, 2, vrt.FLAG_TEMPORAL | vrt.FLAG_DENOISE, W, H))
        prev = pose
        acc = s.accum()                      # history of this frame (rgba16f or rgba32f)
        gb = s.gbuffer()
        want = s.denoise(0)                  # the session's a-trous result (dA)
        got, free0, free1 = _run_noalloc(lib, torch, dev, acc, acc_f32, gb, W, H)
        frees.append((free0, free1))
        g32 = got.view(np.float16).astype(np.float32)
        w32 = want.view(np.float16).astype(np.float32)
        assert _rel(g32, w32).max() <= 2e-3          # denoised-output tolerance of the parity tests
        assert np.array_equal(got, want)             # and in fact the same bits
        ref = _oracle_chain(orc, acc, acc_f32, gb, W, H)
        assert np.array_equal(got, ref), f"frame {f}: {int((got != ref).sum())} values differ from the oracle"
    # the second call allocates nothing: free device memory is unchanged across it
    # (the first call on a device may load the library's kernels there)
    assert frees[1][0] == frees[1][1], frees
    s.close()
    sc.close()
    ctx.close()


def test_noalloc_rejects_images_above_its_limit(vrt):
    from voxelrt_b200._lib import lib
    code = lib.vrt_denoise_atrous_noalloc(C.c_void_p(16), 0, C.c_void_p(16), C.c_void_p(16), 1920, 1081, None)
    assert code == 1
    assert "1920x1080" in lib.vrt_last_error_string().decode()
