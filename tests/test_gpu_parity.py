"""GPU parity: every pass of the plain GI path, called through the C ABI,
against the CPU oracle on the same seeded inputs.

Tolerances from the specification are asserted (DDA bit-exact; per-sample
radiance 1e-4 relative; temporal/denoised output 2e-3 relative); because the
kernels and the oracle evaluate the same IEEE expressions, the tests also
assert that the stored buffers are byte-identical.
"""
import math

import numpy as np
import pytest

from helpers import load_voxelbench_states, random_rays

pytestmark = pytest.mark.gpu

HIT_FIELDS = ["t", "n", "mat", "voxel", "face", "steps", "bytes"]


@pytest.fixture(scope="module")
def ctx(vrt):
    c = vrt.Context(0)
    yield c
    c.close()


def assert_hits_equal(a, b, what):
    for f in HIT_FIELDS:
        x, y = a[f], b[f]
        if x.dtype.kind == "f":
            x, y = x.view(np.uint32), y.view(np.uint32)
        bad = np.nonzero(~np.all((x == y).reshape(len(x), -1), axis=1))[0]
        assert bad.size == 0, f"{what}: field {f} differs at {bad[:5]} ({a[bad[:3]]} vs {b[bad[:3]]})"


def rel_err(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-6)


# --------------------------------------------------------------------------
# DDA
# --------------------------------------------------------------------------
def test_trace_rays_golden_states(ctx, vrt, orc):
    for key, n, vox, o, d, hit, vidx, face in load_voxelbench_states():
        b, m = orc.build_bricks(vox, n)
        sc = vrt.Scene(ctx, vox, n)
        tmax = np.full(o.shape[0], 1e9 / 16.0, np.float32)
        got = sc.trace_rays(o, d, tmax)
        ref = orc.trace(vox, b, m, n, o, d, tmax)
        assert_hits_equal(got, ref, key)
        h = hit == 1
        assert np.array_equal(got["t"] >= 0, h)
        sc.close()


@pytest.mark.parametrize("kind,n,seed", [(1, 64, 1), (2, 256, 2), (0, 256, 1337), (3, 128, 4), (3, 512, 6)])
def test_trace_rays_random_bit_exact(ctx, vrt, orc, kind, n, seed):
    vox, _ = vrt.generate_scene(kind, n, seed)
    b, m = orc.build_bricks(vox, n)
    sc = vrt.Scene(ctx, vox, n)
    for inside in (True, False):
        o, d, tmax = random_rays(30000, n, seed * 7 + inside, inside=inside)
        got = sc.trace_rays(o, d, tmax)
        ref = orc.trace(vox, b, m, n, o, d, tmax)
        assert_hits_equal(got, ref, f"kind{kind} n{n} inside={inside}")
    sc.close()


def test_trace_rays_edge_cases(ctx, vrt, orc):
    n = 64
    vox, _ = vrt.generate_scene(1, n, 1)
    b, m = orc.build_bricks(vox, n)
    sc = vrt.Scene(ctx, vox, n)
    assert sc.trace_rays(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0)).size == 0
    ext = n / 16
    o = np.array([[ext / 2, ext / 2, -1.0], [ext / 2, 3.0, ext / 2], [-5, -5, -5], [0, 0, 0], [ext, ext, ext],
                  [ext / 2, ext / 2, ext / 2], [1.0, 1.0, 1.0], [2.0, 5.0, 2.0]], np.float32)
    d = np.array([[0, 0, 1], [0, -1, 0], [1, 1, 1], [1, 0, 0], [-1, -1, -1], [0, 0, -1], [0, 1, 0],
                  [0.0, -1.0, 0.0]], np.float32)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    tmax = np.array([1e4, 1e4, 1e4, 1e4, 1e4, 0.0, 0.01, 1e4], np.float32)
    assert_hits_equal(sc.trace_rays(o, d, tmax), orc.trace(vox, b, m, n, o, d, tmax), "edge rays")
    sc.close()


# --------------------------------------------------------------------------
# Scene build and edits (scene.js:411-433)
# --------------------------------------------------------------------------
@pytest.mark.parametrize("kind,n,seed", [(1, 64, 1), (2, 256, 2), (3, 8, 1)])
def test_brick_build_matches_oracle(ctx, vrt, orc, kind, n, seed):
    vox, _ = vrt.generate_scene(kind, n, seed)
    b, m = orc.build_bricks(vox, n)
    sc = vrt.Scene(ctx, vox, n)
    v2, b2, m2 = sc.read()
    assert np.array_equal(v2, vox) and np.array_equal(b2, b) and np.array_equal(m2, m)
    sc2 = vrt.Scene(ctx, vox, n, bricks=b, masks=m)
    _, b3, m3 = sc2.read()
    assert np.array_equal(b3, b) and np.array_equal(m3, m)
    sc.close(); sc2.close()


def test_edit_box_updates_bricks_and_traces(ctx, vrt, orc):
    n = 128
    vox, _ = vrt.generate_scene(3, n, 21)
    sc = vrt.Scene(ctx, vox, n)
    rng = np.random.default_rng(5)
    cur = vox.reshape(n, n, n).copy()
    for k in range(12):
        lo = rng.integers(-4, n, 3)
        size = rng.integers(1, 17, 3)
        hi = lo + size - 1
        val = 0 if k % 3 == 0 else int(rng.integers(1, 2 ** 24)) | (int(rng.integers(0, 2)) << 28)
        sc.edit_box(*lo, *hi, val)
        lo_c, hi_c = np.clip(lo, 0, n - 1), np.clip(hi, 0, n - 1)
        if (lo <= n - 1).all() and (hi >= 0).all():
            cur[lo_c[2]:hi_c[2] + 1, lo_c[1]:hi_c[1] + 1, lo_c[0]:hi_c[0] + 1] = val
    ref_v = cur.ravel()
    b, m = orc.build_bricks(ref_v, n)
    v2, b2, m2 = sc.read()
    assert np.array_equal(v2, ref_v)
    assert np.array_equal(b2, b) and np.array_equal(m2, m)
    o, d, tmax = random_rays(20000, n, 77)
    assert_hits_equal(sc.trace_rays(o, d, tmax), orc.trace(ref_v, b, m, n, o, d, tmax), "after edits")
    sc.close()


# --------------------------------------------------------------------------
# Path-trace pass (pathtrace.wgsl:248-330)
# --------------------------------------------------------------------------
def _pathtrace_pair(vrt, orc, ctx, kind, n, seed, W, H, bounces, fclamp, frame, pose=None, rows=None,
                    kernel="wavefront"):
    vox, spawn = vrt.generate_scene(kind, n, seed)
    pose = pose or spawn
    b, m = orc.build_bricks(vox, n)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=fclamp, keep_radiance_f32=True, path_kernel=kernel)
    u = vrt.make_uniforms(pose, None, vrt.Lighting(), frame, bounces, 3, W, H, 1.0, 64.0)
    s.set_timing(True)
    s.frame(u)
    st = s.stats()
    got = {"rad16": s.radiance(), "rad32": s.radiance_f32(), "alb8": s.albedo(), "gbuf": s.gbuffer()}
    r0, r1, rs = (0, H, 1) if rows is None else rows
    ref = orc.pathtrace(vox, b, m, n, vrt.uniforms_bytes(u), fclamp, W, H, r0, r1, rs)
    s.close(); sc.close()
    return got, ref, st


def _compare_pathtrace(got, ref, rows=slice(None)):
    # per-sample radiance within 1e-4 relative of the fp32 oracle (spec) ...
    assert rel_err(got["rad32"][rows], ref["rad32"][rows]).max() <= 1e-4
    # ... and in fact bit-identical in every stored buffer
    for k in ("rad16", "alb8"):
        assert np.array_equal(got[k][rows], ref[k][rows]), k
    for k in ("rad32", "gbuf"):
        assert np.array_equal(got[k][rows].view(np.uint32), ref[k][rows].view(np.uint32)), k


@pytest.mark.parametrize("kernel", ["wavefront", "megakernel"])
@pytest.mark.parametrize("bounces", [0, 1, 2, 4, 6])
def test_pathtrace_small_config(ctx, vrt, orc, bounces, kernel):
    got, ref, st = _pathtrace_pair(vrt, orc, ctx, 1, 64, 1, 256, 144, bounces, 10.0, 3, kernel=kernel)
    _compare_pathtrace(got, ref)
    assert st.rays == ref["stats"]["rays"]
    assert st.dda_outer == ref["stats"]["outer"] and st.dda_inner == ref["stats"]["inner"]
    assert st.voxel_reads == ref["stats"]["vreads"]
    assert st.pixels == 256 * 144


@pytest.mark.parametrize("kernel", ["wavefront", "megakernel"])
def test_pathtrace_full_config_rows(ctx, vrt, orc, kernel):
    """1920x1080 on the 256^3 world: every 27th row checked against the oracle."""
    got, ref, st = _pathtrace_pair(vrt, orc, ctx, 2, 256, 2, 1920, 1080, 2, 10.0, 0, rows=(0, 1080, 27),
                                   kernel=kernel)
    _compare_pathtrace(got, ref, rows=slice(0, 1080, 27))
    assert st.pixels == 1920 * 1080


@pytest.mark.parametrize("W,H", [(37, 23), (1, 1), (17, 300)])
def test_pathtrace_odd_sizes(ctx, vrt, orc, W, H):
    got, ref, _ = _pathtrace_pair(vrt, orc, ctx, 0, 128, 1337, W, H, 2, 48.0, 11,
                                  pose=vrt.CameraPose((4.0, 3.0, 1.0), 0.3, -0.1, math.radians(70)))
    _compare_pathtrace(got, ref)


def test_pathtrace_firefly_clamp_off(ctx, vrt, orc):
    got, ref, _ = _pathtrace_pair(vrt, orc, ctx, 1, 64, 1, 128, 72, 3, 0.0, 5)
    _compare_pathtrace(got, ref)


def test_wavefront_invariant_to_launch_shape(ctx, vrt):
    """Queue order and refill policy must not change any bit of the image."""
    W, H, n = 320, 180, 256
    vox, spawn = vrt.generate_scene(2, n, 2)
    sc = vrt.Scene(ctx, vox, n)
    u = vrt.make_uniforms(vrt.camera_spline(spawn, 40), None, vrt.Lighting(), 9, 4, 3, W, H)
    outs = []
    for kernel, tune in [("megakernel", None), ("wavefront", (16, 0, 8, 0)), ("wavefront", (1, 1, 1, 0)),
                         ("wavefront", (32, 2, 32, 1)), ("wavefront", (8, 0, 4, 2)), ("wavefront", (12, 0, 16, 1))]:
        s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, keep_radiance_f32=True, path_kernel=kernel)
        if tune:
            s.set_tuning(*tune)
        s.set_timing(True)
        s.frame(u)
        st = s.stats()
        outs.append((s.radiance_f32().copy(), s.gbuffer().copy(), s.albedo().copy(),
                     (st.rays, st.dda_outer, st.dda_inner, st.voxel_reads, st.pixels)))
        s.close()
    for o in outs[1:]:
        assert np.array_equal(o[0].view(np.uint32), outs[0][0].view(np.uint32))
        assert np.array_equal(o[1].view(np.uint32), outs[0][1].view(np.uint32))
        assert np.array_equal(o[2], outs[0][2])
        assert o[3] == outs[0][3]
    sc.close()


# --------------------------------------------------------------------------
# Whole frames: temporal (temporal.wgsl), a-trous (atrous.wgsl), present
# --------------------------------------------------------------------------
def _run_frames(ctx, vrt, orc, kind, n, seed, W, H, frames, acc_f32, flags=3, step_m=0.05):
    vox, spawn = vrt.generate_scene(kind, n, seed)
    b, m = orc.build_bricks(vox, n)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, accum_f32=acc_f32)
    light = vrt.Lighting()
    acc_prev = np.zeros((H, W, 4), np.float32 if acc_f32 else np.uint16)
    gprev = np.zeros((H, W, 4), np.float32)
    prev = None
    for f in range(frames):
        pose = vrt.camera_spline(spawn, f) if step_m else spawn
        u = vrt.make_uniforms(pose, prev, light, f, 2, flags, W, H, 1.0, 64.0)
        s.frame(u)
        ub = vrt.uniforms_bytes(u)
        ref = orc.frame(vox, b, m, n, ub, 10.0, W, H, acc_prev, gprev, acc_f32)
        acc = s.accum()
        if acc_f32:
            assert rel_err(acc, ref["accum"]).max() <= 2e-3
            assert np.array_equal(acc.view(np.uint32), ref["accum"].view(np.uint32)), f"frame {f} accum"
        else:
            assert np.array_equal(acc, ref["accum"]), f"frame {f} accum"
        if flags & 2:
            assert np.array_equal(s.denoise(1), ref["den"][1]), f"frame {f} dB"
            assert np.array_equal(s.denoise(0), ref["den"][2]), f"frame {f} dA"
        fin = s.final(bool(flags & 2))
        assert np.array_equal(fin.view(np.uint8), ref["final"].view(np.uint8)), f"frame {f} final"
        assert np.array_equal(s.ldr(), ref["ldr"]), f"frame {f} ldr"
        assert np.array_equal(s.hdr().view(np.uint32), ref["hdr"].view(np.uint32)), f"frame {f} hdr"
        acc_prev, gprev, prev = ref["accum"], ref["gbuf"], pose
    s.close(); sc.close()


def test_frames_small_moving_camera(ctx, vrt, orc):
    _run_frames(ctx, vrt, orc, 1, 64, 1, 256, 144, 6, False)


def test_frames_accum_f32(ctx, vrt, orc):
    _run_frames(ctx, vrt, orc, 1, 64, 1, 160, 90, 4, True)


def test_frames_no_denoise_and_no_temporal(ctx, vrt, orc):
    _run_frames(ctx, vrt, orc, 1, 64, 1, 96, 54, 3, False, flags=1)
    _run_frames(ctx, vrt, orc, 1, 64, 1, 96, 54, 3, False, flags=0)


def test_frames_full_world_static(ctx, vrt, orc):
    _run_frames(ctx, vrt, orc, 2, 256, 2, 320, 180, 3, False, step_m=0.0)


def test_full_size_temporal_atrous_from_device_inputs(ctx, vrt, orc):
    """1080p: the image passes of frame 2 checked against the oracle fed with
    the device's own frame-1 history and frame-2 path-trace outputs."""
    W, H, n = 1920, 1080, 256
    vox, spawn = vrt.generate_scene(2, n, 2)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0)
    light = vrt.Lighting()
    p0, p1 = vrt.camera_spline(spawn, 0), vrt.camera_spline(spawn, 1)
    s.frame(vrt.make_uniforms(p0, None, light, 0, 2, 3, W, H))
    acc0, g0 = s.accum(), s.gbuffer()
    u1 = vrt.make_uniforms(p1, p0, light, 1, 2, 3, W, H)
    s.frame(u1)
    rad, alb, g1 = s.radiance(), s.albedo(), s.gbuffer()
    ub = vrt.uniforms_bytes(u1)
    acc1 = orc.temporal(ub, W, H, rad, g1, acc0, g0, False)
    assert np.array_equal(s.accum(), acc1)
    da = orc.atrous(W, H, acc1, False, g1, 1)
    db = orc.atrous(W, H, da, False, g1, 2)
    da2 = orc.atrous(W, H, db, False, g1, 4)
    assert np.array_equal(s.denoise(1), db)
    assert np.array_equal(s.denoise(0), da2)
    assert np.array_equal(s.ldr(), orc.present(ub, W, H, da2, False, alb))
    s.close(); sc.close()


def test_present_table_is_exact_over_its_range(ctx):
    """The present pass codes channel values below 8 through the context's
    threshold table; every float of [0, 8) gives the exact arithmetic's code."""
    bad, first = ctx.selftest_present()
    assert bad == 0, f"{bad} values differ, first bit pattern {first:#x}"
    assert first == 0xFFFFFFFF


@pytest.mark.parametrize("exposure", [1.0, 2.5])
def test_present_edge_values_match_oracle(ctx, vrt, orc, exposure):
    """Present on chosen values through the pass entry point: uniform and
    log-spread values, denormals, signed zeros, values at and above the table's
    range, the half maximum, infinities and NaN."""
    W, H = 64, 48
    vox, spawn = vrt.generate_scene(1, 64, 1)
    sc = vrt.Scene(ctx, vox, 64)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, accum_f32=True)
    light = vrt.Lighting()
    for f in range(2):                          # albedo from a real frame; history parity 1 next
        s.pathtrace(vrt.make_uniforms(spawn, None, light, f, 2, 0, W, H))
        s.end_frame()
    rng = np.random.default_rng(7)
    n = W * H * 4
    v = np.concatenate([
        rng.uniform(0.0, 8.0, n // 4),
        10.0 ** rng.uniform(-40.0, 6.0, n // 4),
        rng.uniform(-1.0, 20.0, n // 4),
        np.array([0.0, -0.0, 1e-45, 1.1754942e-38, 7.9999995, 8.0, 8.000001, 65504.0, 3.4e38,
                  np.inf, -np.inf, np.nan, -1e-30, -5.0], np.float32),
    ]).astype(np.float32)
    v = np.resize(v, n).reshape(H, W, 4)
    s.write_history(v, None)                   # history slot 1
    s.end_frame()
    u = vrt.make_uniforms(spawn, None, light, 2, 2, 0, W, H, exposure)
    s.present(u)
    got = s.ldr()
    want = orc.present(vrt.uniforms_bytes(u), W, H, v, True, s.albedo())
    assert np.array_equal(got, want)
    s.close(); sc.close()


# --------------------------------------------------------------------------
# Behaviour
# --------------------------------------------------------------------------
def test_determinism_and_reset(ctx, vrt):
    vox, spawn = vrt.generate_scene(1, 64, 1)
    sc = vrt.Scene(ctx, vox, 64)
    s = vrt.Session(ctx, sc, 128, 72, firefly_clamp=10.0)
    outs = []
    for _ in range(2):
        s.reset()
        for f in range(3):
            s.frame(vrt.make_uniforms(spawn, spawn if f else None, vrt.Lighting(), f, 2, 3, 128, 72))
        outs.append((s.ldr().copy(), s.accum().copy()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    s.close(); sc.close()


def test_invalid_calls_fail_on_host(ctx, vrt):
    vox, spawn = vrt.generate_scene(1, 64, 1)
    sc = vrt.Scene(ctx, vox, 64)
    s = vrt.Session(ctx, sc, 64, 36)
    u = vrt.make_uniforms(spawn, None, vrt.Lighting(), 0, 2, 3, 65, 36)
    with pytest.raises(vrt.VrtError):
        s.frame(u)                            # size mismatch
    u = vrt.make_uniforms(spawn, None, vrt.Lighting(), 0, 2, 3, 64, 36)
    u.params2[0] = 1 | 32768                  # RF_CONFDENOISE: not implemented
    with pytest.raises(vrt.VrtError):
        s.frame(u)
    u.params2[0] = 2                          # RF_TEMPORAL without RF_RESTIR
    with pytest.raises(vrt.VrtError):
        s.frame(u)
    with pytest.raises(vrt.VrtError):
        vrt.Scene(ctx, np.zeros(12 ** 3, np.uint32), 12)
    s.close(); sc.close()


def test_hbm_budget_admission(vrt):
    c = vrt.Context(0, hbm_budget_bytes=8 << 20)
    vox, spawn = vrt.generate_scene(1, 64, 1)
    sc = vrt.Scene(c, vox, 64)                 # ~1.1 MB fits
    with pytest.raises(vrt.VrtError) as e:
        vrt.Session(c, sc, 1920, 1080)         # ~170 MB does not
    assert e.value.code == 5
    used = c.bytes_in_use
    s = vrt.Session(c, sc, 64, 36)
    assert c.bytes_in_use > used
    s.close()
    assert c.bytes_in_use == used
    sc.close()
    assert c.bytes_in_use == 0
    c.close()


def test_autotune_picks_a_candidate_and_keeps_results(ctx, vrt):
    W, H, n = 320, 180, 128
    vox, spawn = vrt.generate_scene(2, n, 3)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, keep_radiance_f32=True)
    u = vrt.make_uniforms(spawn, None, vrt.Lighting(), 4, 2, 3, W, H)
    s.frame(u)
    before = s.radiance_f32().copy()
    tune, ms = s.autotune(u, frames=2)
    assert ms > 0 and tune[0] in (4, 8, 12, 16, 24) and tune[3] in (0, 1, 2) and s.get_tuning() == tune
    s.frame(u)                                  # history was reset: same first frame again
    assert np.array_equal(s.radiance_f32().view(np.uint32), before.view(np.uint32))
    s.close(); sc.close()


def test_atrous_tile_shape_invariant(ctx, vrt):
    """The autotuner's a-trous tile shapes (8/8/8 and 16/16/8 output rows per
    tile) give the same denoised image bit for bit."""
    W, H, n = 320, 180, 64
    vox, spawn = vrt.generate_scene(1, n, 1)
    sc = vrt.Scene(ctx, vox, n)
    outs = []
    for rows in (0, 16):
        s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0)
        s.set_tuning(0, 0, 0, 0, rows)
        assert s.get_tuning()[4] == rows
        prev = None
        for f in range(3):
            pose = vrt.camera_spline(spawn, f)
            s.frame(vrt.make_uniforms(pose, prev, vrt.Lighting(), f, 2, 3, W, H))
            prev = pose
        outs.append((s.denoise(0).copy(), s.denoise(1).copy(), s.ldr().copy()))
        s.close()
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)
    sc.close()


@pytest.mark.parametrize("bounces", [2, 4, 6])
def test_tail_kernel_invariant(ctx, vrt, bounces):
    """Finishing the remaining paths one thread each from wave 2 or 3
    (k_wf_tail) gives the same image and traversal counters as running every
    wave."""
    W, H, n = 320, 180, 128
    vox, spawn = vrt.generate_scene(2, n, 3)
    sc = vrt.Scene(ctx, vox, n)
    u = vrt.make_uniforms(vrt.camera_spline(spawn, 20), None, vrt.Lighting(), 5, bounces, 3, W, H)
    outs = []
    for tail in (0, 2, 3):
        s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, keep_radiance_f32=True)
        s.set_tuning(tail_wave=tail)
        s.frame(u)
        st = s.stats()
        outs.append((s.radiance_f32().copy(), s.gbuffer().copy(), s.albedo().copy(),
                     (st.rays, st.dda_outer, st.dda_inner, st.voxel_reads)))
        s.close()
    for o in outs[1:]:
        assert np.array_equal(o[0].view(np.uint32), outs[0][0].view(np.uint32))
        assert np.array_equal(o[1].view(np.uint32), outs[0][1].view(np.uint32))
        assert np.array_equal(o[2], outs[0][2])
        assert o[3] == outs[0][3]
    sc.close()
