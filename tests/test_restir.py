"""GPU parity of the ReSTIR `gi` preset (RF_RESTIR | RF_TEMPORAL | RF_SPATIAL,
main.js:44): the initial-candidate pass (pathtrace.wgsl:332-457), temporal
reuse (reuse_temporal.wgsl), spatial reuse + shading (reuse_spatial.wgsl),
then the unchanged temporal / a-trous / present passes, each called through
the C ABI and compared with the CPU oracle fed the same seeded inputs.

Reservoirs are integer/bit records (positions, W and confidence included)
and must match word for word; radiance is asserted within the 1e-4 relative
per-sample tolerance and, since both sides evaluate the same IEEE
expressions, byte-identical as well.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(vrt):
    c = vrt.Context(0)
    yield c
    c.close()


def rel_err(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-6)


def _first_diff(a, b):
    bad = np.argwhere(np.any(a.reshape(a.shape[0], a.shape[1], -1) != b.reshape(b.shape[0], b.shape[1], -1),
                             axis=2))
    return bad[:4].tolist()


def _eq(a, b, what):
    assert a.shape == b.shape, what
    assert np.array_equal(a, b), f"{what}: first differing pixels (y, x) {_first_diff(a, b)}"


def _run_restir(ctx, vrt, orc, kind, n, seed, W, H, frames, *, flags=3, bounces=2, fclamp=10.0, preset="gi",
                move=True, taps=3, ccap=20.0, radius=30.0, pose=None, restir_flags=None, check_stages=True,
                kernel="wavefront", extra_flags=0, sigma=16.0, tweak=None):
    """Renders `frames` frames pass by pass on the device and with the oracle;
    asserts every stage of every frame.  Returns the device stats of the
    last frame and the oracle's last frame."""
    vox, spawn = vrt.generate_scene(kind, n, seed)
    spawn = pose or spawn
    b, m = orc.build_bricks(vox, n)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=fclamp, keep_radiance_f32=True, path_kernel=kernel)
    s.set_timing(True)
    if sigma != 16.0:
        s.set_pairing_sigma(sigma)
    light = vrt.Lighting()
    acc_prev = np.zeros((H, W, 4), np.uint16)
    gprev = np.zeros((H, W, 4), np.float32)
    res_b = np.zeros((H, W, 8), np.uint32)
    dup = np.zeros((H, W), np.float32)
    lights, nlights = None, 0
    rf0 = (vrt.api.preset_flags(preset) if restir_flags is None else restir_flags) | extra_flags
    if rf0 & 128:
        sc.build_lights()
        words, alias, grid = sc.lights()
        lights = {"words": words, "alias": alias, "grid": grid}
        nlights = len(words)
    prev = None
    st = ref = None
    tot = {"rays": 0, "outer": 0, "inner": 0, "vreads": 0}
    for f in range(frames):
        p = vrt.camera_spline(spawn, f) if move else spawn
        u = vrt.make_uniforms(p, prev, light, f, bounces, flags, W, H, preset=preset, taps=taps, ccap=ccap,
                              radius=radius, light_count=nlights)
        u.params2[0] = rf0
        if tweak:
            tweak(u)
        rf = int(u.params2[0])
        pairing = None
        if rf & 8:
            wide = max(0.8, float(np.float32(u.params5[0]))) if rf & 8192 else max(0.8, sigma)
            pairing = orc.pairing_buffer([wide, max(0.8, sigma), max(0.8, sigma)])
        ref = orc.frame(vox, b, m, n, vrt.uniforms_bytes(u), fclamp, W, H, acc_prev, gprev, False, res_b, dup,
                        lights, pairing)
        s.pathtrace(u)
        if check_stages:
            _eq(s.reservoirs(0), ref["resA0"], f"frame {f} reservoirs A (initial)")
            _eq(s.direct(), ref["direct"], f"frame {f} direct")
        if rf & 2:
            s.reuse_temporal(u)
        if check_stages:
            _eq(s.reservoirs(0), ref["resA"], f"frame {f} reservoirs A (temporal reuse)")
        s.reuse_spatial(u)
        s.dupmap(u)
        if rf & 16:
            _eq(s.dupmap_image().view(np.uint32), ref["dup"].view(np.uint32), f"frame {f} dupmap")
        s.temporal(u)
        if flags & 2:
            for it in range(3):
                s.atrous(u, it)
        s.present(u)
        s.end_frame()
        _eq(s.reservoirs(1), ref["resB"], f"frame {f} reservoirs B")
        rad32 = s.radiance_f32()
        assert rel_err(rad32, ref["rad32"]).max() <= 1e-4, f"frame {f} radiance"
        _eq(rad32.view(np.uint32), ref["rad32"].view(np.uint32), f"frame {f} radiance f32")
        _eq(s.radiance(), ref["rad16"], f"frame {f} radiance f16")
        _eq(s.albedo(), ref["alb8"], f"frame {f} albedo")
        _eq(s.gbuffer().view(np.uint32), ref["gbuf"].view(np.uint32), f"frame {f} gbuffer")
        _eq(s.accum(), ref["accum"], f"frame {f} accum")
        _eq(s.ldr(), ref["ldr"], f"frame {f} ldr")
        # counters accumulate over passes driven one by one (vrt_frame clears them)
        for k in tot:
            tot[k] += ref["stats"][k]
        st = s.stats()
        assert st.rays == tot["rays"], f"frame {f} rays"
        assert st.dda_outer == tot["outer"] and st.dda_inner == tot["inner"] and st.voxel_reads == tot["vreads"]
        assert st.pixels == W * H * (f + 1)
        acc_prev, gprev, res_b, dup, prev = ref["accum"], ref["gbuf"], ref["resB"], ref["dup"], p
    s.close(); sc.close()
    return st, ref


def _kinds(res):
    return (res[..., 5] >> 16) & 3


def _conf(res):
    return (res[..., 5] >> 18) & 0xFF


@pytest.mark.parametrize("kernel", ["wavefront", "megakernel"])
def test_restir_gi_moving_camera(ctx, vrt, orc, kernel):
    _, ref = _run_restir(ctx, vrt, orc, 1, 64, 1, 160, 90, 5, kernel=kernel)
    # the chain did real work: point and direction samples, reuse confidence > 1
    k = _kinds(ref["resB"])
    assert (k == 1).any() and (k == 2).any()
    assert _conf(ref["resB"]).max() > 1


def test_restir_gi_static_world_256(ctx, vrt, orc):
    """Static camera on the 256^3 world: confidence climbs to the cap."""
    _, ref = _run_restir(ctx, vrt, orc, 2, 256, 2, 320, 180, 6, move=False)
    c = _conf(ref["resA"])
    assert c.max() <= 255 and c.max() > 20


@pytest.mark.parametrize("restir_flags", [1, 1 | 2, 1 | 4])
def test_restir_flag_subsets(ctx, vrt, orc, restir_flags):
    _run_restir(ctx, vrt, orc, 1, 64, 1, 128, 72, 3, restir_flags=restir_flags)


@pytest.mark.parametrize("kernel", ["wavefront", "megakernel"])
@pytest.mark.parametrize("bounces", [0, 1, 4, 6])
def test_restir_bounce_counts(ctx, vrt, orc, bounces, kernel):
    _run_restir(ctx, vrt, orc, 1, 64, 1, 128, 72, 3, bounces=bounces, kernel=kernel)


@pytest.mark.parametrize("taps,radius,ccap", [(0, 30.0, 20.0), (1, 2.0, 1.0), (3, 120.0, 255.0), (7, 5.5, 0.0)])
def test_restir_tuning(ctx, vrt, orc, taps, radius, ccap):
    _run_restir(ctx, vrt, orc, 3, 128, 4, 128, 72, 3, taps=taps, radius=radius, ccap=ccap)


def test_restir_firefly_clamp_off_no_denoise(ctx, vrt, orc):
    _run_restir(ctx, vrt, orc, 1, 64, 1, 96, 54, 3, fclamp=0.0, flags=1)


@pytest.mark.parametrize("W,H", [(37, 23), (1, 1), (17, 300)])
def test_restir_odd_sizes(ctx, vrt, orc, W, H):
    _run_restir(ctx, vrt, orc, 0, 128, 1337, W, H, 3,
                pose=vrt.CameraPose((4.0, 3.0, 1.0), 0.3, -0.1, math.radians(70)))


@pytest.mark.parametrize("kernel", ["wavefront", "megakernel"])
def test_restir_full_size(ctx, vrt, orc, kernel):
    """1920x1080 on the 256^3 world, two frames, every stage against the oracle."""
    _run_restir(ctx, vrt, orc, 2, 256, 2, 1920, 1080, 2, kernel=kernel)


@pytest.mark.parametrize("preset", ["lin", "ours", "ours_motion"])
def test_restir_reference_presets(ctx, vrt, orc, preset):
    """The reference's presets (main.js:40-62) on a moving camera."""
    _, ref = _run_restir(ctx, vrt, orc, 0, 128, 1337, 160, 90, 4, preset=preset)
    assert (_kinds(ref["resB"]) == 1).any()


@pytest.mark.parametrize("extra", [8, 8 | 8192, 16, 64, 64 | 1024, 1024, 128, 128 | 4096, 128 | 65536,
                                   128 | 16384, 256, 512, 32, 2048, 262144, 8 | 16 | 256 | 512 | 2048])
def test_restir_flags(ctx, vrt, orc, extra):
    """Each flag (and a few combinations) on top of `gi`, every stage against
    the oracle: paired (8), mixsigma (8192), dupmap (16), vector (64), fullv
    (1024), unified (128) with lightpower (4096) / lightgrid (65536) /
    adaptcand (16384), plane (256), rescue (512), footprint (32), rclamp
    (2048), histisolate (262144)."""
    _run_restir(ctx, vrt, orc, 1, 64, 1, 128, 72, 4, extra_flags=extra)


def test_restir_ours_bounces_and_sizes(ctx, vrt, orc):
    """`ours` with 6 bounces (the reference's published configuration), an
    odd size and the megakernel, and a second pairing sigma."""
    _run_restir(ctx, vrt, orc, 0, 128, 1337, 97, 61, 3, preset="ours", bounces=6)
    _run_restir(ctx, vrt, orc, 3, 128, 4, 128, 72, 3, preset="ours", kernel="megakernel", sigma=6.0)
    _run_restir(ctx, vrt, orc, 1, 64, 1, 128, 72, 3, preset="gi", extra_flags=8 | 8192,
                tweak=lambda u: u.params5.__setitem__(0, 24.0))


def test_restir_ours_full_size(ctx, vrt, orc):
    """`ours` at 1920x1080 on the 256^3 world, two frames."""
    _run_restir(ctx, vrt, orc, 2, 256, 2, 1920, 1080, 2, preset="ours", bounces=6)


def test_restir_frame_equals_passes(ctx, vrt):
    """vrt_frame runs exactly the pass sequence of main.js:736-749."""
    W, H, n = 128, 72, 64
    vox, spawn = vrt.generate_scene(1, n, 1)
    sc = vrt.Scene(ctx, vox, n)
    a = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0)
    b = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, path_kernel="megakernel")
    prev = None
    for f in range(3):
        p = vrt.camera_spline(spawn, f)
        u = vrt.make_uniforms(p, prev, vrt.Lighting(), f, 2, 3, W, H, preset="gi")
        a.frame(u)
        b.pathtrace(u); b.reuse_temporal(u); b.reuse_spatial(u); b.temporal(u)
        for it in range(3):
            b.atrous(u, it)
        b.present(u); b.end_frame()
        prev = p
    assert np.array_equal(a.ldr(), b.ldr())
    assert np.array_equal(a.reservoirs(1), b.reservoirs(1))
    a.close(); b.close(); sc.close()


def test_restir_reset_and_invalid_calls(ctx, vrt):
    W, H, n = 96, 54, 64
    vox, spawn = vrt.generate_scene(1, n, 1)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H)
    u = vrt.make_uniforms(spawn, None, vrt.Lighting(), 0, 2, 3, W, H, preset="gi")
    with pytest.raises(vrt.VrtError):
        s.reservoirs(0)                       # no ReSTIR frame yet
    with pytest.raises(vrt.VrtError):
        s.reuse_spatial(u)                    # reuse before the initial pass
    plain = vrt.make_uniforms(spawn, None, vrt.Lighting(), 0, 2, 3, W, H)
    s.frame(plain)
    with pytest.raises(vrt.VrtError):
        s.reservoirs(1)                       # a plain frame allocates no reservoirs
    outs = []
    for _ in range(2):
        s.reset()
        for f in range(3):
            s.frame(vrt.make_uniforms(spawn, spawn if f else None, vrt.Lighting(), f, 2, 3, W, H, preset="gi"))
        outs.append((s.ldr().copy(), s.reservoirs(1).copy()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    with pytest.raises(vrt.VrtError):
        s.reservoirs(2)
    bad = vrt.make_uniforms(spawn, None, vrt.Lighting(), 0, 2, 3, W, H, preset="gi")
    for unbuilt in (32768, 131072, 524288):   # confdenoise, mutate, worldgi: not implemented
        bad.params2[0] = 7 | unbuilt
        with pytest.raises(vrt.VrtError):
            s.frame(bad)
    s.close()
    bs = vrt.Session(ctx, sc, W, H, path_kernel="batch_only")
    batch = vrt.Batch(ctx, [bs])
    with pytest.raises(vrt.VrtError):
        batch.frame([u])                      # batches render the plain path
    batch.close(); bs.close(); sc.close()


def test_restir_energy_matches_plain_path(ctx, vrt):
    """The reuse chain keeps the estimator's energy: the mean HDR radiance of
    a static view over 48 frames agrees with the plain path's within 3%."""
    W, H, n, frames = 192, 108, 64, 48
    vox, spawn = vrt.generate_scene(1, n, 1)
    sc = vrt.Scene(ctx, vox, n)
    means = {}
    for preset in ("base", "gi"):
        s = vrt.Session(ctx, sc, W, H, firefly_clamp=0.0, keep_radiance_f32=True)
        s.hdr_accum_reset()
        for f in range(frames):
            s.frame(vrt.make_uniforms(spawn, spawn if f else None, vrt.Lighting(), f, 2, 0, W, H, preset=preset))
            s.hdr_accum_add()
        means[preset] = float(s.hdr_accum()[0].mean())
        s.close()
    sc.close()
    assert abs(means["gi"] / means["base"] - 1.0) < 0.03, means
