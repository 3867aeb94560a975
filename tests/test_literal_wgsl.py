"""Parity against the literal restatement of the shaders.

The bit-exact parity tests compare the kernels with an oracle that evaluates
the same reformulated expressions they do (one exp per a-trous tap, skipped
zero-weight taps, fused multiply-adds, the project's own sin/cos/exp/pow).
These tests compare against the oracle's literal mode instead -- the WGSL as
written (atrous.wgsl:60-79 with two exps per tap and every tap summed,
dot products unfused, pow(x, 8) and pow(x, 32) as pow, C-library binary32
transcendentals) -- at the specification's tolerances:

  * per-sample radiance within 1e-4 relative wherever both took the same
    discrete path (every trace with the same outcome; a last-bit difference
    in a direction may flip a DDA tie, after which the two are different
    samples), and at most 0.1% of pixels on a different path;
  * temporal and denoised output (rgba16f / rgba32f) within 2e-3 relative,
    each pass fed the same inputs;
  * the LDR present output within one 8-bit step.

The CPU tests check the oracle's own reformulations against its literal
mode; the GPU tests check the kernels against the literal mode directly.
"""
import numpy as np
import pytest

RAD_TOL = 1e-4
IMG_TOL = 2e-3
MAX_PATH_DIFF = 1e-3


def _f16(a):
    return np.ascontiguousarray(a).view(np.float16).astype(np.float64)


def _rel(a, b, floor=1e-30):
    """|a - b| / max(|b|, floor); 0 where both are 0.  Stored images use a
    floor of 1e-6, as the bit-exact parity tests do."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    r = np.abs(a - b) / np.maximum(np.abs(b), floor)
    r[(a == 0) & (b == 0)] = 0.0
    return r


def _img(a, f32):
    return np.asarray(a, np.float64) if f32 else _f16(a)


def check_radiance(rad32, sig, lit, rows=slice(None)):
    """rad32 / sig: the tested side's fp32 radiance and path signatures;
    lit: the literal oracle's path_signatures() output."""
    same = sig[rows] == lit["sig"][rows]
    frac = 1.0 - same.mean()
    assert frac <= MAX_PATH_DIFF, f"{frac:.2%} of pixels took another path"
    r = _rel(rad32[rows][..., :3], lit["rad32"][rows][..., :3])
    worst = r[same].max() if same.any() else 0.0
    assert worst <= RAD_TOL, worst
    return frac, worst


def literal_passes(orc, ub, W, H, rad16, gbuf, acc_prev, gprev, acc_f32, alb8, accum, den):
    """Temporal, the three a-trous iterations and present of the literal mode,
    each pass fed the tested side's own inputs."""
    with orc.literal_wgsl():
        acc = orc.temporal(ub, W, H, rad16, gbuf, acc_prev, gprev, acc_f32)
        d0 = orc.atrous(W, H, accum, acc_f32, gbuf, 1)
        d1 = orc.atrous(W, H, den[0], False, gbuf, 2)
        d2 = orc.atrous(W, H, den[1], False, gbuf, 4)
        ldr = orc.present(ub, W, H, den[2], False, alb8)
    return acc, (d0, d1, d2), ldr


def check_passes(accum, den, ldr, lit, acc_f32):
    acc_l, den_l, ldr_l = lit
    assert _rel(_img(accum, acc_f32), _img(acc_l, acc_f32), 1e-6).max() <= IMG_TOL
    for k in range(3):
        assert _rel(_f16(den[k]), _f16(den_l[k]), 1e-6).max() <= IMG_TOL, f"a-trous iteration {k}"
    assert np.abs(ldr.astype(np.int32) - ldr_l.astype(np.int32)).max() <= 1


def _frames(vrt, orc, kind, n, seed, W, H, frames, acc_f32, run_side):
    vox, spawn = vrt.generate_scene(kind, n, seed)
    b, m = orc.build_bricks(vox, n)
    acc_prev = np.zeros((H, W, 4), np.float32 if acc_f32 else np.uint16)
    gprev = np.zeros((H, W, 4), np.float32)
    prev = None
    diffs = []
    for f in range(frames):
        pose = vrt.camera_spline(spawn, f)
        u = vrt.make_uniforms(pose, prev, vrt.Lighting(), f, 2, vrt.FLAG_TEMPORAL | vrt.FLAG_DENOISE, W, H, 1.0, 64.0)
        ub = vrt.uniforms_bytes(u)
        side = run_side(vox, b, m, n, u, ub, acc_prev, gprev)
        with orc.literal_wgsl():
            lit = orc.path_signatures(vox, b, m, n, ub, 10.0, W, H)
        sig = orc.path_signatures(vox, b, m, n, ub, 10.0, W, H)["sig"]   # the tested side's path (bit-exact)
        diffs.append(check_radiance(side["rad32"], sig, lit))
        check_passes(side["accum"], side["den"], side["ldr"],
                     literal_passes(orc, ub, W, H, side["rad16"], side["gbuf"], acc_prev, gprev, acc_f32,
                                    side["alb8"], side["accum"], side["den"]), acc_f32)
        acc_prev, gprev, prev = side["accum"], side["gbuf"], pose
    return diffs


@pytest.mark.parametrize("kind,n,seed,W,H,acc_f32", [(1, 64, 1, 256, 144, False), (2, 256, 2, 480, 270, True)])
def test_oracle_reformulations_within_spec_of_literal_wgsl(vrt, orc, kind, n, seed, W, H, acc_f32):
    def oracle_side(vox, b, m, n_, u, ub, acc_prev, gprev):
        r = orc.frame(vox, b, m, n_, ub, 10.0, W, H, acc_prev, gprev, acc_f32)
        r["den"] = list(r["den"])
        return r
    _frames(vrt, orc, kind, n, seed, W, H, 3, acc_f32, oracle_side)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,n,seed,W,H,acc_f32", [(1, 64, 1, 256, 144, False), (2, 256, 2, 480, 270, True)])
def test_kernels_within_spec_of_literal_wgsl(vrt, orc, kind, n, seed, W, H, acc_f32):
    ctx = vrt.Context(0)
    vox0, _ = vrt.generate_scene(kind, n, seed)
    sc = vrt.Scene(ctx, vox0, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, accum_f32=acc_f32, keep_radiance_f32=True)

    # the session keeps only dA and dB (the chain accum -> dA -> dB -> dA):
    # the per-pass entry points let dA be read after the first iteration too.
    # History and G-buffer are read after vrt_end_frame, which makes this
    # frame's parity the one the read calls return.
    def kernel_side_passes(vox, b, m, n_, u, ub, acc_prev, gprev):
        s.pathtrace(u)
        s.temporal(u)
        s.atrous(u, 0)
        d0 = s.denoise(0)
        s.atrous(u, 1)
        s.atrous(u, 2)
        s.present(u)
        s.end_frame()
        return {"rad32": s.radiance_f32(), "rad16": s.radiance(), "gbuf": s.gbuffer(), "alb8": s.albedo(),
                "accum": s.accum(), "den": [d0, s.denoise(1), s.denoise(0)], "ldr": s.ldr()}

    diffs = _frames(vrt, orc, kind, n, seed, W, H, 3, acc_f32, kernel_side_passes)
    print(f"path differences / worst same-path radiance error per frame: {diffs}")
    s.close()
    sc.close()
    ctx.close()


@pytest.mark.gpu
def test_kernels_full_config_rows_within_spec_of_literal_wgsl(vrt, orc):
    """1920x1080 on the 256^3 world, every 27th row: radiance against the
    literal mode."""
    W, H, n = 1920, 1080, 256
    vox, spawn = vrt.generate_scene(2, n, 2)
    b, m = orc.build_bricks(vox, n)
    ctx = vrt.Context(0)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, keep_radiance_f32=True)
    u = vrt.make_uniforms(vrt.camera_spline(spawn, 30), None, vrt.Lighting(), 7, 2, 3, W, H)
    ub = vrt.uniforms_bytes(u)
    s.frame(u)
    rows = slice(0, H, 27)
    with orc.literal_wgsl():
        lit = orc.path_signatures(vox, b, m, n, ub, 10.0, W, H, 0, H, 27)
    sig = orc.path_signatures(vox, b, m, n, ub, 10.0, W, H, 0, H, 27)["sig"]
    print(check_radiance(s.radiance_f32(), sig, lit, rows))
    s.close()
    sc.close()
    ctx.close()
