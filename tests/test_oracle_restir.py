"""CPU checks of the oracle's ReSTIR `gi` restatement (reservoir records,
confidence bookkeeping, pass-through radiance) on small seeded cases.  The
GPU parity tests hold the kernels to these same records word for word."""
import numpy as np
import pytest


def _scene(vrt, orc, kind=1, n=64, seed=1):
    vox, spawn = vrt.generate_scene(kind, n, seed)
    b, m = orc.build_bricks(vox, n)
    return vox, b, m, n, spawn


def _chain(vrt, orc, W, H, frames, move=False, preset="gi", **kw):
    vox, b, m, n, spawn = _scene(vrt, orc)
    acc = np.zeros((H, W, 4), np.uint16)
    gprev = np.zeros((H, W, 4), np.float32)
    res_b = np.zeros((H, W, 8), np.uint32)
    prev = None
    out = []
    for f in range(frames):
        p = vrt.camera_spline(spawn, f) if move else spawn
        u = vrt.make_uniforms(p, prev, vrt.Lighting(), f, 2, 3, W, H, preset=preset, **kw)
        r = orc.frame(vox, b, m, n, vrt.uniforms_bytes(u), 10.0, W, H, acc, gprev, False, res_b)
        out.append((u, r))
        acc, gprev, res_b, prev = r["accum"], r["gbuf"], r.get("resB", res_b), p
    return out


def _kind(res):
    return (res[..., 5] >> 16) & 3


def _conf(res):
    return (res[..., 5] >> 18) & 0xFF


def _f16(bits):
    return bits.view(np.float16).astype(np.float32)


def test_initial_reservoirs_records(vrt, orc):
    W, H = 64, 36
    (u, r), = _chain(vrt, orc, W, H, 1)
    a0 = r["resA0"]
    sky = r["gbuf"][..., 3] <= 0
    assert sky.any() and (~sky).any()
    # sky pixels: empty record, direct = radiance = sky colour
    assert not a0[sky].any()
    assert np.array_equal(r["direct"][sky], r["rad16"][sky])
    # hit pixels: confidence 1, a known kind, seed = pcgHash(pixIdx + frame*(W*H+1))
    assert (_conf(a0[~sky]) == 1).all()
    assert np.isin(_kind(a0[~sky]), [0, 1, 2]).all()
    idx = np.arange(W * H).reshape(H, W)
    for y, x in [(int(i // W), int(i % W)) for i in np.flatnonzero(~sky)[:50]]:
        assert a0[y, x, 7] == orc.pcg_hash(int(idx[y, x]))
    w = a0[..., 3].view(np.float32)
    assert np.isfinite(w).all() and (w >= 0).all()
    # a direction sample stores a unit vector, a null one W = 0
    d = _kind(a0) == 2
    v = a0[d][:, :3].view(np.float32)
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-5)
    assert (w[_kind(a0) == 0] == 0).all()


def test_confidence_bookkeeping_static_view(vrt, orc):
    W, H, cap = 48, 27, 20.0
    chain = _chain(vrt, orc, W, H, 5, ccap=cap)
    for f, (u, r) in enumerate(chain):
        hit = r["gbuf"][..., 3] > 0
        ca = _conf(r["resA"])[hit]
        # temporal merge: fresh 1 + history capped at ccap
        assert ca.max() <= 1 + cap
        if f > 0:
            assert ca.max() > 1
        # spatial merge pools up to four domains, clamped to 255
        cb = _conf(r["resB"])[hit]
        assert cb.min() >= 1 and cb.max() <= 255
        # shading adds a non-negative contribution to the pass-through radiance
        rad = _f16(r["rad16"][..., :3])
        dr = _f16(r["direct"][..., :3])
        assert (rad[hit] >= dr[hit]).all()
        assert np.isfinite(rad).all()


def test_deterministic_and_flag_gated(vrt, orc):
    W, H = 40, 24
    a = _chain(vrt, orc, W, H, 2, move=True)
    b = _chain(vrt, orc, W, H, 2, move=True)
    for (_, x), (_, y) in zip(a, b):
        for k in ("resA0", "resA", "resB", "rad16", "accum", "ldr"):
            assert np.array_equal(x[k], y[k]), k
    # without RF_TEMPORAL the working set stays the initial candidates
    vox, bb, m, n, spawn = _scene(vrt, orc)
    u = vrt.make_uniforms(spawn, None, vrt.Lighting(), 3, 2, 3, W, H, preset="gi")
    u.params2[0] = 1 | 4
    r = orc.frame(vox, bb, m, n, vrt.uniforms_bytes(u), 10.0, W, H, np.zeros((H, W, 4), np.uint16),
                  np.zeros((H, W, 4), np.float32), False, a[0][1]["resB"])
    assert np.array_equal(r["resA0"], r["resA"])


def test_plain_preset_unchanged(vrt, orc):
    """params2.x = 0 keeps the plain path (no reservoirs in the result)."""
    (u, r), = _chain(vrt, orc, 32, 18, 1, preset="base")
    assert "resB" not in r and int(u.params2[0]) == 0


@pytest.mark.parametrize("preset,flags", [("base", 0), ("gi", 7)])
def test_preset_flags(vrt, preset, flags):
    assert vrt.api.preset_flags(preset) == flags


@pytest.mark.parametrize("sigmas", [(16.0, 16.0, 16.0), (48.0, 16.0, 16.0), (0.8, 3.0, 100.0)])
def test_pairing_textures(vrt, orc, sigmas):
    """The library's pairing buffer equals the oracle's restatement of
    pairing.js; partners are mutual and spread with about the target sigma."""
    a = vrt.api.make_pairing(sigmas)
    b = orc.pairing_buffer(sigmas)
    assert np.array_equal(a, b)
    off = 0
    for S, sg in zip((254, 230, 210), sigmas):
        tex = a[off:off + S * S].reshape(S, S)
        off += S * S
        dx = (tex & 0xFFFF).astype(np.uint16).view(np.int16).astype(np.int64)
        dy = (tex >> 16).astype(np.uint16).view(np.int16).astype(np.int64)
        ys, xs = np.mgrid[0:S, 0:S]
        px, py = (xs + dx) % S, (ys + dy) % S
        assert np.array_equal((px + dx[py, px]) % S, xs) and np.array_equal((py + dy[py, px]) % S, ys)
        assert not ((dx == 0) & (dy == 0)).any()
        if 2.0 <= sg <= 20.0:
            assert abs(dx.std() / sg - 1.0) < 0.1


def test_ours_chain_invariants(vrt, orc):
    """The `ours` preset through the oracle: unified NEE produces light-face
    samples, the duplication map stays in [0, 1], confidence stays capped."""
    W, H = 64, 36
    vox, spawn = vrt.generate_scene(0, 128, 1337)
    b, m = orc.build_bricks(vox, 128)
    words, weights = orc.light_list(vox, 128)
    lights = {"words": words, "alias": orc.light_alias(weights), "grid": orc.light_grid(128, words, weights)}
    pairing = orc.pairing_buffer([16.0, 16.0, 16.0])
    acc = np.zeros((H, W, 4), np.uint16)
    g = np.zeros((H, W, 4), np.float32)
    rb = np.zeros((H, W, 8), np.uint32)
    dup = np.zeros((H, W), np.float32)
    for f in range(4):
        u = vrt.make_uniforms(spawn, spawn if f else None, vrt.Lighting(), f, 2, 3, W, H, preset="ours",
                              light_count=len(words))
        r = orc.frame(vox, b, m, 128, vrt.uniforms_bytes(u), 10.0, W, H, acc, g, False, rb, dup, lights, pairing)
        acc, g, rb, dup = r["accum"], r["gbuf"], r["resB"], r["dup"]
        assert (dup >= 0).all() and (dup <= 1).all()
        assert np.isfinite(_f16(r["rad16"])).all()
    assert (_kind(rb) == 1).any() and (_kind(rb) == 2).any()
    assert dup.max() > 0
