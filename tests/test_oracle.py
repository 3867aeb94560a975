"""CPU tests of the oracle (the checker) against the reference's own traversal
and against independent numpy restatements.  No GPU needed."""
import math

import numpy as np
import pytest

from helpers import load_voxelbench_states, random_rays


# --------------------------------------------------------------------------
# Pin: oracle DDA (voxel.wgsl:73-153 restated) vs the reference's traceNaive
# (VoxelBench core.cpp:23-50) on the reference's own scenes.
# --------------------------------------------------------------------------
@pytest.mark.parametrize("state", list(range(8)))
def test_dda_matches_voxelbench_tracenaive(orc, state):
    key, n, vox, o, d, hit, vidx, face = list(load_voxelbench_states())[state]
    bricks, masks = orc.build_bricks(vox, n)
    tmax = np.full(o.shape[0], 1e9 / 16.0, np.float32)
    r = orc.trace(vox, bricks, masks, n, o, d, tmax)
    ours_hit = r["t"] >= 0
    assert np.array_equal(ours_hit, hit == 1), f"{key}: hit/miss differs"
    h = hit == 1
    # Voxel and face agree except where the ray crosses a voxel edge/corner
    # within float32 rounding (single vs double precision tie): the entry t
    # then agrees to 1e-3 voxel and the voxels are neighbours.  At most 1 such
    # ray per 1000 hits.
    tref = np.load(__import__("helpers").GOLDEN / "voxelbench_rays.npz")[key + "_t"]
    diff = h & (~(r["voxel"] == vidx).all(1) | (r["face"] != face))
    assert diff.sum() <= max(1, h.sum() // 1000), f"{key}: {diff.sum()} voxel/face mismatches"
    assert (np.abs(r["t"][diff] * 16.0 - tref[diff]) < 1e-3).all(), f"{key}: mismatch is not a tie"
    assert (np.abs(r["voxel"][diff] - vidx[diff]).max(initial=0) <= 1), f"{key}: mismatch not adjacent"
    assert (r["mat"][h] != 0).all()


def test_oracle_naive_matches_voxelbench(orc):
    for key, n, vox, o, d, hit, vidx, face in load_voxelbench_states():
        tmax = np.full(o.shape[0], 1e9 / 16.0, np.float32)
        r = orc.trace_naive(vox, n, o, d, tmax)
        h = hit == 1
        assert np.array_equal(r["t"] >= 0, h), key
        assert np.array_equal(r["voxel"][h], vidx[h]), key
        assert np.array_equal(r["face"][h], face[h]), key


# --------------------------------------------------------------------------
# Two-level vs per-voxel traversal on the packed-u32 layout (the equivalence
# test of harness.cpp:205-239, rewritten for 8^3 bricks).
# --------------------------------------------------------------------------
@pytest.mark.parametrize("kind,n,seed", [(1, 64, 1), (0, 128, 1337), (2, 128, 2), (3, 64, 5)])
def test_two_level_equals_naive(orc, vrt, kind, n, seed):
    vox, _ = vrt.generate_scene(kind, n, seed)
    bricks, masks = orc.build_bricks(vox, n)
    o, d, tmax = random_rays(20000, n, seed + 11, inside=True)
    vi = np.floor(o * 16).astype(np.int64).clip(0, n - 1)
    empty = vox[vi[:, 0] + vi[:, 1] * n + vi[:, 2] * n * n] == 0
    o, d, tmax = o[empty], d[empty], tmax[empty]
    a = orc.trace(vox, bricks, masks, n, o, d, tmax)
    b = orc.trace_naive(vox, n, o, d, tmax)
    same_hit = (a["t"] >= 0) == (b["t"] >= 0)
    both = (a["t"] >= 0) & (b["t"] >= 0)
    same_vox = (a["voxel"] == b["voxel"]).all(1)
    bad = (~same_hit) | (both & ~same_vox)
    # float32 vs float64 walks may part only at exact ties / maxT boundaries
    assert bad.sum() <= max(2, len(o) // 2000), f"{bad.sum()} of {len(o)} differ"


def test_brick_build_semantics(orc, vrt):
    vox, _ = vrt.generate_scene(3, 64, 9)
    bricks, masks = orc.build_bricks(vox, 64)
    g = vox.reshape(64, 64, 64)  # [z, y, x]
    bg = 8
    for bi in range(bg ** 3):
        bx, by, bz = bi % bg, (bi // bg) % bg, bi // (bg * bg)
        blk = g[bz * 8:bz * 8 + 8, by * 8:by * 8 + 8, bx * 8:bx * 8 + 8]
        assert bricks[bi] == (1 if (blk != 0).any() else 0)
        bits = np.zeros(512, bool)
        lz, ly, lx = np.nonzero(blk)
        bits[lx + 8 * ly + 64 * lz] = True
        words = np.packbits(bits.reshape(16, 32)[:, ::-1], axis=1, bitorder="big").view(">u4").ravel()
        assert np.array_equal(masks[bi * 16:(bi + 1) * 16], words.astype(np.uint32))


# --------------------------------------------------------------------------
# Project transcendentals and storage conversions
# --------------------------------------------------------------------------
def test_sincos_accuracy(orc):
    x = np.linspace(0, 2 * np.pi, 200001).astype(np.float32)
    s = orc.math_eval(0, x).astype(np.float64)
    c = orc.math_eval(1, x).astype(np.float64)
    assert np.max(np.abs(s - np.sin(x.astype(np.float64)))) < 3e-7
    assert np.max(np.abs(c - np.cos(x.astype(np.float64)))) < 3e-7


def test_exp_log_pow_accuracy(orc):
    x = np.linspace(-80, 0, 100001).astype(np.float32)
    e = orc.math_eval(2, x).astype(np.float64)
    ref = np.exp(x.astype(np.float64))
    assert np.max(np.abs(e - ref) / ref) < 4e-7
    y = np.geomspace(1e-30, 1.0, 100001).astype(np.float32)
    l2 = orc.math_eval(3, y).astype(np.float64)
    ref2 = np.log2(y.astype(np.float64))
    assert np.all(np.abs(l2 - ref2) < 2e-6 + 1e-7 * np.abs(ref2))
    yy = np.linspace(0, 1, 100001).astype(np.float32)
    p = orc.math_eval(4, yy).astype(np.float64)
    assert np.max(np.abs(p - yy.astype(np.float64) ** 0.55)) < 2e-6
    p2 = orc.math_eval(5, yy).astype(np.float64)
    assert np.max(np.abs(p2 - yy.astype(np.float64) ** np.float64(np.float32(1 / 2.2)))) < 2e-6


def test_f16_round_trip_matches_numpy(orc):
    rng = np.random.default_rng(3)
    bits = rng.integers(0, 2 ** 32, 400000, dtype=np.uint64).astype(np.uint32)
    x = bits.view(np.float32)
    x = x[np.isfinite(x)]
    special = np.array([0.0, -0.0, 65504, 65519.99, 65520, 1e9, -1e9, 2 ** -24, 2 ** -25, 1.5 * 2 ** -25,
                        2 ** -14, 6.1e-5, 1 / 3, 10000.0, 43000.0], np.float32)
    for arr in (x, special, rng.random(100000).astype(np.float32) * 100):
        got = orc.math_eval(6, arr)
        with np.errstate(over="ignore"):
            ref = arr.astype(np.float16).astype(np.float32)
        # finite values beyond the half range store as the largest finite half
        ref = np.where(np.isinf(ref) & np.isfinite(arr), np.copysign(np.float32(65504), arr), ref).astype(np.float32)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def _pcg_np(v):
    v = np.uint32(v)
    with np.errstate(over="ignore"):
        v = v * np.uint32(747796405) + np.uint32(2891336453)
        w = ((v >> ((v >> np.uint32(28)) + np.uint32(4))) ^ v) * np.uint32(277803737)
    return int((w >> np.uint32(22)) ^ w)


def test_pcg_hash(orc):
    for v in [0, 1, 2, 12345, 2 ** 31, 2 ** 32 - 1, 747796405]:
        assert orc.pcg_hash(v) == _pcg_np(v)


def test_camera_matrices_inverse(orc):
    vp, ivp = orc.camera_matrices((8.0, 5.2, 2.5), -0.52, -0.05, math.radians(60), 16 / 9)
    m = vp.reshape(4, 4).T.astype(np.float64) @ ivp.reshape(4, 4).T.astype(np.float64)
    assert np.allclose(m, np.eye(4), atol=1e-4)


# --------------------------------------------------------------------------
# Frame-level behaviour of the oracle (static camera)
# --------------------------------------------------------------------------
def test_temporal_history_grows_and_caps(orc, vrt):
    vox, spawn = vrt.generate_scene(1, 64, 1)
    b, m = orc.build_bricks(vox, 64)
    W, H = 64, 36
    acc = np.zeros((H, W, 4), np.uint16)
    gprev = np.zeros((H, W, 4), np.float32)
    light = vrt.Lighting()
    prev = None
    for f in range(5):
        u = vrt.make_uniforms(spawn, prev, light, f, 2, 1, W, H, 1.0, 3.0)
        r = orc.frame(vox, b, m, 64, vrt.uniforms_bytes(u), 10.0, W, H, acc, gprev)
        acc, gprev, prev = r["accum"], r["gbuf"], spawn
    hist = acc[..., 3].view(np.float16).astype(np.float32)
    geo = r["gbuf"][..., 3] >= 0
    # max history 3 -> history = min(prev, 3) + 1 <= 4 on surfaces, 1 on sky
    assert hist[geo].max() == 4.0
    assert (hist[~geo] == 1.0).all()
    assert np.median(hist[geo]) == 4.0


@pytest.mark.parametrize("kind,n,seed", [(0, 256, 1337), (2, 256, 2), (2, 128, 5), (0, 64, 9)])
def test_oracle_world_matches_library(vrt, orc, kind, n, seed):
    """The oracle's restatement of the world generator (scene.js, seeded) and
    of the benchmark world gives the library's voxels and spawn pose."""
    vox, sp = orc.generate_scene(kind, n, seed)
    want, wsp = vrt.generate_scene(kind, n, seed)
    assert np.array_equal(vox, want.ravel())
    assert tuple(sp["pos"]) == tuple(wsp.pos) and sp["yaw"] == wsp.yaw and sp["pitch"] == wsp.pitch
    assert sp["fov_y"] == wsp.fov_y


@pytest.mark.parametrize("frame", [0, 1, 57, 119])
def test_oracle_uniforms_match_library(vrt, orc, frame):
    """Benchmark camera path and uniform block restated without the library."""
    _, sp = orc.generate_scene(2, 256, 2)
    _, wsp = vrt.generate_scene(2, 256, 2)
    pose = orc.camera_spline(sp, frame)
    prev = orc.camera_spline(sp, frame - 1) if frame else None
    wpose = vrt.camera_spline(wsp, frame)
    wprev = vrt.camera_spline(wsp, frame - 1) if frame else None
    got = orc.uniforms(pose, prev, frame, 2, 3, 1920, 1080, 1.0, 64.0)
    want = vrt.uniforms_bytes(vrt.make_uniforms(wpose, wprev, vrt.Lighting(), frame, 2, 3, 1920, 1080, 1.0, 64.0))
    assert got == want
