"""Pin of the shading against the reference's own converged statistics.

The reference's estimator-correctness gate (test/eval/correctness-manifest.v1.json,
record test/eval/estimator-correctness.v1.json, both read into
tests/golden/estimator_correctness_rows.json by make_estimator_rows.py)
renders three static scenarios of its world at 1920x1080 with its WebGPU
renderer: a reference capture of 1600 frames at 12 bounces and, per
configuration, a test capture of 800 frames at 8 bounces, both with
`maxhist=1000000&fclamp=0&denoise=0&fseed=0`, and records each capture's
per-channel HDR mean and the HDR error between the two.

Here the same captures are rendered by this library (same world, poses, sun,
camera, RNG streams and capture) and compared with those records:
  * every channel mean within 1% of the reference's (the gate's own
    maxChannelMeanRelativeDelta), for the reference capture and the test
    capture of each configuration;
  * the HDR MSE between this library's test and reference captures within
    5% (plain path) or 25% (ReSTIR) of the MSE the reference recorded between
    its own two captures.
The reference renders the same per-pixel RNG streams, so the plain path's
channel means agree far more closely than the 1% gate (within 0.5% is
asserted); the achieved deltas are printed.
"""
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROWS = json.loads((Path(__file__).parent / "golden" / "estimator_correctness_rows.json").read_text())
W, H = ROWS["resolution"]["width"], ROWS["resolution"]["height"]
REF_FRAMES, REF_BOUNCES = ROWS["reference"]["frames"], ROWS["reference"]["bounces"]
MEAN_TOL = ROWS["thresholds"]["maxChannelMeanRelativeDelta"]     # 0.01


def _row(scenario, config):
    return next(r for r in ROWS["rows"] if r["scenario"] == scenario and r["config"] == config)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b) / np.abs(b)


@pytest.fixture(scope="module")
def world(vrt):
    ctx = vrt.Context(0)
    scenes = {}
    yield ctx, scenes
    for sc in scenes.values():
        sc[0].close()
    ctx.close()


def _scene(vrt, world, variant):
    ctx, scenes = world
    if variant not in scenes:
        kind = vrt.VRT_SCENE_VOXELRT_LAMPS if variant == "lamps" else vrt.VRT_SCENE_VOXELRT
        vox, _ = vrt.generate_scene(kind, 256, 1337)
        sc = vrt.Scene(ctx, vox, 256)
        scenes[variant] = (sc, int(sc.build_lights().count))
    return scenes[variant]


_CAPTURES = {}


def _capture(vrt, world, scenario, frames, bounces, config):
    key = (scenario, frames, bounces, config)
    if key not in _CAPTURES:
        _CAPTURES[key] = _render(vrt, world, scenario, frames, bounces, config)
    return _CAPTURES[key]


def _render(vrt, world, scenario, frames, bounces, config):
    from voxelrt_b200 import quality
    ctx, _ = world
    s = ROWS["scenarios"][scenario]
    sc, nlights = _scene(vrt, world, s["scene"])
    p = s["pose"]
    pose = vrt.CameraPose((p["px"], p["py"], p["pz"]), p["yaw"], p["pitch"])
    return quality.accumulated_capture(ctx, sc, pose, vrt.Lighting.reference_default(), W, H, frames, bounces,
                                       quality.config_flags(config), nlights, fseed=0)


@pytest.mark.parametrize("scenario", ["interior_static", "exterior_static", "lamps_static"])
def test_base_captures_match_reference_statistics(vrt, world, scenario):
    from voxelrt_b200 import quality
    row = _row(scenario, "base")
    ref = _capture(vrt, world, scenario, REF_FRAMES, REF_BOUNCES, "base")
    test = _capture(vrt, world, scenario, row["frames"], row["bounces"], "base")
    m = quality.hdr_metrics(ref, test)
    d_ref = _rel(m["referenceMeanRgb"], row["referenceMeanRgb"])
    d_test = _rel(m["testMeanRgb"], row["testMeanRgb"])
    print(f"{scenario}: reference means {np.round(m['referenceMeanRgb'], 5)} vs {row['referenceMeanRgb']} "
          f"(max delta {d_ref.max():.2e}); test means {np.round(m['testMeanRgb'], 5)} vs {row['testMeanRgb']} "
          f"(max delta {d_test.max():.2e}); hdrMse {m['hdrMse']:.5f} vs {row['hdrMse']:.5f}, "
          f"PSNR {m['hdrPsnrPeak']:.2f} vs {row['hdrPsnrPeak']:.2f} dB")
    assert d_ref.max() <= MEAN_TOL, d_ref
    assert d_test.max() <= MEAN_TOL, d_test
    # the same per-pixel RNG streams: far inside the gate (measured 0.06-0.15%)
    assert max(d_ref.max(), d_test.max()) <= 0.005, (d_ref, d_test)
    assert abs(m["hdrMse"] / row["hdrMse"] - 1.0) <= 0.05, (m["hdrMse"], row["hdrMse"])


def test_ours_unbiased_capture_matches_reference_statistics(vrt, world):
    """The reference's default ReSTIR preset in its unbiased form (temporal
    reuse, duplication map, contribution clamp and footprint off) on the
    interior scenario: 800 frames at 8 bounces against the recorded test
    means, and its MSE against this library's 12-bounce plain reference."""
    from voxelrt_b200 import quality
    row = _row("interior_static", "ours_unbiased")
    ref = _capture(vrt, world, "interior_static", REF_FRAMES, REF_BOUNCES, "base")
    test = _capture(vrt, world, "interior_static", row["frames"], row["bounces"], "ours_unbiased")
    m = quality.hdr_metrics(ref, test)
    d_test = _rel(m["testMeanRgb"], row["testMeanRgb"])
    print(f"ours_unbiased interior: test means {np.round(m['testMeanRgb'], 5)} vs {row['testMeanRgb']} "
          f"(max delta {d_test.max():.2e}); hdrMse {m['hdrMse']:.5f} vs {row['hdrMse']:.5f}")
    assert d_test.max() <= MEAN_TOL, d_test
    assert abs(m["hdrMse"] / row["hdrMse"] - 1.0) <= 0.25, (m["hdrMse"], row["hdrMse"])
