"""Image-quality helpers for comparing estimators against a converged
reference: the HDR radiance image of a frame (the demodulated radiance
re-modulated by the stored albedo, as the reference's HDR capture forms it,
main.js:571-661) and its mean squared error."""
from __future__ import annotations

import numpy as np


def hdr_image(session) -> np.ndarray:
    """H x W x 3 float64 radiance of the session's last frame (needs
    keep_radiance_f32): demodulated radiance x (albedo byte / 255)^2."""
    rad = session.radiance_f32()[..., :3].astype(np.float64)
    a = session.albedo()[..., :3].astype(np.float64) / 255.0
    return rad * a * a


def mse(img: np.ndarray, ref: np.ndarray) -> float:
    d = np.asarray(img, np.float64) - np.asarray(ref, np.float64)
    return float(np.mean(d * d))


def write_rgbf32(stem, img: np.ndarray, meta: dict | None = None) -> None:
    """The reference benchmark's reference-image files: <stem>.rgbf32 (raw
    little-endian float32 RGB, row-major from the top row) and <stem>.json
    (width, height, format and the caller's metadata)."""
    import json
    from pathlib import Path
    stem = Path(stem)
    a = np.ascontiguousarray(img, "<f4")
    if a.ndim != 3 or a.shape[2] != 3:
        raise ValueError("image must be H x W x 3")
    stem.with_suffix(".rgbf32").write_bytes(a.tobytes())
    m = {"w": int(a.shape[1]), "h": int(a.shape[0]), "hdrFormat": "rgbf32"}
    m.update(meta or {})
    stem.with_suffix(".json").write_text(json.dumps(m, indent=2))


def read_rgbf32(stem) -> np.ndarray:
    import json
    from pathlib import Path
    stem = Path(stem)
    m = json.loads(stem.with_suffix(".json").read_text())
    a = np.frombuffer(stem.with_suffix(".rgbf32").read_bytes(), "<f4")
    if a.size != m["w"] * m["h"] * 3:
        raise ValueError("reference byte length does not match its metadata")
    return a.reshape(m["h"], m["w"], 3)


def hdr_metrics(ref: np.ndarray, test: np.ndarray) -> dict:
    """The reference's HDR comparison (test/metrics.py:28-49): MSE, RMSE, PSNR
    against the larger image peak, RMSE relative to the reference's RMS, mean
    absolute relative error (denominator floored at 1e-3), per-channel means
    and their relative differences."""
    ref = np.asarray(ref, np.float32)
    test = np.asarray(test, np.float32)
    diff = test - ref
    mse_v = float(np.mean(diff * diff))
    peak = float(max(np.max(ref), np.max(test), 1e-6))
    psnr = float(10.0 * np.log10((peak * peak) / max(mse_v, 1e-20)))
    ref_mean = np.mean(ref, axis=(0, 1))
    test_mean = np.mean(test, axis=(0, 1))
    delta = np.abs(test_mean - ref_mean) / np.maximum(np.abs(ref_mean), 1e-6)
    ref_rms = float(np.sqrt(np.mean(ref * ref)))
    return {"hdrMse": mse_v, "hdrRmse": float(np.sqrt(mse_v)), "hdrPsnrPeak": psnr, "hdrPeak": peak,
            "hdrRelativeRmse": float(np.sqrt(mse_v) / max(ref_rms, 1e-6)),
            "meanAbsRelative": float(np.mean(np.abs(diff) / np.maximum(np.abs(ref), 1e-3))),
            "referenceMeanRgb": [float(v) for v in ref_mean], "testMeanRgb": [float(v) for v in test_mean],
            "channelMeanRelativeDelta": [float(v) for v in delta], "maxChannelMeanRelativeDelta": float(np.max(delta))}


# The reference's estimator-correctness configurations (test/eval/
# correctness-manifest.v1.json): a preset plus per-flag URL overrides
# (main.js:63-69), all with maxhist=1e6 and firefly clamp 0.
CORRECTNESS_CONFIGS = {
    "base": ("base", {}),
    "gi": ("gi", {"treuse": 0}),
    "unified": ("gi", {"unified": 1, "treuse": 0}),
    "lin_unbiased": ("lin", {"treuse": 0, "dupmap": 0, "footprint": 0}),
    "ours_unbiased": ("ours", {"treuse": 0, "dupmap": 0, "rclamp": 0, "footprint": 0}),
}


def config_flags(config: str) -> int:
    """params2.x of a correctness configuration: the preset's flags with the
    overrides applied as main.js:66-69 applies URL flags."""
    from .api import RF, preset_flags
    preset, over = CORRECTNESS_CONFIGS[config]
    f = preset_flags(preset)
    for k, v in over.items():
        f = (f | RF[k]) if v else (f & ~RF[k])
    return f


def accumulated_capture(ctx, scene, pose, light, width: int, height: int, frames: int, bounces: int,
                        flags2: int = 0, light_count: int = 0, fseed: int = 0, session=None) -> np.ndarray:
    """The HDR capture of the reference's converged-image protocol
    (test/bench.mjs reference(): `preset=...&denoise=0&maxhist=1000000&
    fclamp=0&fseed=<seed>`, `stopat=<frames>`): `frames` frames of a static
    camera with temporal accumulation into an rgba32f history capped at 1e6
    frames (a running mean), denoiser off, then the capture
    final x (albedo byte / 255)^2 (main.js:628-659).  Frame f uses RNG stream
    f + fseed, as main.js:415 does.  Returns H x W x 3 float32."""
    from .api import FLAG_TEMPORAL, Session, make_uniforms
    own = session is None
    s = session or Session(ctx, scene, width, height, firefly_clamp=0.0, accum_f32=True)
    try:
        s.reset()
        for f in range(frames):
            u = make_uniforms(pose, pose if f > 0 else None, light, f + fseed, bounces, FLAG_TEMPORAL, width,
                              height, 1.0, 1e6, light_count=light_count)
            u.params2[0] = int(flags2)
            s.frame(u)
        return s.hdr()
    finally:
        if own:
            s.close()
