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
