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
