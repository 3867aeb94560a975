"""Shared inputs for the parity tests: seeded scenes, cameras and rays."""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_voxelbench_states():
    """Yields (key, N, vox, o_m, d, hit, vox_idx, face) from the VoxelBench
    golden fixture, with the grid embedded in an N^3 packed-u32 cube
    (N = max dim rounded up to a multiple of 8) and origins in metres."""
    z = np.load(GOLDEN / "voxelbench_rays.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in z.files})
    for key in keys:
        nx, ny, nz = (int(v) for v in z[key + "_dims"])
        occ = np.unpackbits(z[key + "_occ"])[: nx * ny * nz].reshape(nz, ny, nx)
        n = (max(nx, ny, nz) + 7) // 8 * 8
        g = np.zeros((n, n, n), np.uint32)
        g[:nz, :ny, :nx] = occ.astype(np.uint32) * np.uint32(0x00C8C8C8)
        yield (key, n, np.ascontiguousarray(g).ravel(), (z[key + "_o"] / 16.0).astype(np.float32), z[key + "_d"],
               z[key + "_hit"], z[key + "_vox"], z[key + "_face"])


def random_rays(n_rays: int, N: int, seed: int, inside: bool = True):
    """Origins in metres (inside the grid, or anywhere in a box around it),
    unit directions, maxT; includes axis-aligned and zero-component dirs."""
    rng = np.random.default_rng(seed)
    ext = N / 16.0
    if inside:
        o = rng.random((n_rays, 3)) * ext
    else:
        o = rng.random((n_rays, 3)) * (3 * ext) - ext
    z = rng.random(n_rays) * 2 - 1
    ph = rng.random(n_rays) * 2 * np.pi
    rr = np.sqrt(1 - z * z)
    d = np.stack([rr * np.cos(ph), z, rr * np.sin(ph)], 1)
    k = n_rays // 16
    axes = np.eye(3)[rng.integers(0, 3, k)] * rng.choice([-1.0, 1.0], (k, 1))
    d[:k] = axes                                   # axis-aligned: two zero components
    d[k:2 * k, rng.integers(0, 3)] = 0.0           # one zero component
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.where(rng.random(n_rays) < 0.2, rng.random(n_rays) * ext, 1e4)
    return o.astype(np.float32), d.astype(np.float32), tmax.astype(np.float32)


def small_setup(vrt, kind=1, n=64, seed=1):
    vox, spawn = vrt.generate_scene(kind, n, seed)
    return vox, spawn


def spline_pose(vrt, spawn, f):
    return vrt.camera_spline(spawn, f)
