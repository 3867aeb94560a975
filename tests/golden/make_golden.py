"""Generates tests/golden/voxelbench_rays.npz from the reference's own CPU
traversal (VoxelBench/pipeline/core.cpp:23-50 traceNaive, double precision),
compiled from the reference sources by `make -C oracle ref`.

For each VoxelBench scene (scenes.h:183-190 makeScene) in its pre- and
post-event state, rays are drawn the way `bench test` draws them
(harness.cpp:205-239: origins 1 + U*(dim-2) per axis, directions uniform on
the sphere) and kept when the origin voxel is empty.  The fixture stores the
bit-packed occupancy grid (index (z*NY+y)*NX+x), the rays
and traceNaive's hit flag, voxel and face.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle  # noqa: E402

SCENES = [b"bunker", b"courtyard", b"cavern", b"town"]
RAYS_PER_STATE = {b"bunker": 3000, b"courtyard": 3000, b"cavern": 3000, b"town": 1500}


def main() -> None:
    oracle.build(ref=True)
    vb = oracle.ref_lib()
    assert vb is not None, "reference traversal library was not built"
    out = {}
    p = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    for si, name in enumerate(SCENES):
        for post in (0, 1):
            dims = (C.c_int * 3)()
            assert vb.vb_build_scene(name, post, dims) == 0
            nx, ny, nz = dims
            g = np.zeros(nx * ny * nz, np.uint8)
            vb.vb_copy_grid(p(g))
            g3 = g.reshape(nz, ny, nx)
            rng = np.random.default_rng(1000 + 2 * si + post)
            want = RAYS_PER_STATE[name]
            n = want * 4
            o = np.stack([1 + rng.random(n) * (nx - 2), 1 + rng.random(n) * (ny - 2), 1 + rng.random(n) * (nz - 2)],
                         1).astype(np.float32)
            z = rng.random(n) * 2 - 1
            ph = rng.random(n) * 2 * np.pi
            rr = np.sqrt(np.maximum(0, 1 - z * z))
            d = np.stack([rr * np.cos(ph), z, rr * np.sin(ph)], 1).astype(np.float32)
            oi = np.floor(o).astype(np.int64)
            keep = g3[oi[:, 2], oi[:, 1], oi[:, 0]] == 0
            o = np.ascontiguousarray(o[keep][:want])
            d = np.ascontiguousarray(d[keep][:want])
            n = o.shape[0]
            tmax = np.full(n, 1e9, np.float32)
            hit = np.zeros(n, np.int32)
            vox = np.zeros(3 * n, np.int32)
            face = np.zeros(n, np.int32)
            t = np.zeros(n, np.float32)
            vb.vb_trace_naive_batch(p(o), p(d), p(tmax), C.c_int(n), p(hit), p(vox), p(face), p(t))
            key = f"{name.decode()}_{'post' if post else 'pre'}"
            out[key + "_dims"] = np.array([nx, ny, nz], np.int32)
            out[key + "_occ"] = np.packbits(g != 0)
            out[key + "_o"] = o
            out[key + "_d"] = d
            out[key + "_hit"] = hit
            out[key + "_vox"] = vox.reshape(n, 3)
            out[key + "_face"] = face
            out[key + "_t"] = t
            print(key, (nx, ny, nz), n, "hits", int(hit.sum()))
    dst = Path(__file__).resolve().parent / "voxelbench_rays.npz"
    np.savez_compressed(dst, **out)
    print("wrote", dst, dst.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
