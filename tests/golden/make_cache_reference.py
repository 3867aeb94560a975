"""Generates the converged images the cache-assisted estimator is scored
against:

  cache_reference_64_256x144.npz   the 64^3 seed-1 test scene (a Cornell room
                                   with an emissive ceiling panel on value-noise
                                   terrain) at 256x144
  cache_reference_256_480x270.npz  the 256^3 seed-2 world (terrain, room, 40
                                   trees, three lanterns) at 480x270

Both from the scene's spawn pose, sun (0.3, 0.8, 0.5), firefly clamp 10.
Estimator: the plain path with 6 bounces (Russian roulette from bounce 2),
4096 samples per pixel (frame indices 2^20 .. 2^20 + 4095, disjoint from the
frames the tests and the bench render), accumulated in FP64 by the CPU oracle
(orc_accumulate_f64) and stored as float32 HDR radiance (demodulated radiance
x (albedo byte / 255)^2).

Run from the repository root: python tests/golden/make_cache_reference.py [64|256]
"""
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
import voxelrt_b200 as vrt  # noqa: E402

# name: (scene kind, grid, seed, width, height)
CASES = {
    64: (vrt.VRT_SCENE_SMALL, 64, 1, 256, 144),
    256: (vrt.VRT_SCENE_FULL, 256, 2, 480, 270),
}
BOUNCES, FCLAMP, SPP, FRAME0 = 6, 10.0, 4096, 1 << 20


def path(n: int) -> Path:
    _, _, _, w, h = CASES[n]
    return Path(__file__).with_name(f"cache_reference_{n}_{w}x{h}.npz")


def make(n: int) -> None:
    kind, N, seed, W, H = CASES[n]
    vox, spawn = vrt.generate_scene(kind, N, seed)
    bricks, masks = oracle.build_bricks(vox, N)
    u = vrt.make_uniforms(spawn, None, vrt.Lighting(), 0, BOUNCES, 0, W, H)
    t = time.time()
    acc = oracle.accumulate_f64(vox, bricks, masks, N, vrt.uniforms_bytes(u), FCLAMP, W, H, FRAME0, SPP)
    ref = (acc / SPP).astype(np.float32)
    print(f"{N}^3 {W}x{H}: {SPP} spp in {time.time() - t:.1f} s; mean {ref.mean(axis=(0, 1))}")
    np.savez_compressed(path(n), ref=ref, meta=np.array([kind, N, seed, W, H, BOUNCES, SPP, FRAME0], np.int64),
                        fclamp=np.float32(FCLAMP))


def main():
    oracle.build(ref=False)
    for n in ([int(a) for a in sys.argv[1:]] or list(CASES)):
        make(n)


if __name__ == "__main__":
    main()
