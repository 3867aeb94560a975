"""The VoxelBench Technique adapter (voxelrt_b200/adapters/method_vrt.h) in the
harness's protocol (VoxelBench/pipeline/harness.cpp:280-330): the reference's
own baseline technique MethodPT (techniques/pt.h) on the CPU and MethodVRT on
the GPU at the same ray budget, on the reference's scenes, scored by the
reference's metrics (metrics.h) against a path-traced reference rendered by
the reference's renderReference -- all compiled from the reference sources
into oracle/_ref/vb_vrt.

MethodVRT runs the same estimator with the same random streams on this
library's DDA, so it must spend the same rays and land on the same quality
and energy; single paths may differ at grazing traversal ties, so the
comparison is on the harness's image metrics, with the tolerances below.
"""
import json
import os
import subprocess

import pytest

import oracle

pytestmark = pytest.mark.gpu


def _run(scene, frames, ref_spp, event=-1, mult=1.0):
    assert oracle.VB_VRT.exists(), "oracle/_ref/vb_vrt is built by __graft_entry__.build() next to the reference"
    cmd = [str(oracle.VB_VRT), scene, str(mult), str(frames), str(ref_spp), str(os.cpu_count() or 1), str(event)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    rows = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    summary = {x["summary"]: x for x in rows if "summary" in x}
    per_frame = {m: [x for x in rows if x.get("method") == m] for m in ("PT", "VRT")}
    return summary, per_frame


@pytest.mark.parametrize("scene,event", [("bunker", 6), ("cavern", 6), ("courtyard", 6), ("town", -1)])
def test_adapter_matches_reference_baseline(scene, event):
    """Same budget, same rays, same quality and energy as the reference's MethodPT,
    before and after the scene's event (geometry edit or lighting change)."""
    summary, per_frame = _run(scene, 12, 32, event)
    pt, vrt = summary["PT"], summary["VRT"]
    assert len(per_frame["VRT"]) == 12
    for a, b in zip(per_frame["PT"], per_frame["VRT"]):
        assert abs(b["rays"] - a["rays"]) <= 0.01 * a["rays"], (a, b)
    assert abs(vrt["psnr"] - pt["psnr"]) < 0.5, (pt, vrt)
    assert abs(vrt["gpsnr"] - pt["gpsnr"]) < 0.5, (pt, vrt)
    assert abs(vrt["ssim"] - pt["ssim"]) < 0.01, (pt, vrt)
    assert abs(vrt["mean_luma"] / pt["mean_luma"] - 1.0) < 0.03, (pt, vrt)


@pytest.mark.parametrize("mult", [0.5, 2.0])
def test_adapter_follows_the_budget(mult):
    """Fractional and multiple path counts per pixel (techniques/pt.h:25-28)."""
    summary, _ = _run("bunker", 6, 16, -1, mult)
    pt, vrt = summary["PT"], summary["VRT"]
    assert abs(vrt["rays_per_frame"] / pt["rays_per_frame"] - 1.0) < 0.01
    assert abs(vrt["psnr"] - pt["psnr"]) < 0.5
