"""Writes tests/golden/estimator_correctness_rows.json from the reference's own
estimator-correctness record and manifests:

  test/eval/estimator-correctness.v1.json   per (scenario, config): the channel
      means of the 1600-frame, 12-bounce reference capture and of the
      800-frame, 8-bounce test capture, and the HDR error between them
  test/eval/correctness-manifest.v1.json    capture settings and configurations
  test/eval/claim-manifest.v1.json          scenario poses and scene variants

The reference produced these numbers with its WebGPU renderer (RTX 3080,
Chromium); they pin this library's shading against the reference's own
converged statistics.  Run with the reference checkout available:

  VRT_REFERENCE_ROOT=<checkout> python tests/golden/make_estimator_rows.py
"""
from __future__ import annotations

import json
import os
from pathlib import Path


def main() -> None:
    root = Path(os.environ["VRT_REFERENCE_ROOT"])
    ev = root / "test" / "eval"
    rec = json.loads((ev / "estimator-correctness.v1.json").read_text())
    man = json.loads((ev / "correctness-manifest.v1.json").read_text())
    claim = json.loads((ev / "claim-manifest.v1.json").read_text())
    scen = {}
    for name in man["scenarios"]:
        s = claim["scenarios"][name]
        scen[name] = {"pose": s["pose"], "scene": s.get("scene", "default")}
    rows = []
    for r in rec["rows"]:
        m = r["metrics"]
        rows.append({"scenario": r["scenario"], "config": r["config"], "query": r["query"], "frames": r["frames"],
                     "bounces": r["bounces"], "seed": r["seed"], "referenceMeanRgb": m["referenceMeanRgb"],
                     "testMeanRgb": m["testMeanRgb"], "hdrMse": m["hdrMse"], "hdrPsnrPeak": m["hdrPsnrPeak"],
                     "hdrRelativeRmse": m["hdrRelativeRmse"],
                     "maxChannelMeanRelativeDelta": m["maxChannelMeanRelativeDelta"]})
    out = {"source": "test/eval/estimator-correctness.v1.json, correctness-manifest.v1.json, "
                     "claim-manifest.v1.json of the reference",
           "resolution": rec["resolution"], "reference": rec["reference"], "thresholds": rec["thresholds"],
           "capture": man["capture"], "fireflyClamp": claim["capture"]["fireflyClamp"],
           "configurations": man["configurations"], "scenarios": scen, "rows": rows}
    dst = Path(__file__).with_name("estimator_correctness_rows.json")
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(dst, len(rows), "rows")


if __name__ == "__main__":
    main()
