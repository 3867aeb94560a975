"""The VoxelBench harness driver (oracle/_ref/vb_vrt) builds from the reference
sources with the adapter header and links the library; without arguments it
prints its usage (no GPU needed)."""
import subprocess

import pytest

import oracle


def test_harness_driver_builds_and_runs():
    have_src = oracle.REF_SRC is not None and oracle.REF_SRC.exists()
    if not have_src and not oracle.VB_VRT.exists():
        pytest.skip("neither the reference sources nor a built driver are present")
    if not oracle.VB_VRT.exists():
        oracle.build(ref=True)
    r = subprocess.run([str(oracle.VB_VRT)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage: vb_vrt" in r.stderr
