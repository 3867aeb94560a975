"""Build voxelrt_b200/libvrt.so (the C-ABI library with the sm_100a kernels).

Kernels are compiled for sm_100a only, with the floating-point contract the
parity tests rely on: no FMA contraction (-fmad=false), IEEE division and
square root, denormals kept.  The CUDA runtime is linked statically so the
library has no dependency beyond the NVIDIA driver.

Usage: python -m voxelrt_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libvrt.so"

CU_SOURCES = ["k_trace.cu", "k_image.cu", "k_atrous_tma.cu", "k_wavefront.cu", "k_noalloc.cu", "k_batch.cu",
              "k_mlp.cu", "k_hdr.cu", "k_lights.cu", "k_restir.cu", "k_vb.cu"]
CPP_SOURCES = ["vrt_api.cpp", "scene_gen.cpp", "pairing.cpp"]
HEADERS = ["vrt_device.cuh", "vrt_internal.h", "wavefront_core.cuh", "image_core.cuh", "umma.cuh",
           "trace_kernel.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FP_CONTRACT = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]


def _nvcc() -> str:
    cands = [os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"]
    for c in cands:
        if c and Path(c, "bin", "nvcc").exists():
            return str(Path(c, "bin", "nvcc"))
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found (set CUDA_HOME)")
    return found


def _host_cxx() -> str:
    # nvcc needs a g++ it supports; prefer the system one.
    for c in ("/usr/bin/g++", shutil.which("g++") or ""):
        if c and Path(c).exists():
            return c
    raise RuntimeError("g++ not found")


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    out = r.stdout + r.stderr
    if verbose and out:
        print(out, flush=True)
    elif "warning" in out:
        # warnings are never silent (a host call of a device-only function,
        # for one, compiles to a stub that ends the process at run time)
        sys.stderr.write(out)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    nvcc = _nvcc()
    cxx = _host_cxx()
    BUILD.mkdir(exist_ok=True)
    hdrs = [CSRC / h for h in HEADERS] + [ROOT / "include" / "vrt.h"]
    objs = []
    common = ["-std=c++17", "-O3", "-ccbin", cxx, "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc, *common, *ARCH, *FP_CONTRACT, "-lineinfo", "-c", str(s), "-o", str(o)]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            _run(cmd, verbose or ptxas_verbose)
    for src in CPP_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            _run([nvcc, *common, "-x", "cu", *ARCH, "-c", str(s), "-o", str(o)], verbose)
    if force or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([nvcc, "-shared", *ARCH, "-ccbin", cxx, "-cudart", "static", *map(str, objs), "-o", str(tmp)], verbose)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
