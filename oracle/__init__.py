"""Test infrastructure: ctypes loader for the CPU oracle (liboracle.so) and the
reference VoxelBench traversal (_ref/libvbref.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this package; the product (voxelrt_b200) never does.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
LITERAL_LIB = HERE / "liboracle_literal.so"
REF_LIB = HERE / "_ref" / "libvbref.so"
# The reference checkout, when it is available (it is only needed to build
# the reference traversal library and the golden fixtures).
REF_ROOT = Path(os.environ["VRT_REFERENCE_ROOT"]) if os.environ.get("VRT_REFERENCE_ROOT") else None
REF_SRC = REF_ROOT / "VoxelBench" / "pipeline" if REF_ROOT else None

HIT_DTYPE = np.dtype([("t", "<f4"), ("n", "<f4", 3), ("mat", "<u4"), ("voxel", "<i4", 3), ("face", "<i4"),
                      ("steps", "<u4"), ("bytes", "<u4"), ("pad", "<u4")])


class OrcStats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("outer", C.c_uint64), ("inner", C.c_uint64), ("vreads", C.c_uint64),
                ("pixels", C.c_uint64)]


VB_VRT = HERE / "_ref" / "vb_vrt"


def build(ref: bool | None = None) -> None:
    """make -C oracle (and, when the reference sources exist, the reference
    traversal library and the VoxelBench harness driver vb_vrt, which links
    voxelrt_b200/libvrt.so)."""
    targets = ["all"]
    if ref and REF_SRC is None:
        raise RuntimeError("oracle.build(ref=True): set VRT_REFERENCE_ROOT to the reference checkout")
    if ref or (ref is None and REF_SRC is not None and REF_SRC.exists()):
        targets += ["ref", "vbvrt"]
    subprocess.run(["make", "-s", "-C", str(HERE), *targets], check=True)


_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build(ref=False)
        _lib = C.CDLL(str(LIB))
    return _lib


_literal = None


@contextlib.contextmanager
def literal_wgsl():
    """Within the block, the oracle's functions run the literal restatement of
    the shaders (liboracle_literal.so): C-library transcendentals, dot
    products and a-trous weights as written, none of the kernels'
    reformulations.  Kernels agree with it within the specification's
    tolerances, not bit for bit."""
    global _lib, _literal
    if _literal is None:
        if not LITERAL_LIB.exists():
            build(ref=False)
        _literal = C.CDLL(str(LITERAL_LIB))
    saved = lib()
    _lib = _literal
    try:
        yield
    finally:
        _lib = saved


def _host_isa_level() -> int:
    """The x86-64 micro-architecture level of this host (1..4) from
    /proc/cpuinfo's flags."""
    try:
        flags = set()
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("flags"):
                flags = set(line.split(":", 1)[1].split())
                break
    except OSError:
        return 1
    v3 = {"avx", "avx2", "bmi1", "bmi2", "f16c", "fma", "movbe", "xsave", "abm"}
    v4 = {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"}
    if not v3 <= flags:
        return 1
    return 4 if v4 <= flags else 3


def ref_lib_best():
    """The reference traversal built for the highest ISA level this host
    supports (VoxelBench's own build uses -march=native), with a label of
    the build; (None, None) when it was not built."""
    global _ref
    level = _host_isa_level()
    for lv, name, label in [(4, "libvbref_v4.so", "-O2 -march=x86-64-v4 -fopenmp"),
                            (3, "libvbref_v3.so", "-O2 -march=x86-64-v3 -fopenmp"),
                            (1, "libvbref.so", "-O2 -fopenmp")]:
        path = HERE / "_ref" / name
        if lv <= level and path.exists():
            if _ref is None:
                _ref = C.CDLL(str(path))
                _ref.vb_time_trace.restype = C.c_double
                _ref.vb_copy_grid.restype = C.c_long
            return _ref, label + " (the host's ISA level)"
    return None, None


def ref_lib() -> C.CDLL | None:
    """The reference's VoxelBench traversal, or None when it was not built."""
    global _ref
    if _ref is None and REF_LIB.exists():
        _ref = C.CDLL(str(REF_LIB))
        _ref.vb_time_trace.restype = C.c_double
        _ref.vb_copy_grid.restype = C.c_long
    return _ref


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def num_threads() -> int:
    return int(lib().orc_num_threads())


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def build_bricks(vox: np.ndarray, n: int):
    bg = n // 8
    bricks = np.zeros(bg ** 3, np.uint32)
    masks = np.zeros(16 * bg ** 3, np.uint32)
    lib().orc_build_bricks(_p(np.ascontiguousarray(vox, np.uint32)), C.c_int(n), _p(bricks), _p(masks))
    return bricks, masks


def trace(vox, bricks, masks, n, o, d, tmax) -> np.ndarray:
    o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
    d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tmax, np.float32).reshape(-1)
    out = np.zeros(o.shape[0], HIT_DTYPE)
    lib().orc_trace(_p(vox), _p(bricks), _p(masks), C.c_int(n), _p(o), _p(d), _p(t), C.c_int(o.shape[0]), _p(out))
    return out


def trace_naive(vox, n, o, d, tmax) -> np.ndarray:
    o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
    d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tmax, np.float32).reshape(-1)
    out = np.zeros(o.shape[0], HIT_DTYPE)
    lib().orc_trace_naive(_p(vox), C.c_int(n), _p(o), _p(d), _p(t), C.c_int(o.shape[0]), _p(out))
    return out


def pathtrace(vox, bricks, masks, n, ubytes: bytes, fclamp: float, w: int, h: int, row0=0, row1=None, row_step=1):
    """Returns dict rad16 (u16 HxWx4), rad32 (f32), alb8 (u8), gbuf (f32), stats."""
    row1 = h if row1 is None else row1
    ub = np.frombuffer(ubytes, np.uint8).copy()
    rad16 = np.zeros((h, w, 4), np.uint16)
    rad32 = np.zeros((h, w, 4), np.float32)
    alb8 = np.zeros((h, w, 4), np.uint8)
    gbuf = np.zeros((h, w, 4), np.float32)
    st = OrcStats()
    lib().orc_pathtrace(_p(vox), _p(bricks), _p(masks), C.c_int(n), _p(ub), C.c_float(fclamp), C.c_int(w), C.c_int(h),
                        C.c_int(row0), C.c_int(row1), C.c_int(row_step), _p(rad16), _p(rad32), _p(alb8), _p(gbuf),
                        C.byref(st))
    return {"rad16": rad16, "rad32": rad32, "alb8": alb8, "gbuf": gbuf,
            "stats": {k: int(getattr(st, k)) for k, _ in OrcStats._fields_}}


def path_signatures(vox, bricks, masks, n, ubytes: bytes, fclamp: float, w: int, h: int, row0=0, row1=None,
                    row_step=1):
    """pathtrace() plus sig: per pixel a hash of its discrete path (every trace
    in order with its outcome: miss, or hit voxel and face)."""
    row1 = h if row1 is None else row1
    ub = np.frombuffer(ubytes, np.uint8).copy()
    rad16 = np.zeros((h, w, 4), np.uint16)
    rad32 = np.zeros((h, w, 4), np.float32)
    alb8 = np.zeros((h, w, 4), np.uint8)
    gbuf = np.zeros((h, w, 4), np.float32)
    sig = np.zeros((h, w), np.uint32)
    st = OrcStats()
    lib().orc_pathtrace_sig(_p(vox), _p(bricks), _p(masks), C.c_int(n), _p(ub), C.c_float(fclamp), C.c_int(w),
                            C.c_int(h), C.c_int(row0), C.c_int(row1), C.c_int(row_step), _p(rad16), _p(rad32),
                            _p(alb8), _p(gbuf), C.byref(st), _p(sig))
    return {"rad16": rad16, "rad32": rad32, "alb8": alb8, "gbuf": gbuf, "sig": sig, "rays": int(st.rays)}


def temporal(ubytes, w, h, rad16, gcur, acc_prev, gprev, acc_f32: bool):
    ub = np.frombuffer(ubytes, np.uint8).copy()
    out = np.zeros((h, w, 4), np.float32 if acc_f32 else np.uint16)
    lib().orc_temporal(_p(ub), C.c_int(w), C.c_int(h), _p(np.ascontiguousarray(rad16)), _p(np.ascontiguousarray(gcur)),
                       _p(np.ascontiguousarray(acc_prev)), _p(np.ascontiguousarray(gprev)), _p(out),
                       C.c_int(int(acc_f32)))
    return out


def atrous(w, h, src, src_f32: bool, gbuf, step: int):
    out = np.zeros((h, w, 4), np.uint16)
    lib().orc_atrous(None, C.c_int(w), C.c_int(h), _p(np.ascontiguousarray(src)), C.c_int(int(src_f32)),
                     _p(np.ascontiguousarray(gbuf)), _p(out), C.c_int(step))
    return out


def present(ubytes, w, h, final, final_f32: bool, alb8):
    ub = np.frombuffer(ubytes, np.uint8).copy()
    out = np.zeros((h, w, 4), np.uint8)
    lib().orc_present(_p(ub), C.c_int(w), C.c_int(h), _p(np.ascontiguousarray(final)), C.c_int(int(final_f32)),
                      _p(np.ascontiguousarray(alb8)), _p(out))
    return out


def hdr(w, h, final, final_f32: bool, alb8):
    out = np.zeros((h, w, 3), np.float32)
    lib().orc_hdr(C.c_int(w), C.c_int(h), _p(np.ascontiguousarray(final)), C.c_int(int(final_f32)),
                  _p(np.ascontiguousarray(alb8)), _p(out))
    return out


def accumulate_f64(vox, bricks, masks, n, ubytes, fclamp, w, h, frame0: int, spp: int, accum=None):
    ub = np.frombuffer(ubytes, np.uint8).copy()
    acc = np.zeros((h, w, 3), np.float64) if accum is None else accum
    lib().orc_accumulate_f64(_p(vox), _p(bricks), _p(masks), C.c_int(n), _p(ub), C.c_float(fclamp), C.c_int(w),
                             C.c_int(h), C.c_uint32(frame0), C.c_int(spp), _p(acc))
    return acc


def collect_rays(vox, bricks, masks, n, ubytes, fclamp, w, h, row0=0, row1=None, row_step=1, cap=None):
    """Rays (N x 7: origin xyz and maxT in voxel units, direction) traced by
    the oracle path for the selected rows."""
    row1 = h if row1 is None else row1
    ub = np.frombuffer(ubytes, np.uint8).copy()
    nrows = len(range(row0, min(row1, h), row_step))
    cap = cap or nrows * w * 8
    out = np.zeros((cap, 7), np.float32)
    f = lib().orc_collect_rays
    f.restype = C.c_long
    total = f(_p(vox), _p(bricks), _p(masks), C.c_int(n), _p(ub), C.c_float(fclamp), C.c_int(w), C.c_int(h),
              C.c_int(row0), C.c_int(row1), C.c_int(row_step), _p(out), C.c_long(cap))
    return out[:min(total, cap)]


def camera_matrices(pos, yaw, pitch, fov_y, aspect, near_z=0.05, far_z=400.0):
    p = (C.c_double * 3)(*pos)
    vp = np.zeros(16, np.float32)
    ivp = np.zeros(16, np.float32)
    lib().orc_camera_matrices(p, C.c_double(yaw), C.c_double(pitch), C.c_double(fov_y), C.c_double(aspect),
                              C.c_double(near_z), C.c_double(far_z), _p(vp), _p(ivp))
    return vp, ivp


def math_eval(fn: int, x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros_like(x)
    lib().orc_math_eval(C.c_int(fn), _p(x), _p(y), C.c_int(x.size))
    return y


CACHE_PIX_DTYPE = np.dtype([("role", "<i4"), ("has_query", "<i4"), ("nrec", "<i4"), ("pad", "<i4"),
                            ("den", "<f4", 3), ("radiance", "<f4", 3), ("tp1", "<f4", 3), ("q9", "<f4", 9),
                            ("rec", "<f4", (8, 15))])


def cache_paths(vox, bricks, masks, n, ubytes, w, h, phase: int, train_bounces: int, rec_vertices: int):
    """Per-pixel cache-assisted estimator parts (CACHE_PIX_DTYPE, h x w)."""
    assert lib().orc_cache_pix_bytes() == CACHE_PIX_DTYPE.itemsize
    ub = np.frombuffer(ubytes, np.uint8).copy()
    out = np.zeros(h * w, CACHE_PIX_DTYPE)
    lib().orc_cache_paths(_p(vox), _p(bricks), _p(masks), C.c_int(n), _p(ub), C.c_int(w), C.c_int(h),
                          C.c_uint32(phase), C.c_uint32(train_bounces), C.c_int(rec_vertices), _p(out))
    return out.reshape(h, w)


def light_list(vox, n: int):
    """(words [k x 2] uint32, weights [k] float64) -- scene.js's emissive-face list."""
    vox = np.ascontiguousarray(vox, np.uint32)
    lib().orc_light_list.restype = C.c_long
    k = lib().orc_light_list(_p(vox), C.c_int(n), None, None, C.c_long(0))
    words = np.zeros((max(k, 1), 2), np.uint32)
    weights = np.zeros(max(k, 1), np.float64)
    lib().orc_light_list(_p(vox), C.c_int(n), _p(words), _p(weights), C.c_long(k))
    return words[:k], weights[:k]


def light_alias(weights):
    w = np.ascontiguousarray(weights, np.float64)
    out = np.zeros((max(len(w), 1), 4), np.float32)
    lib().orc_light_alias(_p(w), C.c_long(len(w)), _p(out))
    return out


def light_grid(n: int, words, weights):
    words = np.ascontiguousarray(words, np.uint32)
    w = np.ascontiguousarray(weights, np.float64)
    bg = n // 8
    out = np.zeros((bg ** 3, 34), np.uint32)
    lib().orc_light_grid(C.c_int(n), _p(words), _p(w), C.c_long(len(w)), _p(out))
    return out


def pcg_hash(v: int) -> int:
    f = lib().orc_pcg_hash
    f.restype = C.c_uint32
    return int(f(C.c_uint32(v)))


PAIRING_WORDS = 254 * 254 + 230 * 230 + 210 * 210


def _ptr_or_none(a):
    return _p(np.ascontiguousarray(a)) if a is not None else None


def restir_initial(vox, bricks, masks, n, ubytes, fclamp: float, w: int, h: int, lights=None):
    """ReSTIR initial-candidate pass (pathtrace.wgsl:332-457).  lights: dict
    with "words", "alias", "grid" (the scene's light data) for RF_UNIFIED.
    Returns rad16, rad32 (sky pixels only), alb8, gbuf, resA (u32 HxWx8, the
    32-byte reservoir records), direct (rgba16f bits), stats."""
    ub = np.frombuffer(ubytes, np.uint8).copy()
    rad16 = np.zeros((h, w, 4), np.uint16)
    rad32 = np.zeros((h, w, 4), np.float32)
    alb8 = np.zeros((h, w, 4), np.uint8)
    gbuf = np.zeros((h, w, 4), np.float32)
    res_a = np.zeros((h, w, 8), np.uint32)
    direct = np.zeros((h, w, 4), np.uint16)
    st = OrcStats()
    lw = la = lg = None
    if lights is not None:
        lw = np.ascontiguousarray(lights["words"], np.uint32)
        la = np.ascontiguousarray(lights["alias"], np.float32)
        lg = np.ascontiguousarray(lights["grid"], np.uint32)
    lib().orc_restir_initial(_p(vox), _p(bricks), _p(masks), C.c_int(n), _p(ub), C.c_float(fclamp), C.c_int(w),
                             C.c_int(h), _ptr_or_none(lw), _ptr_or_none(la), _ptr_or_none(lg), _p(rad16), _p(rad32),
                             _p(alb8), _p(gbuf), _p(res_a), _p(direct), C.byref(st))
    return {"rad16": rad16, "rad32": rad32, "alb8": alb8, "gbuf": gbuf, "resA": res_a, "direct": direct,
            "stats": {k: int(getattr(st, k)) for k, _ in OrcStats._fields_}}


def restir_temporal(ubytes, w: int, h: int, gcur, gprev, res_b, res_a, dup=None):
    """Temporal reservoir reuse (reuse_temporal.wgsl); dup = the previous
    frame's duplication map (RF_DUPMAP).  Returns the merged A."""
    ub = np.frombuffer(ubytes, np.uint8).copy()
    out = np.array(res_a, np.uint32, copy=True, order="C")
    d = np.zeros((h, w), np.float32) if dup is None else np.ascontiguousarray(dup, np.float32)
    lib().orc_restir_temporal(_p(ub), C.c_int(w), C.c_int(h), _p(np.ascontiguousarray(gcur, np.float32)),
                              _p(np.ascontiguousarray(gprev, np.float32)), _p(np.ascontiguousarray(res_b, np.uint32)),
                              _p(d), _p(out))
    return out


def restir_spatial(vox, bricks, masks, n, ubytes, w: int, h: int, gcur, res_a, direct, rad16=None, rad32=None,
                   pairing=None):
    """Spatial reuse + shading (reuse_spatial.wgsl).  Returns rad16, rad32,
    resB (next frame's history) and the visibility rays traced."""
    ub = np.frombuffer(ubytes, np.uint8).copy()
    rad16 = np.zeros((h, w, 4), np.uint16) if rad16 is None else np.array(rad16, np.uint16, copy=True)
    rad32 = np.zeros((h, w, 4), np.float32) if rad32 is None else np.array(rad32, np.float32, copy=True)
    res_b = np.zeros((h, w, 8), np.uint32)
    st = OrcStats()
    pr = None if pairing is None else np.ascontiguousarray(pairing, np.uint32)
    lib().orc_restir_spatial(_p(vox), _p(bricks), _p(masks), C.c_int(n), _p(ub), C.c_int(w), C.c_int(h),
                             _p(np.ascontiguousarray(gcur, np.float32)), _p(np.ascontiguousarray(res_a, np.uint32)),
                             _p(np.ascontiguousarray(direct, np.uint16)), _ptr_or_none(pr), _p(rad16), _p(rad32),
                             _p(res_b), C.byref(st))
    return {"rad16": rad16, "rad32": rad32, "resB": res_b,
            "stats": {k: int(getattr(st, k)) for k, _ in OrcStats._fields_}}


def restir_dupmap(w: int, h: int, res_b):
    """dupmap.wgsl: duplication score per pixel from reservoirs B."""
    out = np.zeros((h, w), np.float32)
    lib().orc_restir_dupmap(C.c_int(w), C.c_int(h), _p(np.ascontiguousarray(res_b, np.uint32)), _p(out))
    return out


def pairing_buffer(sigmas):
    """makePairingBuffer (pairing.js:80-89) for three sigmas."""
    sg = np.ascontiguousarray(sigmas, np.float64)
    out = np.zeros(PAIRING_WORDS, np.uint32)
    lib().orc_pairing_buffer(_p(sg), _p(out))
    return out


def restir_path(vox, bricks, masks, n, ubytes, fclamp, w, h, gprev, res_b_prev, dup_prev=None, lights=None,
                pairing=None):
    """The ReSTIR passes of one frame (main.js:736-741): initial -> temporal
    reuse (RF_TEMPORAL) -> spatial reuse -> duplication map (RF_DUPMAP).
    Returns every intermediate; "resA0" is A after the initial pass, "resA"
    after temporal reuse, "dup" the map this frame leaves for the next."""
    pt = restir_initial(vox, bricks, masks, n, ubytes, fclamp, w, h, lights)
    res = dict(pt)
    res["resA0"] = pt["resA"]
    flags = int(np.frombuffer(ubytes, np.uint32)[56])
    res_a = pt["resA"]
    if flags & 1 and flags & 2:
        res_a = restir_temporal(ubytes, w, h, pt["gbuf"], gprev, res_b_prev, res_a, dup_prev)
    res["resA"] = res_a
    sp = restir_spatial(vox, bricks, masks, n, ubytes, w, h, pt["gbuf"], res_a, pt["direct"], pt["rad16"], pt["rad32"],
                        pairing)
    res["rad16"], res["rad32"], res["resB"] = sp["rad16"], sp["rad32"], sp["resB"]
    res["dup"] = restir_dupmap(w, h, sp["resB"]) if flags & (16 | 131072) else dup_prev
    res["stats"] = dict(pt["stats"])
    for k in ("rays", "outer", "inner", "vreads"):
        res["stats"][k] += sp["stats"][k]
    return res


def frame(vox, bricks, masks, n, ubytes, fclamp, w, h, acc_prev, gprev, acc_f32=False, res_b_prev=None,
          dup_prev=None, lights=None, pairing=None):
    """One full oracle frame: pathtrace (or the ReSTIR passes when params2.x
    has RF_RESTIR; res_b_prev / dup_prev = the previous frame's reservoirs B
    and duplication map, lights / pairing as for restir_path) -> temporal ->
    a-trous x3 (if the denoise flag is set) -> present.  Returns every
    intermediate."""
    if int(np.frombuffer(ubytes, np.uint32)[56]) & 1:
        if res_b_prev is None:
            res_b_prev = np.zeros((h, w, 8), np.uint32)
        if dup_prev is None:
            dup_prev = np.zeros((h, w), np.float32)
        pt = restir_path(vox, bricks, masks, n, ubytes, fclamp, w, h, gprev, res_b_prev, dup_prev, lights, pairing)
    else:
        pt = pathtrace(vox, bricks, masks, n, ubytes, fclamp, w, h)
    flags = np.frombuffer(ubytes, np.uint32)[48 + 2]
    acc = temporal(ubytes, w, h, pt["rad16"], pt["gbuf"], acc_prev, gprev, acc_f32)
    res = dict(pt)
    res["accum"] = acc
    if flags & 2:
        d_a = atrous(w, h, acc, acc_f32, pt["gbuf"], 1)
        d_b = atrous(w, h, d_a, False, pt["gbuf"], 2)
        d_a2 = atrous(w, h, d_b, False, pt["gbuf"], 4)
        res["den"] = (d_a, d_b, d_a2)
        fin, fin_f32 = d_a2, False
    else:
        fin, fin_f32 = acc, acc_f32
    res["final"] = fin
    res["ldr"] = present(ubytes, w, h, fin, fin_f32, pt["alb8"])
    res["hdr"] = hdr(w, h, fin, fin_f32, pt["alb8"])
    return res


# ---------------------------------------------------------------------------
# Inputs of the plain-frame workload without the product library: the world
# (restated from scene.js), the benchmark camera path and the uniform block
# (main.js:399-426), so the CPU reference arm runs in a process that loads
# only oracle libraries.
# ---------------------------------------------------------------------------
def generate_scene(kind: int, n: int, seed: int):
    """kind 0: scene.js's world with noise seed `seed`; kind 2: the benchmark
    world.  Returns (voxels u32[n^3], spawn dict: pos, yaw, pitch, fov_y,
    near_z, far_z)."""
    vox = np.zeros(n * n * n, np.uint32)
    sp = np.zeros(8, np.float64)
    r = lib().orc_scene_generate(C.c_int(kind), C.c_int(n), C.c_uint32(seed), _p(vox), _p(sp))
    if r != 0:
        raise ValueError(f"orc_scene_generate: unsupported kind {kind} / size {n}")
    return vox, {"pos": (sp[0], sp[1], sp[2]), "yaw": sp[3], "pitch": sp[4], "fov_y": sp[5], "near_z": sp[6],
                 "far_z": sp[7]}


def camera_spline(spawn: dict, frame: int) -> dict:
    """The benchmark camera path: yaw advances 0.5 degree per frame and the
    camera moves 0.05 m per frame along its horizontal heading."""
    import math
    x, y, z = spawn["pos"]
    dyaw = 0.5 * math.pi / 180.0
    for f in range(frame):
        yaw = spawn["yaw"] + f * dyaw
        x += 0.05 * math.sin(yaw)
        z += 0.05 * math.cos(yaw)
    out = dict(spawn)
    out["pos"] = (x, y, z)
    out["yaw"] = spawn["yaw"] + frame * dyaw
    return out


def uniforms(pose: dict, prev: dict | None, frame: int, bounces: int, flags: int, w: int, h: int,
             exposure: float = 1.0, max_history: float = 64.0, sun_dir=(0.3, 0.8, 0.5),
             sun_cos_radius: float | None = None, sun_irradiance=(3.0, 3.0, 3.0), sky: float = 1.0) -> bytes:
    """The 304-byte uniform block of main.js writeUniforms (399-426) for the
    plain path (params2.x = 0, the reference's ReSTIR tuning defaults in the
    other slots)."""
    import math
    aspect = w / h

    def mats(p):
        return camera_matrices(p["pos"], p["yaw"], p["pitch"], p["fov_y"], aspect, p["near_z"], p["far_z"])

    vp, ivp = mats(pose)
    pvp = mats(prev)[0] if prev is not None else vp
    pp = prev if prev is not None else pose
    f = np.zeros(76, np.float32)
    u = f.view(np.uint32)
    f[0:16] = ivp
    f[16:32] = pvp
    f[32:35] = np.asarray(pose["pos"], np.float64).astype(np.float32)
    f[36:39] = np.asarray(pp["pos"], np.float64).astype(np.float32)
    sx, sy, sz = (float(np.float32(v)) for v in sun_dir)   # the host API carries the direction as f32
    sl = math.sqrt(sx * sx + sy * sy + sz * sz)
    f[40:43] = (sx / sl, sy / sl, sz / sl)
    f[43] = math.cos(math.radians(0.27)) if sun_cos_radius is None else sun_cos_radius
    f[44:47] = sun_irradiance
    f[47] = sky
    u[48], u[49], u[50] = frame & 0xFFFFFFFF, bounces, flags
    f[52], f[53], f[54] = w, h, exposure
    u[56], u[58] = 0, 3
    f[60:64] = (20.0, 1.0, 0.1, 0.0008)
    f[64:67] = (30.0, max_history, 24.0)
    f[68:72] = (48.0, 1.0, 1.0, 0.5)
    f[72] = 8.0
    return f.tobytes()
