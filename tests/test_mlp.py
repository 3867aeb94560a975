"""Radiance-cache tensor-core kernels: operand layouts (GEMM self-test),
network forward/backward against an fp64 CPU restatement, training."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def to_bf16(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def from_bf16(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("mode,K,N", [(0, 16, 16), (0, 64, 64), (0, 80, 64), (0, 64, 16), (0, 128, 32),
                                      (1, 64, 64), (1, 80, 64), (1, 64, 16), (1, 128, 16)])
def test_umma_gemm_layouts(vrt, mode, K, N):
    import ctypes as C
    rng = np.random.default_rng(K * 7 + N + mode)
    A = to_bf16(rng.normal(size=(128, K)))
    B = to_bf16(rng.normal(size=(N, K) if mode == 0 else (128, N)))
    D = np.zeros((128, N), np.float32)
    code = vrt.lib.vrt_mlp_selftest_gemm(mode, K, N, C.c_void_p(A.ctypes.data), C.c_void_p(B.ctypes.data),
                                         C.c_void_p(D.ctypes.data))
    assert code == 0, vrt.lib.vrt_last_error_string().decode()
    a, b = from_bf16(A).astype(np.float64), from_bf16(B).astype(np.float64)
    ref = a @ b.T if mode == 0 else a.T @ b
    rows = 128 if mode == 0 else K
    err = np.abs(D[:rows] - ref) / (np.abs(ref) + 1.0)
    assert err.max() < 1e-5, f"max err {err.max()}"
