// k_mlp.cu -- the radiance cache's BF16 tensor-core kernels (tcgen05, TMEM).
//
// This file starts with a GEMM self-test of the two operand forms the MLP
// uses: K-major A [128 x K] times K-major B [N x K] (forward and input
// gradients), and MN-major views of two row-chunked tiles X [128 x C],
// Y [128 x N] giving X^T Y (weight gradients).
#include <cuda_runtime.h>
#include <cstdint>
#include "umma.cuh"
#include "vrt_internal.h"

namespace vrt {

constexpr uint32_t kMbarSpin = 1u << 20;   // bounded mbarrier wait (iterations)

// mode 0: D[128 x N] = A[128 x K] * B[N x K]^T   (A, B row-major in global)
// mode 1: D[C x N]   = X[128 x C]^T * Y[128 x N] (rows 0..C-1 of the 128-row tile)
__global__ void __launch_bounds__(128, 1) k_umma_selftest(int mode, int K, int N, const uint16_t* __restrict__ A,
                                                          const uint16_t* __restrict__ B, float* __restrict__ D,
                                                          int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  // operand A at smem[0 .. 32 KB), operand B at smem[32 KB .. 64 KB); 4 KB slack after each
  uint8_t* sA = smem;
  uint8_t* sB = smem + 36 * 1024;
  if (warp == 0) umma::tmem_alloc(&tmem_base, 64);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  if (mode == 0) {
    for (int i = tid; i < 128 * K; i += 128) {
      const int r = i / K, c = i % K;
      *reinterpret_cast<uint16_t*>(sA + umma::canon_off(r, c, K)) = A[i];
    }
    for (int i = tid; i < N * K; i += 128) {
      const int r = i / K, c = i % K;
      *reinterpret_cast<uint16_t*>(sB + umma::canon_off(r, c, K)) = B[i];
    }
  } else {
    const int C = K;   // X has C columns
    for (int i = tid; i < 128 * C; i += 128) {
      const int r = i / C, c = i % C;
      *reinterpret_cast<uint16_t*>(sA + umma::canon_off(r, c, C)) = A[i];
    }
    for (int i = tid; i < 128 * N; i += 128) {
      const int r = i / N, c = i % N;
      *reinterpret_cast<uint16_t*>(sB + umma::canon_off(r, c, N)) = B[i];
    }
  }
  umma::fence_smem_to_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (tid == 0) {
    const uint32_t a0 = umma::smem_u32(sA), b0 = umma::smem_u32(sB);
    if (mode == 0) {
      const uint32_t id = umma::idesc_bf16(128, N, false, false);
      for (int ks = 0; ks < K / 16; ks++)
        umma::mma_bf16(tbase, umma::desc_kmajor(a0 + 256u * ks, K), umma::desc_kmajor(b0 + 256u * ks, K), id,
                       ks > 0 ? 1u : 0u);
    } else {
      const int C = K;
      const uint32_t id = umma::idesc_bf16(128, N, true, true);
      for (int ks = 0; ks < 128 / 16; ks++)
        umma::mma_bf16(tbase, umma::desc_mnmajor(a0 + 2u * 16u * C * ks, C),
                       umma::desc_mnmajor(b0 + 2u * 16u * N * ks, N), id, ks > 0 ? 1u : 0u);
    }
    umma::commit(&mbar);
  }
  const bool ok = __syncthreads_and(umma::mbar_wait(&mbar, 0, kMbarSpin) ? 1 : 0);
  umma::fence_after_sync();
  if (ok) {
    const int rows = mode == 0 ? 128 : K;
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      umma::tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (tid < rows)
        for (int j = 0; j < 16 && c0 + j < N; j++) D[(size_t)tid * N + c0 + j] = v[j];
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, 64);
}

}  // namespace vrt

using namespace vrt;

// Diagnostic of the tensor-core operand layouts (see k_umma_selftest).
extern "C" int vrt_mlp_selftest_gemm(int mode, int K, int N, const uint16_t* A, const uint16_t* B, float* D) {
  if (!A || !B || !D || (mode != 0 && mode != 1) || N < 16 || N > 64 || N % 16 || K < 16 || K > 128 || K % 16)
    return set_error(VRT_ERR_INVALID, "vrt_mlp_selftest_gemm: bad argument");
  const size_t na = (size_t)128 * K, nb = mode == 0 ? (size_t)N * K : (size_t)128 * N;
  const size_t nd = (size_t)128 * N;
  void* buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, (na + nb) * 2 + nd * 4 + 16);
  if (e != cudaSuccess) return set_error(VRT_ERR_OOM, cudaGetErrorString(e));
  uint16_t* dA = (uint16_t*)buf;
  uint16_t* dB = dA + na;
  float* dD = (float*)(dB + nb);
  int* dErr = (int*)(dD + nd);
  e = cudaMemcpy(dA, A, na * 2, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dB, B, nb * 2, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dD, 0, nd * 4 + 16);
  const int smem = 72 * 1024;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_umma_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) {
    k_umma_selftest<<<1, 128, smem>>>(mode, K, N, dA, dB, dD, dErr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&herr, dErr, 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(D, dD, nd * 4, cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) return set_error(VRT_ERR_CUDA, cudaGetErrorString(e));
  if (herr) return set_error(VRT_ERR_TIMEOUT, "vrt_mlp_selftest_gemm: tensor-core completion wait ran out");
  return VRT_OK;
}
