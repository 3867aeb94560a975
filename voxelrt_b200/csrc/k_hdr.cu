// k_hdr.cu -- HDR radiance of a frame accumulated in FP64 on the device, and
// squared errors against a reference image: the reference-image pipeline of
// the reference's benchmark (main.js:571-661 capture, test/bench.mjs
// reference accumulation) done on the GPU.
//
// The HDR value of a pixel is the capture's: demodulated radiance x (albedo
// byte / 255)^2, formed in double as ((double)rad * a) * a -- the same
// operations, in the same order, as the CPU oracle's orc_accumulate_f64, so
// the sums over a frame sequence are bit-identical to it.
#include "vrt_device.cuh"
#include "vrt_internal.h"

namespace vrt {

__device__ __forceinline__ double hdr_of(float rad, uint32_t alb, int c) {
  const double a = (double)((alb >> (8 * c)) & 0xffu) / 255.0;
  return ((double)rad * a) * a;
}

__global__ void __launch_bounds__(256) k_hdr_add(int P, const float4* __restrict__ rad32,
                                                 const uint32_t* __restrict__ alb8, double* __restrict__ acc) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const float4 r = __ldg(rad32 + p);
  const uint32_t a = __ldg(alb8 + p);
  acc[3 * (size_t)p + 0] += hdr_of(r.x, a, 0);
  acc[3 * (size_t)p + 1] += hdr_of(r.y, a, 1);
  acc[3 * (size_t)p + 2] += hdr_of(r.z, a, 2);
}

// Per-block partial sums of squared errors (fixed order within a block):
// mode 0: the last frame's HDR value against ref; mode 1: acc / count
// against ref.
__global__ void __launch_bounds__(256) k_hdr_sq_err(int P, int mode, const float4* __restrict__ rad32,
                                                    const uint32_t* __restrict__ alb8,
                                                    const double* __restrict__ acc, double inv_count,
                                                    const float* __restrict__ ref, double* __restrict__ part) {
  __shared__ double s[256];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (p < P) {
    for (int c = 0; c < 3; c++) {
      double v;
      if (mode == 0) {
        const float4 r = __ldg(rad32 + p);
        v = hdr_of(c == 0 ? r.x : (c == 1 ? r.y : r.z), __ldg(alb8 + p), c);
      } else {
        v = acc[3 * (size_t)p + c] * inv_count;
      }
      const double d = v - (double)__ldg(ref + 3 * (size_t)p + c);
      e += d * d;
    }
  }
  s[threadIdx.x] = e;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

int hdr_blocks(int P) { return (P + 255) / 256; }

cudaError_t launch_hdr_add(int P, const void* rad32, const uint32_t* alb8, double* acc, cudaStream_t st) {
  k_hdr_add<<<hdr_blocks(P), 256, 0, st>>>(P, (const float4*)rad32, alb8, acc);
  return cudaGetLastError();
}

cudaError_t launch_hdr_sq_err(int P, int mode, const void* rad32, const uint32_t* alb8, const double* acc,
                              double inv_count, const float* ref, double* part, cudaStream_t st) {
  k_hdr_sq_err<<<hdr_blocks(P), 256, 0, st>>>(P, mode, (const float4*)rad32, alb8, acc, inv_count, ref, part);
  return cudaGetLastError();
}

}  // namespace vrt
