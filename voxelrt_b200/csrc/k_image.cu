// k_image.cu -- image-space passes (temporal, a-trous, present) and the
// brick/mask builders of the voxel world, for sm_100a.
//
// The image passes are HBM/L2-bound gathers: one thread per pixel in 32x8
// blocks (a warp reads 32 consecutive pixels of a row = 256 B of rgba16f or
// 512 B of rgba32f per request).
#include "vrt_device.cuh"
#include "image_core.cuh"
#include "vrt_internal.h"
#include <cstring>

namespace vrt {

// ---------------------------------------------------------------------------
// temporal.wgsl:17-77 -- reproject through prevViewProj, validate depth
// (8% + 2 cm) and normal (dot > 0.85), blend with the bilinearly fetched
// history (WebGPU linear filter: texel centres at +0.5, clamp to edge).
// ---------------------------------------------------------------------------
template <bool kAccF32>
__global__ void __launch_bounds__(256) k_temporal(Uni u, int W, int H, const uint2* __restrict__ rad,
                                                  const float4* __restrict__ gcur, const void* __restrict__ accPrev,
                                                  const float4* __restrict__ gprev, void* __restrict__ accOut) {
  const int gx = blockIdx.x * 32 + (threadIdx.x & 31);
  const int gy = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (gx >= W || gy >= H) return;
  const float4 res = temporal_pixel(u, W, H, gx, gy, rad, gcur, accPrev, kAccF32, gprev);
  store_px(accOut, kAccF32, (size_t)gy * W + gx, res);
}

// atrous.wgsl:26-83, one iteration at `step` (body in image_core.cuh).
template <bool kSrcF32>
__global__ void __launch_bounds__(256) k_atrous(int W, int H, const void* __restrict__ src,
                                                const float4* __restrict__ gbuf, uint2* __restrict__ dst, int step) {
  const int px = blockIdx.x * 32 + (threadIdx.x & 31);
  const int py = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (px >= W || py >= H) return;
  const float4 v = atrous_pixel(W, H, px, py, src, kSrcF32, gbuf, step);
  dst[(size_t)py * W + px] = pack_h4(v.x, v.y, v.z, v.w);
}

// present.wgsl:40-55 as a compute pass writing a headless rgba8 buffer.  The
// pass is per pixel and the buffers are dense, so each of the first n4
// threads takes four consecutive pixels with 16-byte loads and stores; the
// threads after them take the remaining P - 4 n4 pixels one each (n4 = 0
// when a buffer is not 16-byte aligned).
template <bool kFinF32>
__global__ void __launch_bounds__(256) k_present(float exposure, uint32_t P, uint32_t n4,
                                                 const void* __restrict__ fin, const uint32_t* __restrict__ alb8,
                                                 uint32_t* __restrict__ ldr, const float* __restrict__ lut) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n4) {
    float4 il[4];
    if (kFinF32) {
      const float4* f = reinterpret_cast<const float4*>(fin) + 4u * (size_t)i;
#pragma unroll
      for (int k = 0; k < 4; k++) il[k] = __ldg(f + k);
    } else {
      const uint4* f = reinterpret_cast<const uint4*>(fin) + 2u * (size_t)i;
      const uint4 a = __ldg(f), b = __ldg(f + 1);
      il[0] = unpack_h4(make_uint2(a.x, a.y));
      il[1] = unpack_h4(make_uint2(a.z, a.w));
      il[2] = unpack_h4(make_uint2(b.x, b.y));
      il[3] = unpack_h4(make_uint2(b.z, b.w));
    }
    const uint4 al = __ldg(reinterpret_cast<const uint4*>(alb8) + i);
    uint4 o;
    o.x = present_pixel(exposure, il[0], al.x, lut);
    o.y = present_pixel(exposure, il[1], al.y, lut);
    o.z = present_pixel(exposure, il[2], al.z, lut);
    o.w = present_pixel(exposure, il[3], al.w, lut);
    reinterpret_cast<uint4*>(ldr)[i] = o;
  } else {
    const size_t p = 4u * (size_t)n4 + (i - n4);
    if (p >= P) return;
    ldr[p] = present_pixel(exposure, load_px(fin, kFinF32, p), __ldg(alb8 + p), lut);
  }
}

// Building the present lookup table (image_core.cuh), step 1: every float of
// [0, kPresentFastMax) through the exact arithmetic.  A thread walks a run of
// kPresentScanRun consecutive bit patterns (ordered like the values they
// encode) and, per stretch of equal codes, lowers the code's least bit
// pattern (minb) and raises one past its greatest (maxb; 0: code not seen).
constexpr uint32_t kPresentScanRun = 4096u;
__global__ void __launch_bounds__(256) k_present_scan(unsigned int* __restrict__ minb, unsigned int* __restrict__ maxb) {
  const uint32_t end = kPresentFastMaxBits;
  const uint32_t b0 = (blockIdx.x * blockDim.x + threadIdx.x) * kPresentScanRun;
  if (b0 >= end) return;
  const uint32_t b1 = min(end, b0 + kPresentScanRun);
  uint32_t code = present_code_exact(__uint_as_float(b0)), start = b0;
  for (uint32_t b = b0 + 1u; b < b1; b++) {
    const uint32_t c = present_code_exact(__uint_as_float(b));
    if (c != code) {
      atomicMin(minb + code, start);
      atomicMax(maxb + code, b);
      code = c;
      start = b;
    }
  }
  atomicMin(minb + code, start);
  atomicMax(maxb + code, b1);
}

// Step 2 (256 threads): thread k forms the albedo factor of byte k, lo[k] as
// the least bit pattern of any code >= k and hi[k] as one above the greatest
// bit pattern of any code < k.  maxb holds one past a code's greatest bit
// pattern, so the "not seen" 0 drops out of the maximum.
__global__ void __launch_bounds__(256) k_present_lut(float* __restrict__ lut, const unsigned int* __restrict__ minb,
                                                     const unsigned int* __restrict__ maxb) {
  const int k = threadIdx.x;
  const float as = (float)k / 255.0f;
  lut[k] = as * as;
  uint32_t lo = 0x7f800000u;                       // inf: no code >= k in the range
  for (int c = k; c < 256; c++)
    if (minb[c] < kPresentFastMaxBits) lo = min(lo, minb[c]);
  uint32_t hi = 0u;                                // 0.0f: no code < k in the range
  for (int c = 0; c < k; c++) hi = max(hi, maxb[c]);
  lut[kPresentLoHi + 2 * k] = __uint_as_float(lo);
  lut[kPresentLoHi + 2 * k + 1] = __uint_as_float(hi);
  if (k == 0) {
    lut[kPresentLoHi + 2 * 256] = __int_as_float(0x7f800000);
    uint32_t h = 0u;
    for (int c = 0; c < 256; c++) h = max(h, maxb[c]);
    lut[kPresentLoHi + 2 * 256 + 1] = __uint_as_float(h);
  }
}

// Every float of [0, kPresentFastMax) through present_code and
// present_code_exact; counts the values where they differ and keeps the
// smallest such bit pattern.
__global__ void __launch_bounds__(256) k_present_check(const float* __restrict__ lut, unsigned long long* __restrict__ bad,
                                                       unsigned int* __restrict__ first) {
  const uint32_t end = __float_as_uint(kPresentFastMax);
  unsigned long long n = 0;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < end; b += gridDim.x * blockDim.x) {
    const float v = __uint_as_float(b);
    if (present_code(v, lut) != present_code_exact(v)) {
      n++;
      atomicMin(first, b);
    }
  }
  if (n) atomicAdd(bad, n);
}

// ---------------------------------------------------------------------------
// Brick build (scene.js:411-433): one block per brick, one warp per mask
// word.  Word w holds bits 32w..32w+31 = lz = w/2, ly = 4(w&1) + lane/8,
// lx = lane%8, so a warp ballot over "voxel != 0" is the word itself.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_build_bricks(const uint32_t* __restrict__ vox, int N, int BG,
                                                      uint32_t* __restrict__ bricks, uint32_t* __restrict__ masks,
                                                      int bx0, int by0, int bz0, int nbx, int nby) {
  const int lb = blockIdx.x;
  const int bx = bx0 + lb % nbx;
  const int by = by0 + (lb / nbx) % nby;
  const int bz = bz0 + lb / (nbx * nby);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lx = lane & 7, ly = 4 * (w & 1) + (lane >> 3), lz = w >> 1;
  const size_t x = (size_t)bx * 8 + lx, y = (size_t)by * 8 + ly, z = (size_t)bz * 8 + lz;
  const uint32_t v = vox[x + y * N + z * (size_t)N * N];
  const uint32_t word = __ballot_sync(0xffffffffu, v != 0u);
  const size_t bi = (size_t)bx + (size_t)by * BG + (size_t)bz * BG * BG;
  if (lane == 0) masks[bi * 16 + w] = word;
  const int occ = __syncthreads_or(word != 0u);
  if (threadIdx.x == 0) bricks[bi] = occ ? 1u : 0u;
}

// Occupancy bitmap: bit bi = bricks[bi] != 0.
__global__ void k_build_bits(const uint32_t* __restrict__ bricks, int nb, uint32_t* __restrict__ bits) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool occ = i < nb && bricks[i] != 0u;
  const uint32_t word = __ballot_sync(0xffffffffu, occ);
  if ((threadIdx.x & 31) == 0 && i < ((nb + 31) & ~31)) bits[i >> 5] = word;
}

__global__ void k_fill_box(uint32_t* __restrict__ vox, int N, int x0, int y0, int z0, int sx, int sy, int sz,
                           uint32_t value) {
  const size_t n = (size_t)sx * sy * sz;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t x = x0 + i % sx, y = y0 + (i / sx) % sy, z = z0 + i / ((size_t)sx * sy);
    vox[x + y * N + z * (size_t)N * N] = value;
  }
}

// ---------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------
static Uni to_uni(const VrtUniforms& u) {
  Uni r;
  std::memcpy(&r, &u, sizeof(Uni));
  return r;
}

cudaError_t launch_build_bricks(const SceneDev& s, int bx0, int by0, int bz0, int bx1, int by1, int bz1,
                                cudaStream_t st) {
  const int nbx = bx1 - bx0 + 1, nby = by1 - by0 + 1, nbz = bz1 - bz0 + 1;
  if (nbx <= 0 || nby <= 0 || nbz <= 0) return cudaSuccess;
  const long nblocks = (long)nbx * nby * nbz;
  k_build_bricks<<<(unsigned)nblocks, 512, 0, st>>>(s.vox, s.N, s.BG, s.bricks, s.masks, bx0, by0, bz0, nbx, nby);
  return cudaGetLastError();
}

cudaError_t launch_build_bits(const SceneDev& s, cudaStream_t st) {
  const int nb = s.BG * s.BG * s.BG;
  k_build_bits<<<(nb + 255) / 256, 256, 0, st>>>(s.bricks, nb, s.bits);
  return cudaGetLastError();
}

cudaError_t launch_fill_box(const SceneDev& s, int x0, int y0, int z0, int x1, int y1, int z1, uint32_t value,
                            cudaStream_t st) {
  const int sx = x1 - x0 + 1, sy = y1 - y0 + 1, sz = z1 - z0 + 1;
  const size_t n = (size_t)sx * sy * sz;
  const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_fill_box<<<blocks, 256, 0, st>>>(s.vox, s.N, x0, y0, z0, sx, sy, sz, value);
  return cudaGetLastError();
}

cudaError_t launch_temporal(const VrtUniforms& u, int W, int H, const void* rad16, const void* gcur,
                            const void* acc_prev, const void* gprev, void* acc_out, bool acc_f32, cudaStream_t st) {
  dim3 grid((W + 31) / 32, (H + 7) / 8);
  if (acc_f32)
    k_temporal<true><<<grid, 256, 0, st>>>(to_uni(u), W, H, (const uint2*)rad16, (const float4*)gcur, acc_prev,
                                          (const float4*)gprev, acc_out);
  else
    k_temporal<false><<<grid, 256, 0, st>>>(to_uni(u), W, H, (const uint2*)rad16, (const float4*)gcur, acc_prev,
                                           (const float4*)gprev, acc_out);
  return cudaGetLastError();
}

cudaError_t launch_atrous(int W, int H, const void* src, bool src_f32, const void* gbuf, void* dst, int step,
                          cudaStream_t st) {
  dim3 grid((W + 31) / 32, (H + 7) / 8);
  if (src_f32) k_atrous<true><<<grid, 256, 0, st>>>(W, H, src, (const float4*)gbuf, (uint2*)dst, step);
  else k_atrous<false><<<grid, 256, 0, st>>>(W, H, src, (const float4*)gbuf, (uint2*)dst, step);
  return cudaGetLastError();
}

cudaError_t launch_present(const VrtUniforms& u, int W, int H, const void* fin, bool fin_f32,
                           const uint32_t* alb8, uint32_t* ldr, const float* lut, cudaStream_t st) {
  const uint32_t P = (uint32_t)W * (uint32_t)H;
  const bool aligned = ((reinterpret_cast<uintptr_t>(fin) | reinterpret_cast<uintptr_t>(alb8) |
                         reinterpret_cast<uintptr_t>(ldr)) & 15u) == 0u;
  const uint32_t n4 = aligned ? P >> 2 : 0u;
  const uint32_t threads = n4 + (P - 4u * n4);
  const unsigned blocks = (threads + 255u) / 256u;
  if (fin_f32) k_present<true><<<blocks, 256, 0, st>>>(u.params1[2], P, n4, fin, alb8, ldr, lut);
  else k_present<false><<<blocks, 256, 0, st>>>(u.params1[2], P, n4, fin, alb8, ldr, lut);
  return cudaGetLastError();
}

cudaError_t launch_present_lut(float* lut, cudaStream_t st) {
  unsigned int* minb = reinterpret_cast<unsigned int*>(lut + kPresentLoHi + 2 * 257);
  unsigned int* maxb = minb + 256;
  cudaError_t e = cudaMemsetAsync(minb, 0x7f, 256 * sizeof(unsigned int), st);   // 0x7f7f7f7f: "none"
  if (e == cudaSuccess) e = cudaMemsetAsync(maxb, 0, 256 * sizeof(unsigned int), st);     // "not seen"
  if (e != cudaSuccess) return e;
  const uint32_t runs = (kPresentFastMaxBits + kPresentScanRun - 1u) / kPresentScanRun;
  k_present_scan<<<(runs + 255u) / 256u, 256, 0, st>>>(minb, maxb);
  k_present_lut<<<1, 256, 0, st>>>(lut, minb, maxb);
  return cudaGetLastError();
}

cudaError_t launch_present_check(const float* lut, unsigned long long* bad, unsigned int* first, cudaStream_t st) {
  k_present_check<<<148 * 8, 256, 0, st>>>(lut, bad, first);
  return cudaGetLastError();
}

}  // namespace vrt
