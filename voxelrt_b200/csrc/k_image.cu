// k_image.cu -- image-space passes (temporal, a-trous, present) and the
// brick/mask builders of the voxel world, for sm_100a.
//
// The image passes are HBM/L2-bound gathers: one thread per pixel in 32x8
// blocks (a warp reads 32 consecutive pixels of a row = 256 B of rgba16f or
// 512 B of rgba32f per request).
#include "vrt_device.cuh"
#include "vrt_internal.h"
#include <cstring>

namespace vrt {

VRT_DI float4 load_px(const void* base, bool f32, size_t p) {
  if (f32) return __ldg(reinterpret_cast<const float4*>(base) + p);
  return unpack_h4(__ldg(reinterpret_cast<const uint2*>(base) + p));
}

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
  const size_t p = (size_t)gy * W + gx;
  const float4 c4 = unpack_h4(__ldg(rad + p));
  const float4 g = __ldg(gcur + p);
  const bool temporalOn = (u.params0[2] & 1u) != 0u;
  float4 res;
  if (g.w < 0.0f || !temporalOn) {
    res = make_float4(c4.x, c4.y, c4.z, 1.0f);
  } else {
    const float uvx = ((float)gx + 0.5f) / (float)W;
    const float uvy = ((float)gy + 0.5f) / (float)H;
    const F3 cr = camera_ray(u, uvx, uvy);
    const F3 wp = f3(u.camPos[0], u.camPos[1], u.camPos[2]) + cr * g.w;
    float pc[4];
    matvec4(u.prevViewProj, wp.x, wp.y, wp.z, 1.0f, pc);
    float cx = c4.x, cy = c4.y, cz = c4.z, history = 1.0f;
    if (pc[3] > 0.0f) {
      const float ndx = pc[0] / pc[3], ndy = pc[1] / pc[3];
      const float pux = ndx * 0.5f + 0.5f;
      const float puy = (-ndy) * 0.5f + 0.5f;
      if (pux > 0.0f && puy > 0.0f && pux < 1.0f && puy < 1.0f) {
        const int ppx = min((int)(pux * (float)W), W - 1), ppy = min((int)(puy * (float)H), H - 1);
        const float4 pg = __ldg(gprev + ((size_t)ppy * W + ppx));
        const F3 dv = wp - f3(u.prevCamPos[0], u.prevCamPos[1], u.prevCamPos[2]);
        const float expectedT = __fsqrt_rn(dot3(dv, dv));
        const bool depthOk = pg.w > 0.0f && fabsf(pg.w - expectedT) < 0.08f * expectedT + 0.02f;
        const bool normalOk = ((pg.x * g.x + pg.y * g.y) + pg.z * g.z) > 0.85f;
        if (depthOk && normalOk) {
          const float tx = pux * (float)W - 0.5f, ty = puy * (float)H - 0.5f;
          const float fx0 = floorf(tx), fy0 = floorf(ty);
          const float ax = tx - fx0, ay = ty - fy0;
          const int x0 = (int)fx0, y0 = (int)fy0;
          const int xa = iclamp_(x0, 0, W - 1), xb = iclamp_(x0 + 1, 0, W - 1);
          const int ya = iclamp_(y0, 0, H - 1), yb = iclamp_(y0 + 1, 0, H - 1);
          const float4 p00 = load_px(accPrev, kAccF32, (size_t)ya * W + xa);
          const float4 p10 = load_px(accPrev, kAccF32, (size_t)ya * W + xb);
          const float4 p01 = load_px(accPrev, kAccF32, (size_t)yb * W + xa);
          const float4 p11 = load_px(accPrev, kAccF32, (size_t)yb * W + xb);
          const float bx = 1.0f - ax, by = 1.0f - ay;
          float pr[4];
          pr[0] = (p00.x * bx + p10.x * ax) * by + (p01.x * bx + p11.x * ax) * ay;
          pr[1] = (p00.y * bx + p10.y * ax) * by + (p01.y * bx + p11.y * ax) * ay;
          pr[2] = (p00.z * bx + p10.z * ax) * by + (p01.z * bx + p11.z * ax) * ay;
          pr[3] = (p00.w * bx + p10.w * ax) * by + (p01.w * bx + p11.w * ax) * ay;
          history = fmin_(pr[3], u.params4[1]) + 1.0f;
          const float alpha = 1.0f / history;
          cx = mix_(pr[0], c4.x, alpha);
          cy = mix_(pr[1], c4.y, alpha);
          cz = mix_(pr[2], c4.z, alpha);
        }
      }
    }
    res = make_float4(cx, cy, cz, history);
  }
  if (kAccF32) reinterpret_cast<float4*>(accOut)[p] = res;
  else reinterpret_cast<uint2*>(accOut)[p] = pack_h4(res.x, res.y, res.z, res.w);
}

// ---------------------------------------------------------------------------
// atrous.wgsl:26-83 -- 5x5 B3-spline taps at `step`, weights
// normal^32 * exp(-|dt|/(0.05 t + 0.01)) * exp(-|dL|/sigmaL),
// sigmaL = max(0.08, 2/sqrt(max(history,1))); sky and out-of-image taps skipped.
// ---------------------------------------------------------------------------
// B3-spline taps (atrous.wgsl:26): 3/8, 1/4, 1/16 for |d| = 0, 1, 2.
VRT_DI float b3_weight(int d) { return d == 0 ? 0.375f : ((d == 1 || d == -1) ? 0.25f : 0.0625f); }

template <bool kSrcF32>
__global__ void __launch_bounds__(256) k_atrous(int W, int H, const void* __restrict__ src,
                                                const float4* __restrict__ gbuf, uint2* __restrict__ dst, int step) {
  const int px = blockIdx.x * 32 + (threadIdx.x & 31);
  const int py = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (px >= W || py >= H) return;
  const size_t p = (size_t)py * W + px;
  const float4 center = load_px(src, kSrcF32, p);
  const float4 g = __ldg(gbuf + p);
  if (g.w < 0.0f) {
    dst[p] = pack_h4(center.x, center.y, center.z, center.w);
    return;
  }
  const float history = fmax_(center.w, 1.0f);
  const float lumC = luminance(center.x, center.y, center.z);
  const float sigmaL = fmax_(0.08f, 2.0f / __fsqrt_rn(history));
  float sr = (center.x * 0.375f) * 0.375f;
  float sg = (center.y * 0.375f) * 0.375f;
  float sb = (center.z * 0.375f) * 0.375f;
  float wSum = 0.140625f;
  // exp(-|dt|/(0.05 t + 0.01)) * exp(-|dL|/sigmaL) as one exp of the summed
  // exponents with per-pixel reciprocals (within WGSL's '/' and exp accuracy).
  const float invD = 1.0f / (0.05f * g.w + 0.01f);
  const float invS = 1.0f / sigmaL;
#pragma unroll
  for (int dy = -2; dy <= 2; dy++) {
#pragma unroll
    for (int dx = -2; dx <= 2; dx++) {
      if (dx == 0 && dy == 0) continue;
      const int qx = px + dx * step, qy = py + dy * step;
      if (qx < 0 || qy < 0 || qx >= W || qy >= H) continue;
      const size_t q = (size_t)qy * W + qx;
      const float4 gq = __ldg(gbuf + q);
      if (gq.w < 0.0f) continue;
      const float nd = fmax_((g.x * gq.x + g.y * gq.y) + g.z * gq.z, 0.0f);
      const float n2 = nd * nd, n4 = n2 * n2, n8 = n4 * n4, n16 = n8 * n8, n32 = n16 * n16;
      if (n32 == 0.0f) continue;
      const float4 cq = load_px(src, kSrcF32, q);
      const float wKernel = b3_weight(dx) * b3_weight(dy);
      const float e = exp_(-(fabsf(g.w - gq.w) * invD + fabsf(lumC - luminance(cq.x, cq.y, cq.z)) * invS));
      const float w = (wKernel * n32) * e;
      sr = sr + cq.x * w;
      sg = sg + cq.y * w;
      sb = sb + cq.z * w;
      wSum = wSum + w;
    }
  }
  const float den = fmax_(wSum, 1e-6f);
  dst[p] = pack_h4(sr / den, sg / den, sb / den, center.w);
}

// ---------------------------------------------------------------------------
// present.wgsl:40-55 as a compute pass writing a headless rgba8 buffer:
// illum * sqrtAlb^2 * exposure -> ACES -> pow(1/2.2).
// ---------------------------------------------------------------------------
template <bool kFinF32>
__global__ void __launch_bounds__(256) k_present(float exposure, int W, int H, const void* __restrict__ fin,
                                                 const uint32_t* __restrict__ alb8, uint32_t* __restrict__ ldr) {
  const int x = blockIdx.x * 32 + (threadIdx.x & 31);
  const int y = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (x >= W || y >= H) return;
  const size_t p = (size_t)y * W + x;
  const float4 il = load_px(fin, kFinF32, p);
  const uint32_t a = __ldg(alb8 + p);
  const float iv[3] = {il.x, il.y, il.z};
  uint32_t outw = 255u << 24;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float as = (float)((a >> (8 * c)) & 0xffu) / 255.0f;
    const float v = (iv[c] * (as * as)) * exposure;
    const float num = v * (2.51f * v + 0.03f);
    const float den = v * (2.43f * v + 0.59f) + 0.14f;
    const float t = clamp_(num / den, 0.0f, 1.0f);
    outw |= unorm8_(pow_(t, 0.454545468f)) << (8 * c);
  }
  ldr[p] = outw;
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
                           const uint32_t* alb8, uint32_t* ldr, cudaStream_t st) {
  dim3 grid((W + 31) / 32, (H + 7) / 8);
  if (fin_f32) k_present<true><<<grid, 256, 0, st>>>(u.params1[2], W, H, fin, alb8, ldr);
  else k_present<false><<<grid, 256, 0, st>>>(u.params1[2], W, H, fin, alb8, ldr);
  return cudaGetLastError();
}

}  // namespace vrt
