// image_core.cuh -- per-pixel bodies of the image-space passes (temporal,
// a-trous, present), shared by the single-session kernels (k_image.cu) and the
// batched kernels (k_batch.cu).
#pragma once
#include "vrt_device.cuh"

namespace vrt {

VRT_DI float4 load_px(const void* base, bool f32, size_t p) {
  if (f32) return __ldg(reinterpret_cast<const float4*>(base) + p);
  return unpack_h4(__ldg(reinterpret_cast<const uint2*>(base) + p));
}

// temporal.wgsl:17-77 for pixel (gx, gy): reproject through prevViewProj,
// validate depth (8% + 2 cm) and normal (dot > 0.85), blend with the
// bilinearly fetched history (WebGPU linear filter: texel centres at +0.5,
// clamp to edge).  Returns (colour, history length).
VRT_DI float4 temporal_pixel(const Uni& u, int W, int H, int gx, int gy, const uint2* __restrict__ rad,
                             const float4* __restrict__ gcur, const void* __restrict__ accPrev, bool accF32,
                             const float4* __restrict__ gprev) {
  const size_t p = (size_t)gy * W + gx;
  const float4 c4 = unpack_h4(__ldg(rad + p));
  const float4 g = __ldg(gcur + p);
  const bool temporalOn = (u.params0[2] & 1u) != 0u;
  if (g.w < 0.0f || !temporalOn) return make_float4(c4.x, c4.y, c4.z, 1.0f);
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
        const float4 p00 = load_px(accPrev, accF32, (size_t)ya * W + xa);
        const float4 p10 = load_px(accPrev, accF32, (size_t)ya * W + xb);
        const float4 p01 = load_px(accPrev, accF32, (size_t)yb * W + xa);
        const float4 p11 = load_px(accPrev, accF32, (size_t)yb * W + xb);
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
  return make_float4(cx, cy, cz, history);
}

VRT_DI void store_px(void* base, bool f32, size_t p, float4 v) {
  if (f32) reinterpret_cast<float4*>(base)[p] = v;
  else reinterpret_cast<uint2*>(base)[p] = pack_h4(v.x, v.y, v.z, v.w);
}

// B3-spline taps (atrous.wgsl:26): 3/8, 1/4, 1/16 for |d| = 0, 1, 2.
VRT_DI float b3_weight(int d) { return d == 0 ? 0.375f : ((d == 1 || d == -1) ? 0.25f : 0.0625f); }

// atrous.wgsl:26-83 for pixel (px, py): 5x5 B3-spline taps at `step`,
// weights normal^32 * exp(-(|dt| / (0.05 t + 0.01) + |dL| / sigmaL)),
// sigmaL = max(0.08, 2/sqrt(max(history,1))); sky and out-of-image taps
// skipped.  The two exponentials are evaluated as one exp of the summed
// exponents with per-pixel reciprocals (within WGSL's accuracy for '/' and
// exp); taps of zero normal weight add nothing and are skipped.
VRT_DI float4 atrous_pixel(int W, int H, int px, int py, const void* __restrict__ src, bool srcF32,
                           const float4* __restrict__ gbuf, int step) {
  const size_t p = (size_t)py * W + px;
  const float4 center = load_px(src, srcF32, p);
  const float4 g = __ldg(gbuf + p);
  if (g.w < 0.0f) return center;
  const float history = fmax_(center.w, 1.0f);
  const float lumC = luminance(center.x, center.y, center.z);
  const float sigmaL = fmax_(0.08f, 2.0f / __fsqrt_rn(history));
  float sr = (center.x * 0.375f) * 0.375f;
  float sg = (center.y * 0.375f) * 0.375f;
  float sb = (center.z * 0.375f) * 0.375f;
  float wSum = 0.140625f;
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
      const float nd = fmax_(__fmaf_rn(g.z, gq.z, __fmaf_rn(g.y, gq.y, g.x * gq.x)), 0.0f);
      const float n2 = nd * nd, n4 = n2 * n2, n8 = n4 * n4, n16 = n8 * n8, n32 = n16 * n16;
      if (n32 == 0.0f) continue;
      const float4 cq = load_px(src, srcF32, q);
      const float wKernel = b3_weight(dx) * b3_weight(dy);
      const float e = exp_nonpos_(-__fmaf_rn(fabsf(g.w - gq.w), invD, fabsf(lumC - luminance(cq.x, cq.y, cq.z)) * invS));
      const float w = (wKernel * n32) * e;
      sr = __fmaf_rn(cq.x, w, sr);
      sg = __fmaf_rn(cq.y, w, sg);
      sb = __fmaf_rn(cq.z, w, sb);
      wSum = wSum + w;
    }
  }
  const float den = fmax_(wSum, 1e-6f);
  return make_float4(sr / den, sg / den, sb / den, center.w);
}

// (Accumulating (r, g) and (b, weight) as packed fp32 pairs left the
// iteration's instruction count and time unchanged, so the sums stay scalar.)
// atrous_pixel with the input staged in shared memory: sg = G-buffer tile,
// sc = source tile in fp32 with its luminance in .w, ci = this pixel's index
// in the tile (rows of RW pixels); taps outside the image hold zeros and
// drop out through their zero normal weight.  Same arithmetic in the same
// order as atrous_pixel.
VRT_DI float4 atrous_pixel_tile(float4 center, float4 g, const float4* sg, const float4* sc, int ci, int RW,
                                int step) {
  if (g.w < 0.0f) return center;
  const float history = fmax_(center.w, 1.0f);
  const float lumC = luminance(center.x, center.y, center.z);
  const float sigmaL = fmax_(0.08f, 2.0f / __fsqrt_rn(history));
  float sr = (center.x * 0.375f) * 0.375f;
  float sg_ = (center.y * 0.375f) * 0.375f;
  float sb = (center.z * 0.375f) * 0.375f;
  float wSum = 0.140625f;
  const float invD = 1.0f / (0.05f * g.w + 0.01f);
  const float invS = 1.0f / sigmaL;
#pragma unroll
  for (int dy = -2; dy <= 2; dy++) {
#pragma unroll
    for (int dx = -2; dx <= 2; dx++) {
      if (dx == 0 && dy == 0) continue;
      const int qi = ci + (dy * step) * RW + dx * step;
      const float4 gq = sg[qi];
      if (gq.w < 0.0f) continue;
      const float nd = fmax_(__fmaf_rn(g.z, gq.z, __fmaf_rn(g.y, gq.y, g.x * gq.x)), 0.0f);
      const float n2 = nd * nd, n4 = n2 * n2, n8 = n4 * n4, n16 = n8 * n8, n32 = n16 * n16;
      if (n32 == 0.0f) continue;
      const float4 cq = sc[qi];
      const float wKernel = b3_weight(dx) * b3_weight(dy);
      const float e = exp_nonpos_(-__fmaf_rn(fabsf(g.w - gq.w), invD, fabsf(lumC - cq.w) * invS));
      const float w = (wKernel * n32) * e;
      sr = __fmaf_rn(cq.x, w, sr);
      sg_ = __fmaf_rn(cq.y, w, sg_);
      sb = __fmaf_rn(cq.z, w, sb);
      wSum = wSum + w;
    }
  }
  const float den = fmax_(wSum, 1e-6f);
  return make_float4(sr / den, sg_ / den, sb / den, center.w);
}

// present.wgsl:40-55 for one channel: v = illum * sqrtAlb^2 * exposure ->
// ACES -> clamp -> pow(1/2.2) -> rgba8unorm code.
VRT_DI uint32_t present_code_exact(float v) {
  const float num = v * (2.51f * v + 0.03f);
  const float den = v * (2.43f * v + 0.59f) + 0.14f;
  const float t = clamp_(num / den, 0.0f, 1.0f);
  return unorm8_(pow_(t, 0.454545468f));
}

// Present lookup table (kPresentLut words per device context):
//   [0, 256)    the albedo factor sqrtAlb^2 of each rgba8 byte, (b / 255)^2 as
//               the shader forms it;
//   [256, 770)  (lo[k], hi[k]) pairs for k = 0..256: lo[k] = the least float of
//               [0, kPresentFastMax) whose exact code is >= k (inf if none;
//               non-decreasing in k); hi[k] = the float just above the
//               greatest v of the range whose exact code is < k (0 for k = 0);
// then scratch for the scan that builds them.  The exact code is almost but
// not quite non-decreasing in v: num / den rounds so that at 133 values next
// to a code step it drops back by one.  Every v >= hi[k] has a code >= k and
// every v < lo[k + 1] a code <= k, so outside the windows [lo[k], hi[k]) the
// code is the largest k with lo[k] <= v.
constexpr float kPresentFastMax = 8.0f;
constexpr uint32_t kPresentFastMaxBits = 0x41000000u;   // bit pattern of kPresentFastMax
constexpr int kPresentLoHi = 256;                        // float offset of the (lo, hi) pairs

// present_code_exact out of line, for the table path's rare fallbacks (keeps
// the unrolled per-pixel code small).
static __device__ __noinline__ uint32_t present_code_slow(float v) { return present_code_exact(v); }

// Approximate x^(1/2.2) for the code estimate: the hardware's log2 and exp2
// with denormal inputs and results flushed to zero (a flushed estimate only
// starts the table search elsewhere; the table decides the code).
VRT_DI float present_gamma_estimate(float x) {
  float l, r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(x));
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(l * 0.454545468f));
  return r;
}

// present_code_exact(v) through the table: the code is the largest k with
// lo[k] <= v unless v lies in that code's window [lo[k], hi[k]).  An estimate
// c0 from the hardware's approximate reciprocal / log2 / exp2, held to
// [1, 254], is within one code of the answer; the table entries c0 - 1 .. c0 + 2
// are read at once (no chain of dependent loads), and the answer is c0 - 1, c0
// or c0 + 1.  Values whose code is further from the estimate, values in a
// window, values outside [0, kPresentFastMax) and NaN take the exact
// arithmetic.
VRT_DI uint32_t present_code(float v, const float* __restrict__ lut) {
  if (!(v >= 0.0f && v < kPresentFastMax)) return present_code_slow(v);
  const float2* lh = reinterpret_cast<const float2*>(lut + kPresentLoHi);
  const float num = v * __fmaf_rn(2.51f, v, 0.03f);
  const float den = __fmaf_rn(v, __fmaf_rn(2.43f, v, 0.59f), 0.14f);
  float rden;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rden) : "f"(den));
  const float t = fminf(fmaxf(num * rden, 0.0f), 1.0f);
  const int c0 = min(max(__float2int_rn(255.0f * present_gamma_estimate(t)), 1), 254);
  const float2 em = __ldg(lh + c0 - 1), e0 = __ldg(lh + c0), e1 = __ldg(lh + c0 + 1);
  const float l2 = __ldg(lut + kPresentLoHi + 2 * (c0 + 2));
  int c = c0;
  float h = e0.y;
  bool far = false;
  if (v < e0.x) { c = c0 - 1; h = em.y; far = v < em.x; }
  else if (v >= e1.x) { c = c0 + 1; h = e1.y; far = v >= l2; }
  if (far || v < h) return present_code_slow(v);
  return (uint32_t)c;
}

// present.wgsl:40-55 for one pixel with the context's lookup table.
VRT_DI uint32_t present_pixel(float exposure, float4 il, uint32_t a, const float* __restrict__ lut) {
  const float iv[3] = {il.x, il.y, il.z};
  uint32_t outw = 255u << 24;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float v = (iv[c] * __ldg(lut + ((a >> (8 * c)) & 0xffu))) * exposure;
    outw |= present_code(v, lut) << (8 * c);
  }
  return outw;
}

}  // namespace vrt
