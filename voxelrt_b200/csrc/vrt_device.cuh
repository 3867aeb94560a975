// vrt_device.cuh -- device-side building blocks of the plain GI path.
//
// Every routine here states the reference computation it implements; the
// arithmetic is written as single IEEE binary32 operations in the order the
// WGSL expresses them.  Files including this header are compiled with
// -fmad=false (no contraction), -prec-div=true, -prec-sqrt=true, -ftz=false,
// which makes the results bit-identical to a scalar IEEE evaluation of the
// same expressions on the host.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>

#define VRT_DI __device__ __forceinline__

namespace vrt {

// ---------------------------------------------------------------------------
// Constants (common.wgsl:7-11, scene.js:5-6)
// ---------------------------------------------------------------------------
constexpr float kPi = 3.14159274f;          // f32(3.14159265358979)
constexpr float kTwoPi = 6.28318548f;       // f32(2 * 3.14159265358979)
constexpr float kInvPi = 0.318309873f;      // f32(0.31830988618)
constexpr float kVoxelSize = 0.0625f;       // 1/16 m
constexpr float kInvVoxel = 16.0f;
constexpr int kBrick = 8;
constexpr float kEmissiveScale = 24.0f;

// Uniform block, same layout as VrtUniforms / common.wgsl:13-35.
struct Uni {
  float invViewProj[16], prevViewProj[16];
  float camPos[4], prevCamPos[4], sunDir[4], sunRadiance[4];
  uint32_t params0[4];
  float params1[4];
  uint32_t params2[4];
  float params3[4], params4[4], params5[4], params6[4];
};
static_assert(sizeof(Uni) == 304, "uniform block is 304 bytes");

// ---------------------------------------------------------------------------
// Scalar helpers.  min/max are written as selects so that signed zeros and
// NaNs resolve the same way on every backend.
// ---------------------------------------------------------------------------
VRT_DI float fmin_(float a, float b) { return b < a ? b : a; }
VRT_DI float fmax_(float a, float b) { return a < b ? b : a; }
VRT_DI float clamp_(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
VRT_DI float mix_(float a, float b, float t) { return a * (1.0f - t) + b * t; }
VRT_DI int iclamp_(int x, int lo, int hi) { return min(max(x, lo), hi); }
// floor to int with saturation (NaN -> 0): cvt.rmi.s32.f32.
VRT_DI int ifloor_(float x) { return __float2int_rd(x); }

// safeInv (voxel.wgsl:65-71): sg / max(|v|, 1e-8) with sg = +-1, evaluated as
// sg times the correctly rounded reciprocal (__frcp_rn, IEEE round to
// nearest): multiplying by +-1 is exact, so the value equals the IEEE
// quotient for every input, NaN and infinity included.
VRT_DI float safe_inv(float sg, float v) { return sg * __frcp_rn(fmax_(fabsf(v), 1e-8f)); }

struct F3 { float x, y, z; };
VRT_DI F3 f3(float x, float y, float z) { return F3{x, y, z}; }
VRT_DI F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
VRT_DI F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
VRT_DI F3 operator*(F3 a, F3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
VRT_DI F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
VRT_DI float dot3(F3 a, F3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
VRT_DI F3 cross3(F3 a, F3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
VRT_DI F3 normalize3(F3 a) {
  float l = __fsqrt_rn(dot3(a, a));
  return f3(a.x / l, a.y / l, a.z / l);
}
VRT_DI F3 min3(F3 a, F3 b) { return f3(fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)); }
VRT_DI F3 max3(F3 a, F3 b) { return f3(fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)); }
VRT_DI F3 mix3(F3 a, F3 b, float t) { return f3(mix_(a.x, b.x, t), mix_(a.y, b.y, t), mix_(a.z, b.z, t)); }

// ---------------------------------------------------------------------------
// Project transcendentals.  WGSL leaves sin/cos/exp/pow precision to the
// implementation; this project defines them as:
//   sincos: quadrant k = floor(x*2/pi + 0.5), remainder r = (x - k*201/128)
//           - k*PIO2_LO, Taylor series of sin to r^9 and of cos to r^10.
//   exp:    k = floor(x*log2(e) + 0.5), r = (x - k*LN2_HI) - k*LN2_LO,
//           e^r by its Taylor series to r^7, scaled by 2^k.
//   log2:   x = m*2^e, m in [sqrt(1/2), sqrt(2)], log2 m = (2/ln 2)*atanh(s)
//           with s = (m-1)/(m+1) and atanh by its odd series to s^9.
//   pow:    x^y = 2^(y*log2 x) for x > 0 (0 for x <= 0).
// The CPU oracle evaluates the same definitions, so both sides agree bitwise.
// ---------------------------------------------------------------------------
VRT_DI void sincos_(float x, float& s, float& c) {
  const float TWO_OVER_PI = 0.636619747f;
  const float PIO2_HI = 1.5703125f;
  const float PIO2_LO = 0.000483826792f;
  float kf = floorf(x * TWO_OVER_PI + 0.5f);
  int k = (int)kf;
  float r = (x - kf * PIO2_HI) - kf * PIO2_LO;
  float r2 = r * r;
  float sp = r + (r * r2) * (-0.166666672f + r2 * (0.00833333377f +
                 r2 * (-0.000198412701f + r2 * 2.75573188e-06f)));
  float cp = 1.0f + r2 * (-0.5f + r2 * (0.0416666679f + r2 * (-0.00138888892f +
                 r2 * (2.48015876e-05f + r2 * -2.755732e-07f))));
  switch (k & 3) {
    case 0: s = sp; c = cp; break;
    case 1: s = cp; c = -sp; break;
    case 2: s = -sp; c = -cp; break;
    default: s = -cp; c = sp; break;
  }
}

// Packed fp32 pairs (sm_100a's f32x2 arithmetic): each lane rounds exactly
// as the scalar instruction would, so a pair of independent scalar
// operations can run as one instruction without changing a bit.
VRT_DI float2 f2_mul(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 a, b, d;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t"
      "mul.rn.f32x2 d, a, b;\n\tmov.b64 {%0, %1}, d;\n\t}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
VRT_DI float2 f2_add(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 a, b, d;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t"
      "add.rn.f32x2 d, a, b;\n\tmov.b64 {%0, %1}, d;\n\t}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
VRT_DI float2 f2_sub(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 a, b, d;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t"
      "sub.rn.f32x2 d, a, b;\n\tmov.b64 {%0, %1}, d;\n\t}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
VRT_DI float pow2i_(int k) { return __uint_as_float((uint32_t)(k + 127) << 23); }

// Horner steps as explicit fused multiply-adds (one rounding each; the CPU
// restatement uses std::fmaf, so both sides round identically).
VRT_DI float exp_poly_(float r) {
  float p = __fmaf_rn(r, 0.000198412701f, 0.00138888892f);
  p = __fmaf_rn(r, p, 0.00833333377f);
  p = __fmaf_rn(r, p, 0.0416666679f);
  p = __fmaf_rn(r, p, 0.166666672f);
  p = __fmaf_rn(r, p, 0.5f);
  p = __fmaf_rn(r, p, 1.0f);
  return __fmaf_rn(r, p, 1.0f);
}

VRT_DI float exp_(float x) {
  if (!(x > -87.0f)) return 0.0f;
  if (x > 88.0f) return __int_as_float(0x7f800000);
  const float LOG2E = 1.44269502f;
  const float LN2_HI = 0.693145751953125f;
  const float LN2_LO = 1.42860677e-06f;
  float kf = floorf(__fmaf_rn(x, LOG2E, 0.5f));
  float r = __fmaf_rn(-kf, LN2_LO, __fmaf_rn(-kf, LN2_HI, x));
  return exp_poly_(r) * pow2i_((int)kf);
}

// exp_ for x <= 0 (and NaN), as the a-trous weights use it: the same
// reduction and polynomial, with the scaling by 2^k done by adding k to the
// exponent field.  That equals exp_'s multiplication exactly because every
// result for x in (-87, 0] is normal: the polynomial p lies in [0.707, 1.415)
// and k >= -126, with p > 1 whenever k = -126 (x < -86.988).
VRT_DI float exp_nonpos_(float x) {
  if (!(x > -87.0f)) return 0.0f;
  const float LOG2E = 1.44269502f;
  const float LN2_HI = 0.693145751953125f;
  const float LN2_LO = 1.42860677e-06f;
  const float kf = floorf(__fmaf_rn(x, LOG2E, 0.5f));
  const float r = __fmaf_rn(-kf, LN2_LO, __fmaf_rn(-kf, LN2_HI, x));
  return __int_as_float(__float_as_int(exp_poly_(r)) + ((int)kf << 23));
}

VRT_DI float exp2_(float z) {
  if (!(z > -126.0f)) return 0.0f;
  if (z > 127.0f) return __int_as_float(0x7f800000);
  float kf = floorf(z + 0.5f);
  float f = z - kf;
  return exp_poly_(f * 0.693147182f) * pow2i_((int)kf);
}

VRT_DI float log2_(float x) {
  uint32_t b = __float_as_uint(x);
  int e = (int)(b >> 23) - 127;
  if ((b >> 23) == 0) {
    x = x * 8388608.0f; b = __float_as_uint(x); e = (int)(b >> 23) - 127 - 23;
  }
  float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421354f) { m = m * 0.5f; e += 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float q = __fmaf_rn(s2, 0.111111112f, 0.142857149f);
  q = __fmaf_rn(s2, q, 0.200000003f);
  q = __fmaf_rn(s2, q, 0.333333343f);
  const float at = __fmaf_rn(s * s2, q, s);
  return __fmaf_rn(at, 2.88539004f, (float)e);
}

VRT_DI float pow_(float x, float y) {
  if (!(x > 0.0f)) return 0.0f;
  return exp2_(y * log2_(x));
}

// ---------------------------------------------------------------------------
// Storage formats
// ---------------------------------------------------------------------------
// rgba16float store: round to nearest even; finite values beyond the half
// range store as the largest finite half (65504).  WebGPU leaves the overflow
// to the backend (Vulkan allows the largest finite value or infinity); an
// infinite texel would turn a running history mean infinite for good.
VRT_DI uint32_t h2bits(float x) {
  const float ax = fabsf(x);
  if (ax > 65504.0f && ax < INFINITY) x = copysignf(65504.0f, x);
  return (uint32_t)__half_as_ushort(__float2half_rn(x));
}
VRT_DI float bits2f(uint32_t h) { return __half2float(__ushort_as_half((unsigned short)h)); }
VRT_DI uint2 pack_h4(float a, float b, float c, float d) {
  return make_uint2(h2bits(a) | (h2bits(b) << 16), h2bits(c) | (h2bits(d) << 16));
}
VRT_DI float4 unpack_h4(uint2 v) {
  return make_float4(bits2f(v.x & 0xffffu), bits2f(v.x >> 16), bits2f(v.y & 0xffffu), bits2f(v.y >> 16));
}
// rgba8unorm store: nearest of clamp(x,0,1)*255.
VRT_DI uint32_t unorm8_(float x) { return (uint32_t)floorf(clamp_(x, 0.0f, 1.0f) * 255.0f + 0.5f); }

// ---------------------------------------------------------------------------
// RNG -- PCG hash, one stream per pixel per frame (common.wgsl:69-84)
// ---------------------------------------------------------------------------
VRT_DI uint32_t pcg_hash(uint32_t v) {
  v = v * 747796405u + 2891336453u;
  uint32_t w = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  return (w >> 22u) ^ w;
}
VRT_DI uint32_t init_rng(uint32_t px, uint32_t py, uint32_t frame) {
  return pcg_hash(px + pcg_hash(py + pcg_hash(frame)));
}
VRT_DI float rand_(uint32_t& s) {
  s = pcg_hash(s);
  return __uint2float_rn(s) * 2.3283064365386963e-10f;
}

// ---------------------------------------------------------------------------
// Camera, sky, sampling (common.wgsl:90-139)
// ---------------------------------------------------------------------------
// mat4 (column-major) * vec4, summed column by column.
VRT_DI void matvec4(const float* m, float v0, float v1, float v2, float v3, float out[4]) {
#pragma unroll
  for (int r = 0; r < 4; r++) out[r] = ((m[r] * v0 + m[4 + r] * v1) + m[8 + r] * v2) + m[12 + r] * v3;
}

VRT_DI F3 camera_ray(const Uni& u, float uvx, float uvy) {
  float far[4];
  matvec4(u.invViewProj, uvx * 2.0f - 1.0f, 1.0f - uvy * 2.0f, 1.0f, 1.0f, far);
  F3 fp = f3(far[0] / far[3], far[1] / far[3], far[2] / far[3]);
  return normalize3(fp - f3(u.camPos[0], u.camPos[1], u.camPos[2]));
}

VRT_DI F3 sky_color(const Uni& u, F3 rd, bool withSunDisc) {
  float up = clamp_(rd.y, -1.0f, 1.0f);
  F3 sky = mix3(f3(0.55f, 0.68f, 0.85f), f3(0.15f, 0.32f, 0.62f), pow_(fmax_(up, 0.0f), 0.55f));
  if (up < 0.0f) sky = mix3(sky, f3(0.28f, 0.26f, 0.24f), fmin_(1.0f, -up * 4.0f));
  F3 sd = f3(u.sunDir[0], u.sunDir[1], u.sunDir[2]);
  float sunAmt = fmax_(dot3(rd, sd), 0.0f);
  float s2 = sunAmt * sunAmt, s4 = s2 * s2, s8 = s4 * s4;
  sky = sky + (f3(1.0f, 0.75f, 0.5f) * s8) * 0.2f;
  if (withSunDisc && sunAmt > u.sunDir[3]) {
    float d = fmax_(kTwoPi * (1.0f - u.sunDir[3]), 1e-4f);
    sky = sky + f3(u.sunRadiance[0] / d, u.sunRadiance[1] / d, u.sunRadiance[2] / d);
  }
  return sky * u.sunRadiance[3];
}

VRT_DI F3 sample_sun_dir(const Uni& u, uint32_t& rng) {
  float rx = rand_(rng);
  float ry = rand_(rng);
  float cosT = mix_(1.0f, u.sunDir[3], rx);
  float sinT = __fsqrt_rn(fmax_(0.0f, 1.0f - cosT * cosT));
  float phi = kTwoPi * ry;
  F3 w = f3(u.sunDir[0], u.sunDir[1], u.sunDir[2]);
  F3 a = fabsf(w.x) > 0.9f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
  F3 tang = normalize3(cross3(a, w));
  F3 bitan = cross3(w, tang);
  float sp, cp;
  sincos_(phi, sp, cp);
  return normalize3((tang * (cp * sinT) + bitan * (sp * sinT)) + w * cosT);
}

VRT_DI F3 cosine_hemisphere(F3 n, uint32_t& rng) {
  float rx = rand_(rng);
  float ry = rand_(rng);
  float phi = kTwoPi * rx;
  float sr = __fsqrt_rn(ry);
  F3 a = fabsf(n.x) > 0.9f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
  F3 tang = normalize3(cross3(a, n));
  F3 bitan = cross3(n, tang);
  float sp, cp;
  sincos_(phi, sp, cp);
  return normalize3((tang * (cp * sr) + bitan * (sp * sr)) + n * __fsqrt_rn(fmax_(0.0f, 1.0f - ry)));
}

// Material unpack (voxel.wgsl:41-51)
struct Mat { F3 albedo; float emissive; };
VRT_DI Mat unpack_material(uint32_t m) {
  const float s = 1.0f / 255.0f;
  F3 a = f3((float)(m & 0xffu), (float)((m >> 8) & 0xffu), (float)((m >> 16) & 0xffu)) * s;
  Mat r;
  r.albedo = a * a;
  r.emissive = (float)((m >> 24) & 0xffu) * s;
  return r;
}

// ---------------------------------------------------------------------------
// Voxel world + two-level DDA (voxel.wgsl:18-153)
// ---------------------------------------------------------------------------
struct DScene {
  const uint32_t* __restrict__ vox;     // N^3 packed voxels
  const uint32_t* __restrict__ masks;   // 16 words per brick
  const uint32_t* __restrict__ bits;    // 1 bit per brick: bricks[bi] != 0
  int N, BG;
};

struct DHit {
  float t;            // metres, < 0 miss
  F3 n;
  uint32_t mat;
  int vx, vy, vz;
};

struct DCount {
  uint32_t rays, outer, inner, vreads;
};

// Block-reduced traversal counters: stats[0..4] += rays, brick iterations,
// voxel iterations, voxel reads, pixels of the block (the frame counters'
// first five slots); one atomic per counter per block of 256 threads, since
// every block adds to the same counters.  All threads of the block call it.
VRT_DI void block_flush_stats(unsigned long long* stats, const DCount& c, uint32_t pix) {
  __shared__ uint32_t s_part[8][5];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t v[5] = {__reduce_add_sync(full, c.rays), __reduce_add_sync(full, c.outer),
                         __reduce_add_sync(full, c.inner), __reduce_add_sync(full, c.vreads),
                         __reduce_add_sync(full, pix)};
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 5; k++) s_part[w][k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    unsigned long long tot = 0ull;
    const int nw = (int)(blockDim.x >> 5);   // blocks of up to 256 threads
    for (int q = 0; q < nw; q++) tot += s_part[q][threadIdx.x];
    if (tot) atomicAdd(stats + threadIdx.x, tot);
  }
}

// Block-reduced single counter: *dst += the sum of v over the block (one
// atomic per block).  All threads of the block call it.
VRT_DI void block_flush_one(unsigned long long* dst, uint32_t v) {
  __shared__ uint32_t s_one[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t r = __reduce_add_sync(0xffffffffu, v);
  if (lane == 0) s_one[w] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tot = 0ull;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) tot += s_one[q];
    if (tot) atomicAdd(dst, tot);
  }
}

// Brick occupancy bit of brick bi from the bitmap `occ` (shared memory when
// the kernel staged it, global otherwise).
VRT_DI bool brick_occupied(const uint32_t* occ, uint32_t bi) {
  return (occ[bi >> 5] >> (bi & 31u)) & 1u;
}

// One component of hit.n = -vmask * vec3<f32>(stepDir) (voxel.wgsl:126) with
// IEEE signed zeros: -1*s on the stepped axis, -0*s elsewhere.  The sign bit
// is set exactly when s >= 0; the magnitude is 1 only on the stepped axis with
// s != 0.  Written on the bits so no compiler rewrite can drop a -0.
VRT_DI float face_normal_component(bool on_axis, int s) {
  const uint32_t sign = s >= 0 ? 0x80000000u : 0u;
  const uint32_t mag = (on_axis && s != 0) ? 0x3f800000u : 0u;
  return __uint_as_float(sign | mag);
}

// trace(): the reference's two-level Amanatides-Woo walk.  Outer loop over
// 8^3 bricks (at most 3*BGRID+2 steps), inner per-voxel loop (at most 24
// steps) inside occupied bricks; brick occupancy comes from a 1-bit-per-brick
// bitmap, voxel occupancy from the 16-word brick mask (read-only path), and
// the packed voxel is read on a hit.  Counters track iterations entered.
template <bool kCount>
VRT_DI DHit trace(const DScene& S, const uint32_t* occ, F3 roW, F3 rd, float maxTW, DCount& cnt) {
  DHit hit;
  hit.t = -1.0f; hit.mat = 0u; hit.n = f3(-rd.x, -rd.y, -rd.z);
  hit.vx = hit.vy = hit.vz = -1;
  if (kCount) cnt.rays++;
  const int BG = S.BG;

  const F3 ro = roW * kInvVoxel;
  const float maxT = maxTW * kInvVoxel;
  const float sgx = rd.x >= 0.0f ? 1.0f : -1.0f;
  const float sgy = rd.y >= 0.0f ? 1.0f : -1.0f;
  const float sgz = rd.z >= 0.0f ? 1.0f : -1.0f;
  const F3 invRd = f3(safe_inv(sgx, rd.x), safe_inv(sgy, rd.y), safe_inv(sgz, rd.z));
  const int sx = rd.x > 0.0f ? 1 : (rd.x < 0.0f ? -1 : 0);
  const int sy = rd.y > 0.0f ? 1 : (rd.y < 0.0f ? -1 : 0);
  const int sz = rd.z > 0.0f ? 1 : (rd.z < 0.0f ? -1 : 0);
  const F3 stepGE = f3(rd.x >= 0.0f ? 1.0f : 0.0f, rd.y >= 0.0f ? 1.0f : 0.0f, rd.z >= 0.0f ? 1.0f : 0.0f);

  const float G = (float)S.N;
  // 0 - ro, not -ro: +0 stays +0 (voxel.wgsl:86).
  const F3 t0 = f3(__fsub_rn(0.0f, ro.x), __fsub_rn(0.0f, ro.y), __fsub_rn(0.0f, ro.z)) * invRd;
  const F3 t1 = (f3(G, G, G) - ro) * invRd;
  const F3 tmin3 = min3(t0, t1);
  const F3 tmax3 = max3(t0, t1);
  const float tEnter = fmax_(fmax_(tmin3.x, tmin3.y), fmax_(tmin3.z, 0.0f));
  const float tExit = fmin_(fmin_(tmax3.x, tmax3.y), fmin_(tmax3.z, maxT));
  if (tEnter > tExit) return hit;

  int ax;
  if (tmin3.x >= tmin3.y && tmin3.x >= tmin3.z) ax = 0;
  else if (tmin3.y >= tmin3.z) ax = 1;
  else ax = 2;

  float t = tEnter;
  const F3 startP = ro + rd * (t + 1e-4f);
  int bx = iclamp_(ifloor_(startP.x * 0.125f), 0, BG - 1);
  int by = iclamp_(ifloor_(startP.y * 0.125f), 0, BG - 1);
  int bz = iclamp_(ifloor_(startP.z * 0.125f), 0, BG - 1);
  const F3 absInv = f3(fabsf(invRd.x), fabsf(invRd.y), fabsf(invRd.z));
  const F3 tDeltaB = absInv * 8.0f;
  F3 tMaxB = ((f3((float)bx, (float)by, (float)bz) + stepGE) * 8.0f - ro) * invRd;

  const int outerMax = 3 * BG + 2;
  for (int iter = 0; iter < outerMax; iter++) {
    if (t > tExit) break;
    if (kCount) cnt.outer++;
    const uint32_t bi = (uint32_t)bx + (uint32_t)by * (uint32_t)BG + (uint32_t)bz * (uint32_t)(BG * BG);
    if (brick_occupied(occ, bi)) {
      const int mnx = bx * kBrick, mny = by * kBrick, mnz = bz * kBrick;
      const F3 p = ro + rd * (t + 1e-4f);
      int vx = iclamp_(ifloor_(p.x), mnx, mnx + 7);
      int vy = iclamp_(ifloor_(p.y), mny, mny + 7);
      int vz = iclamp_(ifloor_(p.z), mnz, mnz + 7);
      F3 tMaxV = ((f3((float)vx, (float)vy, (float)vz) + stepGE) - ro) * invRd;
      float tCur = t;
      int vax = ax;
      const uint32_t* __restrict__ bm = S.masks + (size_t)bi * 16u;
      for (int j = 0; j < 3 * kBrick; j++) {
        if (kCount) cnt.inner++;
        const uint32_t bit = (uint32_t)((vx - mnx) + (vy - mny) * 8 + (vz - mnz) * 64);
        const uint32_t word = __ldg(bm + (bit >> 5));
        if ((word >> (bit & 31u)) & 1u) {
          const uint32_t m = __ldg(S.vox + ((uint32_t)vx + (uint32_t)vy * (uint32_t)S.N +
                                            (uint32_t)vz * (uint32_t)(S.N * S.N)));
          if (kCount) cnt.vreads++;
          if (tCur > maxT) return hit;
          hit.t = tCur * kVoxelSize;
          hit.n = f3(face_normal_component(vax == 0, sx), face_normal_component(vax == 1, sy),
                     face_normal_component(vax == 2, sz));
          hit.mat = m;
          hit.vx = vx; hit.vy = vy; hit.vz = vz;
          return hit;
        }
        if (tMaxV.x <= tMaxV.y && tMaxV.x <= tMaxV.z) {
          tCur = tMaxV.x; tMaxV.x = tMaxV.x + absInv.x; vx += sx; vax = 0;
        } else if (tMaxV.y <= tMaxV.z) {
          tCur = tMaxV.y; tMaxV.y = tMaxV.y + absInv.y; vy += sy; vax = 1;
        } else {
          tCur = tMaxV.z; tMaxV.z = tMaxV.z + absInv.z; vz += sz; vax = 2;
        }
        if (vx < mnx || vy < mny || vz < mnz || vx > mnx + 7 || vy > mny + 7 || vz > mnz + 7) break;
      }
    }
    if (tMaxB.x <= tMaxB.y && tMaxB.x <= tMaxB.z) {
      t = tMaxB.x; tMaxB.x = tMaxB.x + tDeltaB.x; bx += sx; ax = 0;
    } else if (tMaxB.y <= tMaxB.z) {
      t = tMaxB.y; tMaxB.y = tMaxB.y + tDeltaB.y; by += sy; ax = 1;
    } else {
      t = tMaxB.z; tMaxB.z = tMaxB.z + tDeltaB.z; bz += sz; ax = 2;
    }
    if (bx < 0 || by < 0 || bz < 0 || bx >= BG || by >= BG || bz >= BG) break;
  }
  return hit;
}

VRT_DI int face_of(F3 n) {
  if (n.x > 0.5f) return 0;
  if (n.x < -0.5f) return 1;
  if (n.y > 0.5f) return 2;
  if (n.y < -0.5f) return 3;
  if (n.z > 0.5f) return 4;
  if (n.z < -0.5f) return 5;
  return -1;
}

VRT_DI float luminance(float r, float g, float b) { return __fmaf_rn(b, 0.0722f, __fmaf_rn(g, 0.7152f, r * 0.2126f)); }

}  // namespace vrt
