// ============================================================================
// vrt_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// Scalar CPU restatement of VoxelRT's plain per-frame GI path, written from the
// reference's WebGPU shaders and host code:
//   src/shaders/voxel.wgsl:18-157     world access + two-level brick->voxel DDA
//   src/shaders/common.wgsl:69-139    PCG RNG, camera ray, sky, sun cone, cosine lobe
//   src/shaders/pathtrace.wgsl:248-330  plain (RF_RESTIR off) 1-spp path tracer
//   src/shaders/temporal.wgsl:17-77   reprojection + history accumulation
//   src/shaders/atrous.wgsl:26-83     edge-aware a-trous iteration
//   src/shaders/present.wgsl:40-55    remodulate, exposure, ACES, gamma
//   src/shaders/pathtrace.wgsl:199-246, 332-457, restir.wgsl,
//   reuse_temporal.wgsl, reuse_spatial.wgsl, dupmap.wgsl, pairing.js
//                                     ReSTIR passes (all flags but the world
//                                     cache, mutation and the quality signal)
//   src/main.js:628-659               HDR capture = illum * (alb8/255)^2
//   src/scene.js:411-433              brick occupancy words + 16-word masks
//   src/math.js:3-74, src/camera.js:47-57   view/projection matrices
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs load
// this library.  It is compiled with -ffp-contract=off so every + - * / is a
// single IEEE-754 binary32 operation in source order, which is the contract
// the CUDA kernels are held to bit-for-bit.
//
// Parity pin: the DDA is pinned to the reference's own CPU traversal
// (VoxelBench/pipeline/core.cpp:23-50 traceNaive, double precision) through
// golden ray fixtures generated from the reference sources (tests/golden).
// The shading math (RNG, sampling, sky, temporal, a-trous, present) restates
// WGSL that cannot execute here (no WebGPU implementation); that part is
// "parity unpinned" against the reference and is checked statistically
// (converged-image agreement with an FP64 accumulation).
//
// Transcendentals.  WGSL leaves sin/cos/exp/pow accuracy to the implementation
// (absolute error up to 2^-11 for sin/cos).  The oracle and the kernels both
// use the project's own definitions below (Cody-Waite reduction + Taylor
// series), so both sides compute identical bits.
//
// Literal mode (compiled with -DORC_LITERAL into liboracle_literal.so): the
// shader text as written, with none of the kernels' reformulations --
// sin/cos/exp/log2/pow from the C library's binary32 functions, pow(x, 8) and
// pow(x, 32) as pow, dot products as (x*x' + y*y') + z*z', and the a-trous
// weight as the product of its two exps with every tap summed (no skip of
// zero-weight taps, no fused multiply-adds).  The kernels are held to this
// mode at the specification's tolerances (per-sample radiance 1e-4 relative,
// temporal and denoised output 2e-3), not bit for bit.
// ============================================================================
#include <cstdint>
#include <cstring>
#include <cmath>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

#ifdef ORC_LITERAL
constexpr bool kLiteral = true;
#else
constexpr bool kLiteral = false;
#endif

// ---------------------------------------------------------------------------
// scalar helpers
// ---------------------------------------------------------------------------
inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

struct f3 { float x, y, z; };
inline f3 mk(float x, float y, float z) { return f3{x, y, z}; }
inline f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline f3 mul(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
inline f3 muls(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline f3 divv(f3 a, f3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float dot3(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline f3 cross3(f3 a, f3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length3(f3 a) { return std::sqrt(dot3(a, a)); }
inline f3 normalize3(f3 a) { float l = length3(a); return mk(a.x / l, a.y / l, a.z / l); }
inline float fminf_(float a, float b) { return b < a ? b : a; }   // WGSL min on non-NaN
inline float fmaxf_(float a, float b) { return a < b ? b : a; }
inline f3 min3(f3 a, f3 b) { return mk(fminf_(a.x, b.x), fminf_(a.y, b.y), fminf_(a.z, b.z)); }
inline f3 max3(f3 a, f3 b) { return mk(fmaxf_(a.x, b.x), fmaxf_(a.y, b.y), fmaxf_(a.z, b.z)); }
inline float clampf(float x, float lo, float hi) { return fminf_(fmaxf_(x, lo), hi); }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }  // WGSL mix
inline f3 mix3(f3 a, f3 b, float t) { return mk(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)); }

// ---------------------------------------------------------------------------
// Project transcendentals (shared definition with the CUDA kernels).
// ---------------------------------------------------------------------------
// sin and cos of x, |x| <= 8.  Quadrant k = round(x / (pi/2)); the remainder is
// formed Cody-Waite style with pi/2 = 201/128 + PIO2_LO, then evaluated by the
// Taylor series of sin (to r^9) and cos (to r^10) about zero.
inline void om_sincos(float x, float& s, float& c) {
  if (kLiteral) { s = std::sin(x); c = std::cos(x); return; }
  const float TWO_OVER_PI = 0.636619747f;
  const float PIO2_HI = 1.5703125f;
  const float PIO2_LO = 0.000483826792f;
  float kf = std::floor(x * TWO_OVER_PI + 0.5f);
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

// 2^k for integer k in [-126, 127].
inline float om_pow2i(int k) { return bitsf((uint32_t)(k + 127) << 23); }

// e^r for |r| <= 0.35: Taylor series to r^7, Horner steps as fused
// multiply-adds (the kernels use the same fused steps).
inline float om_exp_poly(float r) {
  float p = std::fmaf(r, 0.000198412701f, 0.00138888892f);
  p = std::fmaf(r, p, 0.00833333377f);
  p = std::fmaf(r, p, 0.0416666679f);
  p = std::fmaf(r, p, 0.166666672f);
  p = std::fmaf(r, p, 0.5f);
  p = std::fmaf(r, p, 1.0f);
  return std::fmaf(r, p, 1.0f);
}

// e^x: k = round(x log2 e), r = x - k ln2 (ln2 split into 0x3f317200 + LN2_LO).
inline float om_exp(float x) {
  if (kLiteral) return std::exp(x);
  if (!(x > -87.0f)) return 0.0f;        // also maps NaN/-inf to 0
  if (x > 88.0f) return INFINITY;
  const float LOG2E = 1.44269502f;
  const float LN2_HI = 0.693145751953125f;
  const float LN2_LO = 1.42860677e-06f;
  float kf = std::floor(std::fmaf(x, LOG2E, 0.5f));
  float r = std::fmaf(-kf, LN2_LO, std::fmaf(-kf, LN2_HI, x));
  return om_exp_poly(r) * om_pow2i((int)kf);
}

// 2^z: k = round(z), f = z - k (exact), 2^f = e^(f ln2).
inline float om_exp2(float z) {
  if (!(z > -126.0f)) return 0.0f;
  if (z > 127.0f) return INFINITY;
  float kf = std::floor(z + 0.5f);
  float f = z - kf;
  return om_exp_poly(f * 0.693147182f) * om_pow2i((int)kf);
}

// log2(x) for finite x > 0: x = m 2^e with m in [sqrt(1/2), sqrt(2)],
// log2(m) = (2/ln2) atanh(s), s = (m-1)/(m+1), atanh by its series to s^9.
inline float om_log2(float x) {
  if (kLiteral) return std::log2(x);
  uint32_t b = fbits(x);
  int e = (int)(b >> 23) - 127;
  if ((b >> 23) == 0) {                    // subnormal input
    x = x * 8388608.0f; b = fbits(x); e = (int)(b >> 23) - 127 - 23;
  }
  float m = bitsf((b & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421354f) { m = m * 0.5f; e += 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float q = std::fmaf(s2, 0.111111112f, 0.142857149f);
  q = std::fmaf(s2, q, 0.200000003f);
  q = std::fmaf(s2, q, 0.333333343f);
  const float at = std::fmaf(s * s2, q, s);
  return std::fmaf(at, 2.88539004f, (float)e);
}

// x^y for x >= 0, y > 0 (the only uses on this path); 0^y = 0.
inline float om_pow(float x, float y) {
  if (kLiteral) return std::pow(x, y);
  if (!(x > 0.0f)) return 0.0f;
  return om_exp2(y * om_log2(x));
}

// ---------------------------------------------------------------------------
// Storage formats
// ---------------------------------------------------------------------------
// binary32 -> binary16, round to nearest even (WebGPU rgba16float store);
// finite values that would round beyond the half range store as the largest
// finite half (65504): WebGPU leaves overflow to the backend (Vulkan allows
// the largest finite value or infinity), and an infinite texel would turn a
// running history mean infinite for good.  Infinity and NaN stay.
inline uint16_t f32_to_f16(float f) {
  uint32_t x = fbits(f);
  uint32_t sign = (x >> 16) & 0x8000u;
  uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return (uint16_t)(sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u));
  if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7bffu);
  if (ax < 0x38800000u) {
    if (ax < 0x33000000u) return (uint16_t)sign;
    uint32_t e = ax >> 23;
    uint32_t m = (ax & 0x7fffffu) | 0x800000u;
    uint32_t shift = 126u - e;
    uint32_t q = m >> shift;
    uint32_t rem = m & ((1u << shift) - 1u);
    uint32_t half = 1u << (shift - 1u);
    if (rem > half || (rem == half && (q & 1u))) q++;
    return (uint16_t)(sign | q);
  }
  uint32_t r = ax - 0x38000000u;
  uint32_t q = r >> 13;
  uint32_t rem = r & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) q++;
  return (uint16_t)(sign | q);
}

inline float f16_to_f32(uint16_t h) {
  uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
  uint32_t e = (h >> 10) & 0x1fu;
  uint32_t m = h & 0x3ffu;
  if (e == 0) {
    float v = (float)m * 5.96046448e-08f;       // m * 2^-24, exact
    return sign ? -v : v;
  }
  if (e == 31) return bitsf(sign | 0x7f800000u | (m << 13));
  return bitsf(sign | ((e + 112u) << 23) | (m << 13));
}

// rgba8unorm store: nearest of clamp(x,0,1)*255.
inline uint8_t unorm8(float x) {
  float c = clampf(x, 0.0f, 1.0f);
  return (uint8_t)(int)std::floor(c * 255.0f + 0.5f);
}

// ---------------------------------------------------------------------------
// Uniform block (common.wgsl:13-35), read by float offsets of the 304-B UBO.
// ---------------------------------------------------------------------------
struct Uni {
  float invViewProj[16], prevViewProj[16];
  float camPos[4], prevCamPos[4], sunDir[4], sunRadiance[4];
  uint32_t params0[4];
  float params1[4];
  uint32_t params2[4];
  float params3[4], params4[4], params5[4], params6[4];
};
static_assert(sizeof(Uni) == 304, "uniform block is 304 bytes");

// WGSL mat4x4 * vec4 with column-major storage, summed column by column.
inline void matvec4(const float* m, const float v[4], float out[4]) {
  for (int r = 0; r < 4; r++) {
    out[r] = ((m[0 + r] * v[0] + m[4 + r] * v[1]) + m[8 + r] * v[2]) + m[12 + r] * v[3];
  }
}

const float PI = 3.14159274f;            // f32(3.14159265358979)
const float TWO_PI = 6.28318548f;        // f32(2 * 3.14159265358979)
const float INV_PI = 0.318309873f;       // f32(0.31830988618)
const float VOXEL_SIZE = 0.0625f;        // scene.js:5
const float INV_VOXEL = 16.0f;
const int BRICK = 8;                     // scene.js:6
const float EMISSIVE_SCALE = 24.0f;      // common.wgsl:11

// ---------------------------------------------------------------------------
// RNG: PCG hash (common.wgsl:69-84)
// ---------------------------------------------------------------------------
inline uint32_t pcg_hash(uint32_t v) {
  v = v * 747796405u + 2891336453u;
  uint32_t w = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  return (w >> 22u) ^ w;
}
struct Rng {
  uint32_t s;
  float next() { s = pcg_hash(s); return (float)s * 2.3283064365386963e-10f; }  // f32(u32) * 2^-32
};
inline Rng init_rng(uint32_t px, uint32_t py, uint32_t frame) {
  return Rng{pcg_hash(px + pcg_hash(py + pcg_hash(frame)))};
}

// ---------------------------------------------------------------------------
// Voxel world + two-level DDA (voxel.wgsl:18-153)
// ---------------------------------------------------------------------------
struct World {
  const uint32_t* vox;
  const uint32_t* bricks;
  const uint32_t* masks;
  int N, BG;
};

struct Hit {
  float t; f3 n; uint32_t mat;
  int vx, vy, vz;
  uint32_t outer, inner, vreads;   // iteration counters (the build's step count)
};

// floor to int with saturation, NaN -> 0 (the semantics of cvt.rmi.s32.f32;
// WGSL's f32 -> i32 conversion also clamps to the i32 range).
inline int ifloor(float x) {
  float f = std::floor(x);
  if (f != f) return 0;
  if (f >= 2147483648.0f) return 2147483647;
  if (f < -2147483648.0f) return (-2147483647 - 1);
  return (int)f;
}
inline int iclamp(int x, int lo, int hi) { return std::min(std::max(x, lo), hi); }

// safeInv (voxel.wgsl:65-71)
inline f3 safe_inv(f3 v) {
  f3 s = mk(v.x >= 0.0f ? 1.0f : -1.0f, v.y >= 0.0f ? 1.0f : -1.0f, v.z >= 0.0f ? 1.0f : -1.0f);
  f3 a = mk(fmaxf_(std::fabs(v.x), 1e-8f), fmaxf_(std::fabs(v.y), 1e-8f), fmaxf_(std::fabs(v.z), 1e-8f));
  return divv(s, a);
}
inline int sgn(float x) { return x > 0.0f ? 1 : (x < 0.0f ? -1 : 0); }

// trace (voxel.wgsl:73-153)
Hit trace(const World& W, f3 roWorld, f3 rd, float maxTWorld) {
  Hit hit;
  hit.t = -1.0f; hit.mat = 0u; hit.n = mk(-rd.x, -rd.y, -rd.z);
  hit.vx = hit.vy = hit.vz = -1;
  hit.outer = hit.inner = hit.vreads = 0;
  const int N = W.N, BG = W.BG;

  f3 ro = muls(roWorld, INV_VOXEL);
  float maxT = maxTWorld * INV_VOXEL;
  f3 invRd = safe_inv(rd);
  int sx = sgn(rd.x), sy = sgn(rd.y), sz = sgn(rd.z);
  f3 stepGE = mk(rd.x >= 0.0f ? 1.0f : 0.0f, rd.y >= 0.0f ? 1.0f : 0.0f, rd.z >= 0.0f ? 1.0f : 0.0f);

  f3 t0 = mul(sub(mk(0, 0, 0), ro), invRd);
  float G = (float)N;
  f3 t1 = mul(sub(mk(G, G, G), ro), invRd);
  f3 tmin3 = min3(t0, t1);
  f3 tmax3 = max3(t0, t1);
  float tEnter = fmaxf_(fmaxf_(tmin3.x, tmin3.y), fmaxf_(tmin3.z, 0.0f));
  float tExit = fminf_(fminf_(tmax3.x, tmax3.y), fminf_(tmax3.z, maxT));
  if (tEnter > tExit) return hit;

  int ax;   // entry face axis (voxel.wgsl:95-98)
  if (tmin3.x >= tmin3.y && tmin3.x >= tmin3.z) ax = 0;
  else if (tmin3.y >= tmin3.z) ax = 1;
  else ax = 2;

  float t = tEnter;
  float tn = t + 1e-4f;
  f3 startP = add(ro, muls(rd, tn));
  int bx = iclamp(ifloor(startP.x / 8.0f), 0, BG - 1);
  int by = iclamp(ifloor(startP.y / 8.0f), 0, BG - 1);
  int bz = iclamp(ifloor(startP.z / 8.0f), 0, BG - 1);
  f3 absInv = mk(std::fabs(invRd.x), std::fabs(invRd.y), std::fabs(invRd.z));
  f3 tDeltaB = muls(absInv, 8.0f);
  f3 tMaxB = mul(sub(muls(add(mk((float)bx, (float)by, (float)bz), stepGE), 8.0f), ro), invRd);

  for (int iter = 0; iter < 3 * BG + 2; iter++) {
    if (t > tExit) break;
    hit.outer++;
    uint32_t bi = (uint32_t)bx + (uint32_t)by * (uint32_t)BG + (uint32_t)bz * (uint32_t)(BG * BG);
    if (W.bricks[bi] != 0u) {
      int mnx = bx * BRICK, mny = by * BRICK, mnz = bz * BRICK;
      int mxx = mnx + BRICK - 1, mxy = mny + BRICK - 1, mxz = mnz + BRICK - 1;
      float tp = t + 1e-4f;
      f3 p = add(ro, muls(rd, tp));
      int vx = iclamp(ifloor(p.x), mnx, mxx);
      int vy = iclamp(ifloor(p.y), mny, mxy);
      int vz = iclamp(ifloor(p.z), mnz, mxz);
      f3 tMaxV = mul(sub(add(mk((float)vx, (float)vy, (float)vz), stepGE), ro), invRd);
      float tCur = t;
      int vax = ax;
      for (int j = 0; j < 3 * BRICK; j++) {
        hit.inner++;
        uint32_t bit = (uint32_t)((vx - mnx) + (vy - mny) * BRICK + (vz - mnz) * BRICK * BRICK);
        uint32_t word = W.masks[bi * 16u + (bit >> 5u)];
        if ((word & (1u << (bit & 31u))) != 0u) {
          uint32_t m = W.vox[(uint32_t)vx + (uint32_t)vy * (uint32_t)N + (uint32_t)vz * (uint32_t)(N * N)];
          hit.vreads++;
          if (tCur > maxT) return hit;
          hit.t = tCur * VOXEL_SIZE;
          // n = -vmask * stepDir with vmask one-hot on axis vax
          float vm[3] = {0.0f, 0.0f, 0.0f};
          vm[vax] = 1.0f;
          hit.n = mk(-vm[0] * (float)sx, -vm[1] * (float)sy, -vm[2] * (float)sz);
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
        if (vx < mnx || vy < mny || vz < mnz || vx > mxx || vy > mxy || vz > mxz) break;
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

// Face index of a hit normal: 0..5 = +x,-x,+y,-y,+z,-z (VoxelBench core.h:106).
inline int face_of(f3 n) {
  if (n.x > 0.5f) return 0;
  if (n.x < -0.5f) return 1;
  if (n.y > 0.5f) return 2;
  if (n.y < -0.5f) return 3;
  if (n.z > 0.5f) return 4;
  if (n.z < -0.5f) return 5;
  return -1;
}

// Material (voxel.wgsl:41-51)
struct Mat { f3 albedo; float emissive; };
inline Mat unpack_material(uint32_t m) {
  Mat r;
  const float s = 1.0f / 255.0f;
  f3 a = muls(mk((float)(m & 0xffu), (float)((m >> 8) & 0xffu), (float)((m >> 16) & 0xffu)), s);
  r.albedo = mul(a, a);
  r.emissive = (float)((m >> 24) & 0xffu) * s;
  return r;
}

// ---------------------------------------------------------------------------
// Camera, sky, sampling (common.wgsl:90-139)
// ---------------------------------------------------------------------------
inline f3 camera_ray(const Uni& u, float uvx, float uvy) {
  float ndc[4] = {uvx * 2.0f - 1.0f, 1.0f - uvy * 2.0f, 1.0f, 1.0f};
  float far[4];
  matvec4(u.invViewProj, ndc, far);
  f3 fp = mk(far[0] / far[3], far[1] / far[3], far[2] / far[3]);
  return normalize3(sub(fp, mk(u.camPos[0], u.camPos[1], u.camPos[2])));
}

inline f3 sky_color(const Uni& u, f3 rd, bool withSunDisc) {
  float up = clampf(rd.y, -1.0f, 1.0f);
  f3 sky = mix3(mk(0.55f, 0.68f, 0.85f), mk(0.15f, 0.32f, 0.62f), om_pow(fmaxf_(up, 0.0f), 0.55f));
  if (up < 0.0f) sky = mix3(sky, mk(0.28f, 0.26f, 0.24f), fminf_(1.0f, -up * 4.0f));
  f3 sd = mk(u.sunDir[0], u.sunDir[1], u.sunDir[2]);
  float sunAmt = fmaxf_(dot3(rd, sd), 0.0f);
  float s2 = sunAmt * sunAmt, s4 = s2 * s2, s8 = s4 * s4;   // pow(sunAmt, 8)
  if (kLiteral) s8 = std::pow(sunAmt, 8.0f);
  sky = add(sky, muls(muls(mk(1.0f, 0.75f, 0.5f), s8), 0.2f));
  if (withSunDisc && sunAmt > u.sunDir[3]) {
    float solidAngle = TWO_PI * (1.0f - u.sunDir[3]);
    float d = fmaxf_(solidAngle, 1e-4f);
    sky = add(sky, mk(u.sunRadiance[0] / d, u.sunRadiance[1] / d, u.sunRadiance[2] / d));
  }
  return muls(sky, u.sunRadiance[3]);
}

inline f3 sample_sun_dir(const Uni& u, Rng& rng) {
  float rx = rng.next();
  float ry = rng.next();
  float cosT = mixf(1.0f, u.sunDir[3], rx);
  float sinT = std::sqrt(fmaxf_(0.0f, 1.0f - cosT * cosT));
  float phi = TWO_PI * ry;
  f3 w = mk(u.sunDir[0], u.sunDir[1], u.sunDir[2]);
  f3 a = std::fabs(w.x) > 0.9f ? mk(0, 1, 0) : mk(1, 0, 0);
  f3 tang = normalize3(cross3(a, w));
  f3 bitan = cross3(w, tang);
  float sp, cp; om_sincos(phi, sp, cp);
  return normalize3(add(add(muls(tang, cp * sinT), muls(bitan, sp * sinT)), muls(w, cosT)));
}

inline f3 cosine_hemisphere(f3 n, Rng& rng) {
  float rx = rng.next();
  float ry = rng.next();
  float phi = TWO_PI * rx;
  float sr = std::sqrt(ry);
  f3 a = std::fabs(n.x) > 0.9f ? mk(0, 1, 0) : mk(1, 0, 0);
  f3 tang = normalize3(cross3(a, n));
  f3 bitan = cross3(n, tang);
  float sp, cp; om_sincos(phi, sp, cp);
  f3 d = add(add(muls(tang, cp * sr), muls(bitan, sp * sr)), muls(n, std::sqrt(fmaxf_(0.0f, 1.0f - ry))));
  return normalize3(d);
}

// sig: a hash of the pixel's discrete path -- every trace issued, in order, by
// its outcome (miss, or hit voxel and face) -- so two restatements that differ
// in their last bits can be compared wherever they took the same path.
struct PixStats { uint64_t rays, outer, inner, vreads; uint32_t sig; };

// When set, every trace() issued by path_pixel appends (origin, direction,
// maxT) in voxel units -- the ray workload replayed by the reference
// traversal timing (bench.py's reference arm).
thread_local std::vector<float>* tl_ray_log = nullptr;

inline Hit trace_logged(const World& W, f3 ro, f3 rd, float maxT) {
  if (tl_ray_log) {
    float r[7] = {ro.x * INV_VOXEL, ro.y * INV_VOXEL, ro.z * INV_VOXEL, rd.x, rd.y, rd.z, maxT * INV_VOXEL};
    tl_ray_log->insert(tl_ray_log->end(), r, r + 7);
  }
  return trace(W, ro, rd, maxT);
}

// One pixel of the plain path (pathtrace.wgsl:248-330, baseline branch).
// Writes radiance (rgba16f bits + optional fp32 copy), albedo (rgba8 sqrt),
// G-buffer (rgba32f n,t).
void path_pixel(const World& W, const Uni& u, float fclamp, uint32_t gx, uint32_t gy,
                uint32_t dimx, uint32_t dimy, float rad_out[4], uint8_t alb_out[4], float gbuf_out[4],
                PixStats& st) {
  Rng rng = init_rng(gx, gy, u.params0[0]);
  float jx = rng.next() - 0.5f;
  float jy = rng.next() - 0.5f;
  float uvx = (((float)gx + 0.5f) + jx) / (float)dimx;
  float uvy = (((float)gy + 0.5f) + jy) / (float)dimy;
  f3 ro = mk(u.camPos[0], u.camPos[1], u.camPos[2]);
  f3 rd = camera_ray(u, uvx, uvy);

  auto count = [&](const Hit& h) {
    st.rays++; st.outer += h.outer; st.inner += h.inner; st.vreads += h.vreads;
    const uint32_t code = h.t < 0.0f ? 0x9e3779b9u
                                     : ((uint32_t)h.vx * 73856093u) ^ ((uint32_t)h.vy * 19349663u) ^
                                           ((uint32_t)h.vz * 83492791u) ^ ((uint32_t)face_of(h.n) << 28);
    st.sig = pcg_hash(st.sig ^ code);
  };
  Hit h0 = trace_logged(W, ro, rd, 1e4f);
  count(h0);
  if (h0.t < 0.0f) {
    f3 sky = sky_color(u, rd, true);
    rad_out[0] = sky.x; rad_out[1] = sky.y; rad_out[2] = sky.z; rad_out[3] = 1.0f;
    alb_out[0] = alb_out[1] = alb_out[2] = alb_out[3] = 255;
    gbuf_out[0] = -rd.x; gbuf_out[1] = -rd.y; gbuf_out[2] = -rd.z; gbuf_out[3] = -1.0f;
    return;
  }
  Mat mat1 = unpack_material(h0.mat);
  f3 x1 = add(ro, muls(rd, h0.t));
  f3 n1 = h0.n;
  alb_out[0] = unorm8(std::sqrt(mat1.albedo.x));
  alb_out[1] = unorm8(std::sqrt(mat1.albedo.y));
  alb_out[2] = unorm8(std::sqrt(mat1.albedo.z));
  alb_out[3] = 255;
  gbuf_out[0] = n1.x; gbuf_out[1] = n1.y; gbuf_out[2] = n1.z; gbuf_out[3] = h0.t;

  f3 radiance = mk(0, 0, 0);
  f3 tp = mk(1, 1, 1);
  f3 pos = x1, n = n1;
  Mat mat = mat1;
  const uint32_t nB = u.params0[1];
  f3 sunRad = mk(u.sunRadiance[0], u.sunRadiance[1], u.sunRadiance[2]);
  for (uint32_t bounce = 0; bounce <= nB; bounce++) {
    if (mat.emissive > 0.0f) {
      radiance = add(radiance, muls(mul(tp, mat.albedo), mat.emissive * EMISSIVE_SCALE));
    }
    f3 surf = add(pos, muls(n, 1e-3f));
    f3 l = sample_sun_dir(u, rng);
    float ndl = dot3(n, l);
    if (ndl > 0.0f && l.y > 0.0f) {
      Hit hs = trace_logged(W, surf, l, 1e4f);
      count(hs);
      if (!(hs.t >= 0.0f)) {
        radiance = add(radiance, mul(muls(muls(mul(tp, mat.albedo), INV_PI), ndl), sunRad));
      }
    }
    if (bounce == nB) break;
    rd = cosine_hemisphere(n, rng);
    tp = mul(tp, mat.albedo);
    if (bounce >= 2u) {
      float p = clampf(fmaxf_(tp.x, fmaxf_(tp.y, tp.z)), 0.05f, 0.95f);
      if (rng.next() > p) break;
      tp = mk(tp.x / p, tp.y / p, tp.z / p);
    }
    Hit h = trace_logged(W, surf, rd, 1e4f);
    count(h);
    if (h.t < 0.0f) {
      radiance = add(radiance, mul(tp, sky_color(u, rd, false)));
      break;
    }
    pos = add(surf, muls(rd, h.t));
    n = h.n;
    mat = unpack_material(h.mat);
  }
  if (!(fclamp <= 0.0f)) radiance = min3(radiance, mk(fclamp, fclamp, fclamp));
  f3 den = max3(mat1.albedo, mk(1e-3f, 1e-3f, 1e-3f));
  f3 demod = divv(radiance, den);
  rad_out[0] = demod.x; rad_out[1] = demod.y; rad_out[2] = demod.z; rad_out[3] = 1.0f;
}

// The cache-assisted estimator (voxelrt_b200/csrc/wavefront_core.cuh), per
// pixel.  No counterpart in the reference: the path is the plain one above
// with two roles.  Training pixels -- (x & 3, y & 3) == (phase & 3,
// phase >> 2) -- trace `train_bounces` bounces and record their vertices
// 0..rec_vertices-1 after the emission pickup (position, normal, albedo,
// radiance so far, throughput); every other path stops at its first bounce
// hit after the emission pickup there, leaving the reflected radiance to the
// network (query = position, normal, albedo; throughput tp1).
struct OrcCachePix {
  int32_t role;        // 0: primary miss, 1: training path, 2: cache-terminated path
  int32_t has_query;   // role 2: the bounce ray hit a surface
  int32_t nrec;        // role 1: vertices recorded
  int32_t pad;
  float den[3];        // max(albedo of vertex 0, 1e-3)
  float radiance[3];   // role 1: final radiance before the clamp; role 2: before the cache term
  float tp1[3];        // role 2: throughput reaching vertex 1
  float q9[9];         // role 2: the query
  float rec[8][15];    // role 1: position, normal, albedo, radiance, throughput
};

void cache_pixel(const World& W, const Uni& u, uint32_t gx, uint32_t gy, uint32_t dimx, uint32_t dimy,
                 uint32_t phase, uint32_t train_bounces, int rec_vertices, OrcCachePix& o) {
  std::memset(&o, 0, sizeof o);
  Rng rng = init_rng(gx, gy, u.params0[0]);
  float jx = rng.next() - 0.5f;
  float jy = rng.next() - 0.5f;
  float uvx = (((float)gx + 0.5f) + jx) / (float)dimx;
  float uvy = (((float)gy + 0.5f) + jy) / (float)dimy;
  f3 ro = mk(u.camPos[0], u.camPos[1], u.camPos[2]);
  f3 rd = camera_ray(u, uvx, uvy);
  Hit h0 = trace(W, ro, rd, 1e4f);
  if (h0.t < 0.0f) return;
  const bool train = (gx & 3u) == (phase & 3u) && (gy & 3u) == (phase >> 2);
  o.role = train ? 1 : 2;
  Mat mat1 = unpack_material(h0.mat);
  f3 den = max3(mat1.albedo, mk(1e-3f, 1e-3f, 1e-3f));
  o.den[0] = den.x; o.den[1] = den.y; o.den[2] = den.z;
  f3 radiance = mk(0, 0, 0);
  f3 tp = mk(1, 1, 1);
  f3 pos = add(ro, muls(rd, h0.t)), n = h0.n;
  Mat mat = mat1;
  const uint32_t nB = train ? train_bounces : 1u;
  f3 sunRad = mk(u.sunRadiance[0], u.sunRadiance[1], u.sunRadiance[2]);
  for (uint32_t bounce = 0; bounce <= nB; bounce++) {
    if (mat.emissive > 0.0f) radiance = add(radiance, muls(mul(tp, mat.albedo), mat.emissive * EMISSIVE_SCALE));
    if (!train && bounce == 1u) {
      o.has_query = 1;
      const float q[9] = {pos.x, pos.y, pos.z, n.x, n.y, n.z, mat.albedo.x, mat.albedo.y, mat.albedo.z};
      std::memcpy(o.q9, q, sizeof q);
      o.tp1[0] = tp.x; o.tp1[1] = tp.y; o.tp1[2] = tp.z;
      break;
    }
    if (train && (int)bounce < rec_vertices) {
      const float r[15] = {pos.x, pos.y, pos.z, n.x, n.y, n.z, mat.albedo.x, mat.albedo.y, mat.albedo.z,
                           radiance.x, radiance.y, radiance.z, tp.x, tp.y, tp.z};
      std::memcpy(o.rec[bounce], r, sizeof r);
      o.nrec = (int)bounce + 1;
    }
    f3 surf = add(pos, muls(n, 1e-3f));
    f3 l = sample_sun_dir(u, rng);
    float ndl = dot3(n, l);
    if (ndl > 0.0f && l.y > 0.0f) {
      Hit hs = trace(W, surf, l, 1e4f);
      if (!(hs.t >= 0.0f)) radiance = add(radiance, mul(muls(muls(mul(tp, mat.albedo), INV_PI), ndl), sunRad));
    }
    if (bounce == nB) break;
    rd = cosine_hemisphere(n, rng);
    tp = mul(tp, mat.albedo);
    if (bounce >= 2u) {
      float p = clampf(fmaxf_(tp.x, fmaxf_(tp.y, tp.z)), 0.05f, 0.95f);
      if (rng.next() > p) break;
      tp = mk(tp.x / p, tp.y / p, tp.z / p);
    }
    Hit h = trace(W, surf, rd, 1e4f);
    if (h.t < 0.0f) {
      radiance = add(radiance, mul(tp, sky_color(u, rd, false)));
      break;
    }
    pos = add(surf, muls(rd, h.t));
    n = h.n;
    mat = unpack_material(h.mat);
  }
  o.radiance[0] = radiance.x; o.radiance[1] = radiance.y; o.radiance[2] = radiance.z;
}

// Bilinear fetch with WebGPU's linear filter conventions: texel centres at
// +0.5, clamp-to-edge addressing (default sampler, main.js:317).
template <typename Fetch>
void bilinear(Fetch fetch, int W, int H, float u, float v, float out[4]) {
  float tx = u * (float)W - 0.5f;
  float ty = v * (float)H - 0.5f;
  float fx0 = std::floor(tx), fy0 = std::floor(ty);
  float ax = tx - fx0, ay = ty - fy0;
  int x0 = (int)fx0, y0 = (int)fy0;
  int xa = iclamp(x0, 0, W - 1), xb = iclamp(x0 + 1, 0, W - 1);
  int ya = iclamp(y0, 0, H - 1), yb = iclamp(y0 + 1, 0, H - 1);
  float p00[4], p10[4], p01[4], p11[4];
  fetch(xa, ya, p00); fetch(xb, ya, p10); fetch(xa, yb, p01); fetch(xb, yb, p11);
  for (int c = 0; c < 4; c++) {
    float top = p00[c] * (1.0f - ax) + p10[c] * ax;
    float bot = p01[c] * (1.0f - ax) + p11[c] * ax;
    out[c] = top * (1.0f - ay) + bot * ay;
  }
}

inline float luminance(const float* c) {
  if (kLiteral) return (c[0] * 0.2126f + c[1] * 0.7152f) + c[2] * 0.0722f;   // dot(c, weights) (atrous.wgsl:22-24)
  return std::fmaf(c[2], 0.0722f, std::fmaf(c[1], 0.7152f, c[0] * 0.2126f));
}


// ---------------------------------------------------------------------------
// ReSTIR pipeline (pathtrace.wgsl:1-246, 332-457, restir.wgsl,
// reuse_temporal.wgsl, reuse_spatial.wgsl, dupmap.wgsl, pairing.js)
// ---------------------------------------------------------------------------
const uint32_t SK_NONE = 0u, SK_POINT = 1u, SK_DIR = 2u;   // restir.wgsl:29-31
// common.wgsl:40-59
const uint32_t RF_TEMPORAL = 2u, RF_SPATIAL = 4u, RF_PAIRED = 8u, RF_DUPMAP = 16u, RF_FOOTPRINT = 32u,
               RF_VECTOR = 64u, RF_UNIFIED = 128u, RF_PLANE = 256u, RF_RESCUE = 512u, RF_FULLV = 1024u,
               RF_CLAMP = 2048u, RF_LIGHTPOWER = 4096u, RF_MIXSIGMA = 8192u, RF_ADAPTCAND = 16384u,
               RF_LIGHTGRID = 65536u, RF_MUTATE = 131072u, RF_HISTISOLATE = 262144u;
inline bool rflag(const Uni& u, uint32_t f) { return (u.params2[0] & f) != 0u; }

// Scene light data and reuse inputs (main.js:223-263).
struct RestirAux {
  const uint32_t* lights;    // 2 words per emissive face
  const float* alias;        // 4 floats per face
  const uint32_t* grid;      // 34 words per brick cell
  const uint32_t* pairing;   // 254^2 + 230^2 + 210^2 words
  const float* dup;          // previous frame's duplication map
};

// Decoded reservoir sample (restir.wgsl:33-41).
struct RSample {
  uint32_t kind;
  f3 pos, n, rad;
  float W, c;
  uint32_t seed;
};

inline RSample null_sample(float c) {
  RSample s;
  s.kind = SK_NONE;
  s.pos = s.n = s.rad = mk(0, 0, 0);
  s.W = 0.0f;
  s.c = c;
  s.seed = 0u;
  return s;
}

// WGSL f32 -> i32 / u32: toward zero, saturating, NaN -> 0.
inline int itrunc(float x) {
  if (x != x) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x < -2147483648.0f) return (-2147483647 - 1);
  return (int)x;
}
inline uint32_t utrunc(float x) {
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967296.0f) return 4294967295u;
  return (uint32_t)x;
}

// pack2x16snorm / unpack2x16snorm, one component (WGSL builtin definitions).
inline uint32_t snorm16(float v) {
  float c = fminf_(1.0f, fmaxf_(-1.0f, v));
  return (uint32_t)(uint16_t)(int16_t)(int)std::floor(0.5f + 32767.0f * c);
}
inline float unsnorm16(uint32_t b) { return fmaxf_((float)(int16_t)(uint16_t)b / 32767.0f, -1.0f); }
inline float sgn_ge0(float x) { return x >= 0.0f ? 1.0f : -1.0f; }

// octEncode (restir.wgsl:43-50)
inline void oct_encode(f3 nIn, float& ex, float& ey) {
  float s = (std::fabs(nIn.x) + std::fabs(nIn.y)) + std::fabs(nIn.z);
  f3 n = mk(nIn.x / s, nIn.y / s, nIn.z / s);
  ex = n.x; ey = n.y;
  if (n.z < 0.0f) {
    ex = (1.0f - std::fabs(n.y)) * sgn_ge0(n.x);
    ey = (1.0f - std::fabs(n.x)) * sgn_ge0(n.y);
  }
}

// octDecode (restir.wgsl:52-59)
inline f3 oct_decode(float ex, float ey) {
  f3 n = mk(ex, ey, (1.0f - std::fabs(ex)) - std::fabs(ey));
  if (n.z < 0.0f) n = mk((1.0f - std::fabs(n.y)) * sgn_ge0(n.x), (1.0f - std::fabs(n.x)) * sgn_ge0(n.y), n.z);
  return normalize3(n);
}

// packReservoir (restir.wgsl:61-71): 8 words, posW then data.
inline void pack_res(const RSample& s, uint32_t* w) {
  uint32_t cq = std::min(utrunc(s.c + 0.5f), 255u);
  f3 nn = s.kind != SK_POINT ? mk(0, 1, 0) : s.n;
  float ex, ey;
  oct_encode(nn, ex, ey);
  w[0] = fbits(s.pos.x); w[1] = fbits(s.pos.y); w[2] = fbits(s.pos.z); w[3] = fbits(s.W);
  w[4] = (uint32_t)f32_to_f16(s.rad.x) | ((uint32_t)f32_to_f16(s.rad.y) << 16);
  w[5] = ((uint32_t)f32_to_f16(s.rad.z) & 0xffffu) | (s.kind << 16) | (cq << 18);
  w[6] = snorm16(ex) | (snorm16(ey) << 16);
  w[7] = s.seed;
}

// unpackReservoir (restir.wgsl:73-84)
inline RSample unpack_res(const uint32_t* w) {
  RSample s;
  s.pos = mk(bitsf(w[0]), bitsf(w[1]), bitsf(w[2]));
  s.W = bitsf(w[3]);
  s.rad = mk(f16_to_f32((uint16_t)(w[4] & 0xffffu)), f16_to_f32((uint16_t)(w[4] >> 16)),
             f16_to_f32((uint16_t)(w[5] & 0xffffu)));
  s.kind = (w[5] >> 16) & 3u;
  s.c = (float)((w[5] >> 18) & 0xffu);
  s.n = oct_decode(unsnorm16(w[6] & 0xffffu), unsnorm16(w[6] >> 16));
  s.seed = w[7];
  return s;
}

// lum (restir.wgsl:90-92), a dot product summed left to right.
inline float rlum(f3 c) { return (c.x * 0.2126f + c.y * 0.7152f) + c.z * 0.0722f; }

// evalF (restir.wgsl:143-159); inverseSqrt(r2) = 1 / sqrt(r2).
inline f3 eval_f(const RSample& s, f3 x1, f3 n1) {
  if (s.kind == SK_POINT) {
    f3 d = sub(s.pos, x1);
    float r2 = fmaxf_(dot3(d, d), 1e-4f);
    f3 dir = muls(d, 1.0f / std::sqrt(r2));
    float cos1 = dot3(n1, dir);
    float cos2 = dot3(s.n, mk(-dir.x, -dir.y, -dir.z));
    if (cos1 <= 0.0f || cos2 <= 0.0f) return mk(0, 0, 0);
    return muls(s.rad, ((INV_PI * cos1) * cos2) / r2);
  }
  if (s.kind == SK_DIR) {
    float cos1 = dot3(n1, s.pos);
    if (cos1 <= 0.0f) return mk(0, 0, 0);
    return muls(s.rad, INV_PI * cos1);
  }
  return mk(0, 0, 0);
}
inline float eval_target(const RSample& s, f3 x1, f3 n1) { return rlum(eval_f(s, x1, n1)); }

// footprintOK (restir.wgsl:172-180)
inline bool footprint_ok(const Uni& u, const RSample& s, f3 x1, f3 n1, float tPrim, float cosView) {
  if (s.kind != SK_POINT) return true;
  f3 d = sub(s.pos, x1);
  float r2 = dot3(d, d);
  f3 dir = muls(d, 1.0f / std::sqrt(fmaxf_(r2, 1e-8f)));
  float cos1 = fmaxf_(dot3(n1, dir), 0.0f);
  float cos2 = fmaxf_(dot3(s.n, mk(-dir.x, -dir.y, -dir.z)), 0.0f);
  return r2 >= u.params3[3] * tPrim * tPrim * cos1 * cos2 / fmaxf_(cosView, 0.05f);
}

// receiverPoint (restir.wgsl:127-137); WGSL round() is half-to-even.
inline f3 receiver_point(f3 ro, f3 rd, float t, f3 n1) {
  f3 approx = add(ro, muls(rd, t));
  int ax = std::fabs(n1.x) > 0.5f ? 0 : (std::fabs(n1.y) > 0.5f ? 1 : 2);
  float ac = ax == 0 ? approx.x : (ax == 1 ? approx.y : approx.z);
  float roA = ax == 0 ? ro.x : (ax == 1 ? ro.y : ro.z);
  float rdA = ax == 0 ? rd.x : (ax == 1 ? rd.y : rd.z);
  if (std::fabs(rdA) < 1e-4f) return approx;
  float d = std::nearbyint(ac * INV_VOXEL) * VOXEL_SIZE;
  float tp = (d - roA) / rdA;
  return tp > 0.0f ? add(ro, muls(rd, tp)) : approx;
}

// surfaceAt (reuse_spatial.wgsl:111-114)
inline f3 surface_at(const Uni& u, int qx, int qy, int Wd, int Hd, const float* g) {
  return receiver_point(mk(u.camPos[0], u.camPos[1], u.camPos[2]),
                        camera_ray(u, ((float)qx + 0.5f) / (float)Wd, ((float)qy + 0.5f) / (float)Hd), g[3],
                        mk(g[0], g[1], g[2]));
}

inline f3 firefly(float fclamp, f3 v) { return fclamp <= 0.0f ? v : min3(v, mk(fclamp, fclamp, fclamp)); }

inline bool shadow_ray(const World& W, f3 o, f3 d, float maxT, PixStats& st) {
  Hit h = trace(W, o, d, maxT);
  st.rays++; st.outer += h.outer; st.inner += h.inner; st.vreads += h.vreads;
  return h.t >= 0.0f;
}

// ---- emissive-face sampling (pathtrace.wgsl:37-199) -------------------------
struct LightPoint { f3 pos, n, Le; float pdfA; };

// sampleGlobalLightIndex (pathtrace.wgsl:49-60)
uint32_t global_light_index(const Uni& u, const RestirAux& ax, Rng& rng) {
  uint32_t count = u.params2[1];
  if (rflag(u, RF_LIGHTPOWER)) {
    float uLight = rng.next() * (float)count;
    uint32_t base = std::min(utrunc(uLight), count - 1u);
    float frac = uLight - (float)base;
    const float* rec = ax.alias + 4 * (size_t)base;
    uint32_t aliasLi = std::min(utrunc(rec[1] + 0.5f), count - 1u);
    return frac >= rec[0] ? aliasLi : base;
  }
  return std::min(utrunc(rng.next() * (float)count), count - 1u);
}

// globalLightPdf (pathtrace.wgsl:62-65)
float global_light_pdf(const Uni& u, const RestirAux& ax, uint32_t li) {
  if (rflag(u, RF_LIGHTPOWER)) return fmaxf_(ax.alias[4 * (size_t)li + 2], 1e-8f);
  return 1.0f / (float)u.params2[1];
}

// pickLightIndex (pathtrace.wgsl:80-121)
uint32_t pick_light_index(const Uni& u, const RestirAux& ax, int BG, f3 pos, Rng& rng, float& pdf) {
  if (!rflag(u, RF_LIGHTGRID)) {
    uint32_t li = global_light_index(u, ax, rng);
    pdf = global_light_pdf(u, ax, li);
    return li;
  }
  const float k = INV_VOXEL / (float)BRICK;
  int bx = iclamp(ifloor(pos.x * k), 0, BG - 1), by = iclamp(ifloor(pos.y * k), 0, BG - 1),
      bz = iclamp(ifloor(pos.z * k), 0, BG - 1);
  const uint32_t* cell = ax.grid + (size_t)(uint32_t)(bx + by * BG + bz * BG * BG) * 34u;
  uint32_t n = std::min(cell[0], 16u);
  float wSum = bitsf(cell[1]);
  if (n == 0u || wSum <= 0.0f) {
    uint32_t li = global_light_index(u, ax, rng);
    pdf = global_light_pdf(u, ax, li);
    return li;
  }
  uint32_t li;
  if (rng.next() < 0.75f) {
    float r = rng.next() * wSum;
    li = cell[2];
    for (uint32_t i = 0; i < n; i++) {
      li = cell[2 + 2 * i];
      r -= bitsf(cell[3 + 2 * i]);
      if (r <= 0.0f) break;
    }
  } else {
    li = global_light_index(u, ax, rng);
  }
  float pCell = 0.0f;
  for (uint32_t i = 0; i < n; i++)
    if (cell[2 + 2 * i] == li) { pCell = bitsf(cell[3 + 2 * i]) / wSum; break; }
  pdf = 0.75f * pCell + (1.0f - 0.75f) * global_light_pdf(u, ax, li);
  return li;
}

// sampleLightFace (pathtrace.wgsl:123-144)
LightPoint sample_light_face(const Uni& u, const RestirAux& ax, int BG, f3 shadePos, Rng& rng) {
  float pdfSelect;
  uint32_t li = pick_light_index(u, ax, BG, shadePos, rng, pdfSelect);
  uint32_t lx = ax.lights[2 * (size_t)li], lm = ax.lights[2 * (size_t)li + 1];
  f3 v = mk((float)(lx & 0x1ffu), (float)((lx >> 9) & 0x1ffu), (float)((lx >> 18) & 0x1ffu));
  uint32_t face = (lx >> 27) & 7u, axis = face >> 1;
  float pos = (face & 1u) == 0u ? 1.0f : 0.0f;
  float r0 = rng.next();
  float r1 = rng.next();
  float r2 = rng.next();
  f3 q = add(v, mk(r0, r1, r2));
  f3 n = mk(0, 0, 0);
  if (axis == 0u) { q.x = v.x + pos; n.x = pos > 0.5f ? 1.0f : -1.0f; }
  else if (axis == 1u) { q.y = v.y + pos; n.y = pos > 0.5f ? 1.0f : -1.0f; }
  else { q.z = v.z + pos; n.z = pos > 0.5f ? 1.0f : -1.0f; }
  Mat mat = unpack_material(lm);
  LightPoint lp;
  lp.pos = muls(q, VOXEL_SIZE);
  lp.n = n;
  lp.Le = muls(mat.albedo, mat.emissive * EMISSIVE_SCALE);
  lp.pdfA = pdfSelect / (VOXEL_SIZE * VOXEL_SIZE);
  return lp;
}

// emissiveCandCount (pathtrace.wgsl:155-159)
uint32_t emissive_cand_count(const Uni& u, uint32_t bounce) {
  if (!rflag(u, RF_ADAPTCAND)) return bounce == 0u ? 4u : 1u;
  float n0 = clampf(std::nearbyint(u.params5[1] * 4.0f * (1.0f + om_log2(1.0f + (float)u.params2[1] / 256.0f))),
                    1.0f, 16.0f);
  return std::max(utrunc(n0) >> std::min(bounce, 31u), 1u);
}

// emissiveNEE (pathtrace.wgsl:167-199)
f3 emissive_nee(const World& W, const Uni& u, const RestirAux& ax, f3 pos, f3 n, f3 albedo, uint32_t nCand, Rng& rng,
                PixStats& st) {
  if (u.params2[1] == 0u) return mk(0, 0, 0);
  f3 surf = add(pos, muls(n, 1e-3f));
  float invM = 1.0f / (float)nCand;
  float wSum = 0.0f, selLum = 0.0f, selR2 = 0.0f;
  f3 sel = mk(0, 0, 0), selDir = mk(0, 0, 0);
  for (uint32_t k = 0; k < nCand; k++) {
    LightPoint lp = sample_light_face(u, ax, W.BG, pos, rng);
    f3 d = sub(lp.pos, surf);
    float r2 = fmaxf_(dot3(d, d), 1e-6f);
    f3 dir = muls(d, 1.0f / std::sqrt(r2));
    float cos1 = dot3(n, dir);
    float cos2 = dot3(lp.n, mk(-dir.x, -dir.y, -dir.z));
    if (cos1 <= 0.0f || cos2 <= 0.0f) continue;
    // albedo * INV_PI * cos1 * cos2 / r2 * lp.Le / lp.pdfA, left to right
    f3 v = muls(muls(muls(albedo, INV_PI), cos1), cos2);
    v = mk(v.x / r2, v.y / r2, v.z / r2);
    v = mul(v, lp.Le);
    v = mk(v.x / lp.pdfA, v.y / lp.pdfA, v.z / lp.pdfA);
    float w = rlum(v) * invM;
    if (w <= 0.0f) continue;
    bool first = wSum == 0.0f;
    wSum += w;
    if (first || rng.next() * wSum < w) { sel = v; selLum = rlum(v); selDir = dir; selR2 = r2; }
  }
  if (wSum <= 0.0f) return mk(0, 0, 0);
  float r = std::sqrt(selR2);
  if (shadow_ray(W, surf, selDir, r - 2e-3f, st)) return mk(0, 0, 0);
  return muls(sel, wSum / selLum);
}

// estimateLo (pathtrace.wgsl:205-246)
f3 estimate_lo(const World& W, const Uni& u, const RestirAux& ax, float fclamp, f3 x2, f3 n2, Mat mat2, Rng& rng,
               PixStats& st) {
  const bool unified = rflag(u, RF_UNIFIED);
  f3 Lo = mk(0, 0, 0), tp = mk(1, 1, 1);
  f3 pos = x2, n = n2;
  Mat mat = mat2;
  const uint32_t nB = u.params0[1];
  f3 sunRad = mk(u.sunRadiance[0], u.sunRadiance[1], u.sunRadiance[2]);
  for (uint32_t v = 1u; v <= nB; v++) {
    if (!unified && mat.emissive > 0.0f && v > 1u)
      Lo = add(Lo, muls(mul(tp, mat.albedo), mat.emissive * EMISSIVE_SCALE));
    f3 surf = add(pos, muls(n, 1e-3f));
    f3 l = sample_sun_dir(u, rng);
    float ndl = dot3(n, l);
    if (ndl > 0.0f && l.y > 0.0f && !shadow_ray(W, surf, l, 1e4f, st))
      Lo = add(Lo, mul(muls(muls(mul(tp, mat.albedo), INV_PI), ndl), sunRad));
    if (unified) Lo = add(Lo, mul(tp, emissive_nee(W, u, ax, pos, n, mat.albedo, emissive_cand_count(u, v), rng, st)));
    if (v == nB) break;
    f3 rd = cosine_hemisphere(n, rng);
    tp = mul(tp, mat.albedo);
    if (v >= 2u) {
      float p = clampf(fmaxf_(tp.x, fmaxf_(tp.y, tp.z)), 0.05f, 0.95f);
      if (rng.next() > p) break;
      tp = mk(tp.x / p, tp.y / p, tp.z / p);
    }
    Hit h = trace(W, surf, rd, 1e4f);
    st.rays++; st.outer += h.outer; st.inner += h.inner; st.vreads += h.vreads;
    if (h.t < 0.0f) {
      Lo = add(Lo, mul(tp, sky_color(u, rd, false)));
      break;
    }
    pos = add(surf, muls(rd, h.t));
    n = h.n;
    mat = unpack_material(h.mat);
  }
  return firefly(fclamp, Lo);
}

// Initial candidates of one pixel (pathtrace.wgsl:248-284, 332-457).
// Outputs: rgba16f radiance (sky pixels only), fp32 copy, albedo, G-buffer,
// reservoir A, rgba16f pass-through radiance.
void restir_initial_pixel(const World& W, const Uni& u, const RestirAux& ax, float fclamp, int gx, int gy, int Wd,
                          int Hd, uint16_t* rad16, float* rad32, uint8_t* alb8, float* gbuf, uint32_t* resA,
                          uint16_t* direct16, PixStats& st) {
  const size_t p = (size_t)gy * Wd + gx;
  Rng rng = init_rng((uint32_t)gx, (uint32_t)gy, u.params0[0]);
  float jx = rng.next() - 0.5f;
  float jy = rng.next() - 0.5f;
  f3 ro = mk(u.camPos[0], u.camPos[1], u.camPos[2]);
  f3 rd = camera_ray(u, (((float)gx + 0.5f) + jx) / (float)Wd, (((float)gy + 0.5f) + jy) / (float)Hd);
  Hit h0 = trace(W, ro, rd, 1e4f);
  st.rays++; st.outer += h0.outer; st.inner += h0.inner; st.vreads += h0.vreads;
  if (h0.t < 0.0f) {
    f3 sky = sky_color(u, rd, true);
    const float v[4] = {sky.x, sky.y, sky.z, 1.0f};
    for (int c = 0; c < 4; c++) {
      rad16[4 * p + c] = f32_to_f16(v[c]);
      if (rad32) rad32[4 * p + c] = v[c];
      direct16[4 * p + c] = f32_to_f16(v[c]);
      alb8[4 * p + c] = 255;
    }
    gbuf[4 * p] = -rd.x; gbuf[4 * p + 1] = -rd.y; gbuf[4 * p + 2] = -rd.z; gbuf[4 * p + 3] = -1.0f;
    std::memset(resA + 8 * p, 0, 32);
    return;
  }
  Mat mat1 = unpack_material(h0.mat);
  f3 x1 = add(ro, muls(rd, h0.t));
  f3 n1 = h0.n;
  f3 surf1 = add(x1, muls(n1, fmaxf_(1e-3f, h0.t * 1e-4f)));
  alb8[4 * p] = unorm8(std::sqrt(mat1.albedo.x));
  alb8[4 * p + 1] = unorm8(std::sqrt(mat1.albedo.y));
  alb8[4 * p + 2] = unorm8(std::sqrt(mat1.albedo.z));
  alb8[4 * p + 3] = 255;
  gbuf[4 * p] = n1.x; gbuf[4 * p + 1] = n1.y; gbuf[4 * p + 2] = n1.z; gbuf[4 * p + 3] = h0.t;

  const bool unified = rflag(u, RF_UNIFIED);
  float em = mat1.emissive * EMISSIVE_SCALE;
  f3 direct = mk(em, em, em);
  float wSum = 0.0f, selP = 0.0f;
  RSample sel = null_sample(0.0f);
  // Candidate: sun cone NEE at x1.
  {
    f3 l = sample_sun_dir(u, rng);
    float ndl = dot3(n1, l);
    if (ndl > 0.0f && l.y > 0.0f && !shadow_ray(W, surf1, l, 1e4f, st)) {
      if (unified) {
        float coneSA = 2.0f * PI * (1.0f - u.sunDir[3]);
        RSample s = null_sample(0.0f);
        s.kind = SK_DIR;
        s.pos = l;
        float den = fmaxf_(coneSA, 1e-5f);
        s.rad = mk(u.sunRadiance[0] / den, u.sunRadiance[1] / den, u.sunRadiance[2] / den);
        float pt = eval_target(s, x1, n1);
        float w = pt * coneSA;
        if (w > 0.0f) {
          wSum += w;
          if (rng.next() * wSum < w) { sel = s; selP = pt; }
        }
      } else {
        direct = add(direct, muls(mk(u.sunRadiance[0], u.sunRadiance[1], u.sunRadiance[2]), INV_PI * ndl));
      }
    }
  }
  // Candidate: light-list NEE at x1, RIS over emissiveCandCount(0) faces.
  if (unified && u.params2[1] > 0u) {
    uint32_t nCand = emissive_cand_count(u, 0u);
    float eSum = 0.0f, eSelP = 0.0f;
    RSample eSel = null_sample(0.0f);
    for (uint32_t k = 0; k < nCand; k++) {
      LightPoint lp = sample_light_face(u, ax, W.BG, x1, rng);
      RSample s = null_sample(0.0f);
      s.kind = SK_POINT;
      s.pos = lp.pos;
      s.n = lp.n;
      s.rad = lp.Le;
      float pt = eval_target(s, x1, n1);
      float w = pt / ((float)nCand * lp.pdfA);
      if (w > 0.0f) {
        eSum += w;
        if (rng.next() * eSum < w) { eSel = s; eSelP = pt; }
      }
    }
    if (eSel.kind != SK_NONE && eSelP > 0.0f) {
      f3 d = sub(eSel.pos, surf1);
      float r = length3(d);
      if (!shadow_ray(W, surf1, mk(d.x / r, d.y / r, d.z / r), r - 2e-3f, st)) {
        float We = eSum / eSelP;
        float w = eSelP * We;
        wSum += w;
        if (rng.next() * wSum < w) { sel = eSel; selP = eSelP; }
      }
    }
  }
  // Candidate: BSDF bounce path, reconnection vertex x2 carries Lo.
  if (u.params0[1] > 0u) {
    f3 brd = cosine_hemisphere(n1, rng);
    Hit h = trace(W, surf1, brd, 1e4f);
    st.rays++; st.outer += h.outer; st.inner += h.inner; st.vreads += h.vreads;
    RSample s = null_sample(0.0f);
    float Wc;
    if (h.t < 0.0f) {
      s.kind = SK_DIR;
      s.pos = brd;
      s.rad = sky_color(u, brd, false);
      Wc = PI / fmaxf_(dot3(n1, brd), 1e-4f);
    } else {
      f3 x2 = add(surf1, muls(brd, h.t));
      Mat mat2 = unpack_material(h.mat);
      f3 Lo = estimate_lo(W, u, ax, fclamp, x2, h.n, mat2, rng, st);
      if (!unified && mat2.emissive > 0.0f) Lo = add(Lo, muls(mat2.albedo, mat2.emissive * EMISSIVE_SCALE));
      s.kind = SK_POINT;
      s.pos = x2;
      s.n = h.n;
      s.rad = firefly(fclamp, Lo);
      f3 d = sub(x2, x1);
      float r2 = fmaxf_(dot3(d, d), 1e-6f);
      f3 dn = normalize3(d);
      float cos1 = fmaxf_(dot3(n1, dn), 1e-4f);
      float cos2 = fmaxf_(dot3(h.n, mk(-dn.x, -dn.y, -dn.z)), 1e-4f);
      Wc = PI / cos1 * r2 / cos2;
    }
    float pt = eval_target(s, x1, n1);
    float w = pt * Wc;
    if (w > 0.0f) {
      wSum += w;
      if (rng.next() * wSum < w) { sel = s; selP = pt; }
    }
  }
  RSample out = null_sample(0.0f);
  if (sel.kind != SK_NONE && selP > 0.0f) {
    out = sel;
    out.W = wSum / selP;
  }
  out.c = 1.0f;
  out.seed = pcg_hash((uint32_t)p + u.params0[0] * ((uint32_t)Wd * (uint32_t)Hd + 1u));
  pack_res(out, resA + 8 * p);
  const float dv[4] = {direct.x, direct.y, direct.z, 1.0f};
  for (int c = 0; c < 4; c++) direct16[4 * p + c] = f32_to_f16(dv[c]);
}

// validPrev (reuse_temporal.wgsl:38-46)
inline bool valid_prev(const Uni& u, int px, int py, int Wd, int Hd, const float* gbufPrev, f3 wp, f3 n1) {
  if (px < 0 || py < 0 || px >= Wd || py >= Hd) return false;
  const float* pg = gbufPrev + 4 * ((size_t)py * Wd + px);
  if (pg[3] <= 0.0f) return false;
  f3 dv = sub(wp, mk(u.prevCamPos[0], u.prevCamPos[1], u.prevCamPos[2]));
  float expectedT = length3(dv);
  bool depthOk = std::fabs(pg[3] - expectedT) < 0.08f * expectedT + 0.02f;
  bool normalOk = dot3(mk(pg[0], pg[1], pg[2]), n1) > 0.9f;
  return depthOk && normalOk;
}

// Temporal reuse of one pixel (reuse_temporal.wgsl:140-279 without the world
// cache and mutation).
void restir_temporal_pixel(const Uni& u, const RestirAux& ax, int gx, int gy, int Wd, int Hd, const float* gbufCur,
                           const float* gbufPrev, const uint32_t* resB, uint32_t* resA) {
  const size_t p = (size_t)gy * Wd + gx;
  const float* g = gbufCur + 4 * p;
  if (g[3] <= 0.0f) return;
  Rng rng = init_rng((uint32_t)gx, (uint32_t)gy, u.params0[0] ^ 0x5f356495u);
  f3 n1 = mk(g[0], g[1], g[2]);
  f3 x1 = surface_at(u, gx, gy, Wd, Hd, g);
  const float wp[4] = {x1.x, x1.y, x1.z, 1.0f};
  float pc[4];
  matvec4(u.prevViewProj, wp, pc);
  if (pc[3] <= 0.0f) return;
  float ndx = pc[0] / pc[3], ndy = pc[1] / pc[3];
  int ppx = itrunc((ndx * 0.5f + 0.5f) * (float)Wd);
  int ppy = itrunc(((-ndy) * 0.5f + 0.5f) * (float)Hd);
  bool found = valid_prev(u, ppx, ppy, Wd, Hd, gbufPrev, x1, n1);
  if (!found && rflag(u, RF_RESCUE)) {
    for (int dy = -1; dy <= 1 && !found; dy++)
      for (int dx = -1; dx <= 1 && !found; dx++) {
        int qx = ppx + dx, qy = ppy + dy;
        if ((dx != 0 || dy != 0) && valid_prev(u, qx, qy, Wd, Hd, gbufPrev, x1, n1)) {
          ppx = qx; ppy = qy;
          found = true;
        }
      }
  }
  if (!found) return;
  const size_t prevIdx = (size_t)ppy * Wd + ppx;
  RSample sT = unpack_res(resB + 8 * prevIdx);
  float dupScore = 0.0f;
  if (rflag(u, RF_DUPMAP) || rflag(u, RF_MUTATE)) dupScore = clampf(ax.dup[prevIdx], 0.0f, 1.0f);
  float cap = u.params3[0];
  if (rflag(u, RF_DUPMAP)) cap = mixf(u.params3[0], u.params3[1], om_pow(dupScore, u.params3[2]));
  float cT = fminf_(sT.c, cap);
  RSample sC = unpack_res(resA + 8 * p);
  float cC = fmaxf_(sC.c, 0.0f);
  float pC = eval_target(sC, x1, n1), pT = eval_target(sT, x1, n1);
  float mDen = fmaxf_(cC + cT, 1e-3f);
  float wC = (cC / mDen) * pC * fmaxf_(sC.W, 0.0f);
  float wT = (cT / mDen) * pT * fmaxf_(sT.W, 0.0f);
  float wSum = wC + wT;
  if (wSum <= 0.0f) {
    pack_res(null_sample(cC + cT), resA + 8 * p);
    return;
  }
  RSample sel = sC;
  float selP = pC;
  if (rng.next() * wSum >= wC) { sel = sT; selP = pT; }
  if (selP <= 0.0f) return;
  sel.W = wSum / selP;
  sel.c = cC + cT;
  pack_res(sel, resA + 8 * p);
}

// pairSize / pairOff / wrapMod / pairedPartner (reuse_spatial.wgsl:65-109)
inline int pair_size(uint32_t ti) { return ti == 0u ? 254 : (ti == 1u ? 230 : 210); }
inline uint32_t pair_off(uint32_t ti) { return ti == 0u ? 0u : (ti == 1u ? 64516u : 117416u); }
inline int wrap_mod(int v, int s) { return ((v % s) + s) % s; }

void paired_partner(const Uni& u, const RestirAux& ax, int px, int py, uint32_t ti, int& qx, int& qy) {
  int s = pair_size(ti);
  uint32_t h = pcg_hash(u.params0[0] * 2654435761u + ti * 0x68bc21ebu + 0x9e3779b9u);
  uint32_t h2 = pcg_hash(h);
  int offx = (int)(h % (uint32_t)s), offy = (int)(h2 % (uint32_t)s);
  bool mx = (h & 0x40000000u) != 0u, my = (h & 0x20000000u) != 0u, sw = (h & 0x10000000u) != 0u;
  int p0 = wrap_mod(px + offx, s), p1 = wrap_mod(py + offy, s);
  if (sw) std::swap(p0, p1);
  if (mx) p0 = s - 1 - p0;
  if (my) p1 = s - 1 - p1;
  uint32_t word = ax.pairing[pair_off(ti) + (uint32_t)(p1 * s + p0)];
  int dTx = (int32_t)(word << 16u) >> 16, dTy = (int32_t)word >> 16;
  int q0 = wrap_mod(p0 + dTx, s), q1 = wrap_mod(p1 + dTy, s);
  if (mx) q0 = s - 1 - q0;
  if (my) q1 = s - 1 - q1;
  if (sw) std::swap(q0, q1);
  int dx = wrap_mod(q0 - offx - px, s), dy = wrap_mod(q1 - offy - py, s);
  if (dx > s / 2) dx -= s;
  if (dy > s / 2) dy -= s;
  qx = px + dx;
  qy = py + dy;
}

// sampleVisible (reuse_spatial.wgsl:117-126)
bool sample_visible(const World& W, const RSample& s, f3 x1, f3 n1, PixStats& st) {
  f3 surf = add(x1, muls(n1, 1e-3f));
  if (s.kind == SK_DIR) return !shadow_ray(W, surf, s.pos, 1e4f, st);
  f3 d = sub(s.pos, surf);
  float r = length3(d);
  if (r < 2e-3f) return true;
  return !shadow_ray(W, surf, mk(d.x / r, d.y / r, d.z / r), r - 2e-3f, st);
}

// Spatial reuse + shading of one pixel (reuse_spatial.wgsl:128-354 without
// the world cache and the quality signal).
void restir_spatial_pixel(const World& W, const Uni& u, const RestirAux& ax, int gx, int gy, int Wd, int Hd,
                          const float* gbufCur, const uint32_t* resA, const uint16_t* direct16, uint16_t* rad16,
                          float* rad32, uint32_t* resB, PixStats& st) {
  const size_t p = (size_t)gy * Wd + gx;
  f3 direct = mk(f16_to_f32(direct16[4 * p]), f16_to_f32(direct16[4 * p + 1]), f16_to_f32(direct16[4 * p + 2]));
  auto out_radiance = [&](f3 v) {
    const float o[4] = {v.x, v.y, v.z, 1.0f};
    for (int c = 0; c < 4; c++) {
      rad16[4 * p + c] = f32_to_f16(o[c]);
      if (rad32) rad32[4 * p + c] = o[c];
    }
  };
  auto write_history = [&](const RSample& s) {
    if (rflag(u, RF_HISTISOLATE)) std::memcpy(resB + 8 * p, resA + 8 * p, 32);
    else pack_res(s, resB + 8 * p);
  };
  const float* g = gbufCur + 4 * p;
  if (g[3] <= 0.0f) {
    out_radiance(direct);
    std::memset(resB + 8 * p, 0, 32);
    return;
  }
  Rng rng = init_rng((uint32_t)gx, (uint32_t)gy, u.params0[0] ^ 0x2c1b3c6du);
  f3 x1 = surface_at(u, gx, gy, Wd, Hd, g);
  f3 n1 = mk(g[0], g[1], g[2]);
  float tPrim = g[3];
  float cosView = fmaxf_(dot3(n1, normalize3(sub(mk(u.camPos[0], u.camPos[1], u.camPos[2]), x1))), 0.0f);
  f3 domX1[4], domN1[4];
  float domC[4];
  RSample cand[4];
  uint32_t candDom[4];
  uint32_t nDom = 1u, nCand = 0u;
  RSample canonical = unpack_res(resA + 8 * p);
  domX1[0] = x1; domN1[0] = n1; domC[0] = canonical.c;
  if (canonical.kind != SK_NONE) { cand[0] = canonical; candDom[0] = 0u; nCand = 1u; }
  const bool paired = rflag(u, RF_PAIRED), planeExact = rflag(u, RF_PLANE);
  uint32_t taps = std::min(u.params2[2], 3u);
  if (rflag(u, RF_SPATIAL)) {
    for (uint32_t ti = 0u; ti < taps; ti++) {
      int qx, qy;
      if (paired) {
        uint32_t tex = ti;
        if (rflag(u, RF_MIXSIGMA)) tex = ti + 1u == taps ? 0u : ti + 1u;
        paired_partner(u, ax, gx, gy, tex, qx, qy);
      } else {
        float r = u.params4[0] * std::sqrt(rng.next());
        float a = 2.0f * PI * rng.next();
        float sa, ca;
        om_sincos(a, sa, ca);
        qx = gx + itrunc(ca * r);
        qy = gy + itrunc(sa * r);
      }
      if ((qx == gx && qy == gy) || qx < 0 || qy < 0 || qx >= Wd || qy >= Hd) continue;
      size_t q = (size_t)qy * Wd + qx;
      const float* gq = gbufCur + 4 * q;
      if (gq[3] <= 0.0f) continue;
      f3 x1q = surface_at(u, qx, qy, Wd, Hd, gq);
      f3 nq = mk(gq[0], gq[1], gq[2]);
      float nDot = dot3(n1, nq);
      bool genericOk = nDot > 0.9f && std::fabs(gq[3] - g[3]) < 0.1f * g[3] + 0.02f;
      bool samePlane = nDot > 0.99f && std::fabs(dot3(n1, sub(x1q, x1))) < 0.02f;
      bool ok = planeExact ? (genericOk || samePlane) : genericOk;
      if (!ok) continue;
      RSample rq = unpack_res(resA + 8 * q);
      bool reconnectable = rq.kind == SK_NONE || !rflag(u, RF_FOOTPRINT) || footprint_ok(u, rq, x1, n1, tPrim, cosView);
      if (!reconnectable) continue;
      domX1[nDom] = x1q; domN1[nDom] = nq; domC[nDom] = rq.c;
      if (rq.kind != SK_NONE) { cand[nCand] = rq; candDom[nCand] = nDom; nCand++; }
      nDom++;
    }
  }
  float cTotal = 0.0f;
  for (uint32_t l = 0u; l < nDom; l++) cTotal += domC[l];
  if (nCand == 0u) {
    out_radiance(direct);
    write_history(null_sample(fminf_(cTotal, 255.0f)));
    return;
  }
  const bool vector = rflag(u, RF_VECTOR), fullV = rflag(u, RF_FULLV);
  float wSum = 0.0f, selP = 0.0f;
  f3 contrib = mk(0, 0, 0);
  RSample sel = null_sample(0.0f);
  uint32_t selJ = 0u;
  for (uint32_t j = 0u; j < nCand; j++) {
    const RSample s = cand[j];
    float denom = 0.0f;
    for (uint32_t l = 0u; l < nDom; l++) denom += domC[l] * eval_target(s, domX1[l], domN1[l]);
    if (denom <= 0.0f) continue;
    uint32_t dj = candDom[j];
    float m = domC[dj] * eval_target(s, domX1[dj], domN1[dj]) / denom;
    float pMe = eval_target(s, x1, n1);
    float w = m * pMe * fmaxf_(s.W, 0.0f);
    if (w > 0.0f) {
      wSum += w;
      if (rng.next() * wSum < w) { sel = s; selP = pMe; selJ = j; }
    }
    if (vector && w > 0.0f) {
      bool vis = true;
      if (j > 0u || fullV) vis = sample_visible(W, s, x1, n1, st);
      if (vis) contrib = add(contrib, muls(eval_f(s, x1, n1), m * fmaxf_(s.W, 0.0f)));
    }
  }
  if (sel.kind == SK_NONE || selP <= 0.0f || wSum <= 0.0f) {
    out_radiance(direct);
    write_history(null_sample(fminf_(cTotal, 255.0f)));
    return;
  }
  sel.W = wSum / selP;
  sel.c = fminf_(cTotal, 255.0f);
  if (!vector) {
    bool vis = true;
    if (selJ > 0u || fullV) vis = sample_visible(W, sel, x1, n1, st);
    if (vis) contrib = muls(eval_f(sel, x1, n1), sel.W);
  }
  if (rflag(u, RF_CLAMP)) {
    float l = rlum(contrib);
    if (l > u.params4[2]) contrib = muls(contrib, u.params4[2] / l);
  }
  out_radiance(add(direct, contrib));
  write_history(sel);
}

// dupmap.wgsl:17-46 for one pixel.
float dupmap_pixel(int gx, int gy, int Wd, int Hd, const uint32_t* resB) {
  const uint32_t* mine = resB + 8 * ((size_t)gy * Wd + gx);
  if (((mine[5] >> 16) & 3u) == SK_NONE) return 0.0f;
  int count = 0;
  for (int dy = -4; dy <= 4; dy++)
    for (int dx = -4; dx <= 4; dx++) {
      if (dx == 0 && dy == 0) continue;
      int qx = gx + dx, qy = gy + dy;
      if (qx < 0 || qy < 0 || qx >= Wd || qy >= Hd) continue;
      const uint32_t* r = resB + 8 * ((size_t)qy * Wd + qx);
      if (((r[5] >> 16) & 3u) != SK_NONE && r[7] == mine[7]) count++;
    }
  return (float)count / (float)((2 * 4 + 1) * (2 * 4 + 1) - 1);
}

// ---- pairing.js -------------------------------------------------------------
// mulberry32 (pairing.js:9-17) on 32-bit integers as JavaScript's imul / >>>.
struct Mulberry {
  uint32_t a;
  double operator()() {
    a += 0x6d2b79f5u;
    uint32_t t = (a ^ (a >> 15)) * (1u | a);
    t = (t + ((t ^ (t >> 7)) * (61u | t))) ^ t;
    return (double)(t ^ (t >> 14)) / 4294967296.0;
  }
};

// makePairingTexture (pairing.js:26-70)
void pairing_texture(int S, double sigma, uint32_t seed, uint32_t* out) {
  Mulberry rand{seed};
  std::vector<int> link((size_t)S * S);
  for (int y = 0; y < S; y++)
    for (int x = 0; x < S; x++) link[(size_t)y * S + x] = (x >> 1) + (S >> 1) * y;
  // shuffleCount (pairing.js:20-24)
  int n = std::max(1, (int)std::floor((sigma * sigma) / 2 + 1.46 / sigma + 1.76 / (sigma * sigma) +
                                      0.656 / std::pow(sigma, 3.0) + 0.5));
  int cell[4];
  for (int it = 0; it < n; it++) {
    int o = it & 1;
    for (int by = 0; by < S; by += 2)
      for (int bx = 0; bx < S; bx += 2) {
        int xs[2] = {(bx + o) % S, (bx + o + 1) % S};
        int ys[2] = {(by + o) % S, (by + o + 1) % S};
        cell[0] = ys[0] * S + xs[0]; cell[1] = ys[0] * S + xs[1];
        cell[2] = ys[1] * S + xs[0]; cell[3] = ys[1] * S + xs[1];
        for (int i = 3; i > 0; i--) {
          int j = (int)(rand() * (i + 1));
          std::swap(link[(size_t)cell[i]], link[(size_t)cell[j]]);
        }
      }
  }
  std::vector<int> first(((size_t)S * S) >> 1, -1);
  auto wrap = [S](int d) {
    int w = d % S;
    if (w > S / 2) w -= S;
    if (w < -S / 2) w += S;
    return w;
  };
  for (int i = 0; i < S * S; i++) {
    int l = link[(size_t)i];
    if (first[(size_t)l] < 0) { first[(size_t)l] = i; continue; }
    int a = first[(size_t)l], b = i;
    int dx = wrap((b % S) - (a % S));
    int dy = wrap(b / S - a / S);
    out[a] = ((uint32_t)(dy & 0xffff) << 16) | (uint32_t)(dx & 0xffff);
    out[b] = ((uint32_t)(-dy & 0xffff) << 16) | (uint32_t)(-dx & 0xffff);
  }
}

}  // namespace

// ============================================================================
// C ABI (ctypes) -- every function is test infrastructure.
// ============================================================================
extern "C" {

struct OrcHit {           // 48 bytes, same field meaning as VrtHit in include/vrt.h
  float t; float n[3]; uint32_t mat;
  int32_t voxel[3]; int32_t face;
  uint32_t steps;         // outer + inner iterations entered
  uint32_t bytes;         // 4 * (brick words + mask words + voxel words read)
  uint32_t pad;
};

struct OrcStats { uint64_t rays, outer, inner, vreads, pixels; };

int orc_version(void) { return 1; }

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// scene.js:411-433 -- brick occupancy word (1 if any voxel solid) and 16 mask
// words per brick with bit = lx + 8 ly + 64 lz.
void orc_build_bricks(const uint32_t* vox, int N, uint32_t* bricks, uint32_t* masks) {
  const int BG = N / BRICK;
  const size_t nb = (size_t)BG * BG * BG;
  std::memset(masks, 0, nb * 16 * sizeof(uint32_t));
  for (int bz = 0; bz < BG; bz++)
    for (int by = 0; by < BG; by++)
      for (int bx = 0; bx < BG; bx++) {
        uint32_t occ = 0;
        size_t bi = (size_t)bx + (size_t)by * BG + (size_t)bz * BG * BG;
        for (int z = bz * BRICK; z < (bz + 1) * BRICK; z++)
          for (int y = by * BRICK; y < (by + 1) * BRICK; y++)
            for (int x = bx * BRICK; x < (bx + 1) * BRICK; x++)
              if (vox[(size_t)x + (size_t)y * N + (size_t)z * N * N] != 0u) {
                occ = 1;
                int bit = (x - bx * BRICK) + (y - by * BRICK) * BRICK + (z - bz * BRICK) * BRICK * BRICK;
                masks[bi * 16 + (bit >> 5)] |= 1u << (bit & 31);
              }
        bricks[bi] = occ;
      }
}

static void fill_hit(const Hit& h, OrcHit& o) {
  o.t = h.t; o.n[0] = h.n.x; o.n[1] = h.n.y; o.n[2] = h.n.z; o.mat = h.mat;
  o.voxel[0] = h.vx; o.voxel[1] = h.vy; o.voxel[2] = h.vz;
  o.face = h.t >= 0.0f ? face_of(h.n) : -1;
  o.steps = h.outer + h.inner;
  o.bytes = 4u * (h.outer + h.inner + h.vreads);
  o.pad = 0;
}

// voxel.wgsl:73-153 over a batch of rays (origins in metres, unit dirs, maxT metres).
void orc_trace(const uint32_t* vox, const uint32_t* bricks, const uint32_t* masks, int N,
               const float* o, const float* d, const float* tmax, int n, OrcHit* out) {
  World W{vox, bricks, masks, N, N / BRICK};
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    Hit h = trace(W, mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]), tmax[i]);
    fill_hit(h, out[i]);
  }
}

// Per-voxel DDA on the same packed-u32 layout (no brick level), in double
// precision -- the equivalence check pattern of VoxelBench harness.cpp:205-239.
// Returns the first solid voxel along the ray within tmax (metres) and its
// entry face.  Origins inside the grid only; the origin voxel is tested too.
void orc_trace_naive(const uint32_t* vox, int N, const float* o, const float* d, const float* tmax,
                     int n, OrcHit* out) {
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    OrcHit& r = out[i];
    std::memset(&r, 0, sizeof(r));
    r.t = -1.0f; r.face = -1; r.voxel[0] = r.voxel[1] = r.voxel[2] = -1;
    double ox = (double)o[3 * i] * 16.0, oy = (double)o[3 * i + 1] * 16.0, oz = (double)o[3 * i + 2] * 16.0;
    double dx = d[3 * i], dy = d[3 * i + 1], dz = d[3 * i + 2];
    double tm = (double)tmax[i] * 16.0;
    int x = (int)std::floor(ox), y = (int)std::floor(oy), z = (int)std::floor(oz);
    if (x < 0 || y < 0 || z < 0 || x >= N || y >= N || z >= N) continue;
    int sx = dx > 0 ? 1 : -1, sy = dy > 0 ? 1 : -1, sz = dz > 0 ? 1 : -1;
    double idx = 1.0 / (std::fabs(dx) + 1e-300), idy = 1.0 / (std::fabs(dy) + 1e-300), idz = 1.0 / (std::fabs(dz) + 1e-300);
    double tx = (sx > 0 ? (x + 1 - ox) : (ox - x)) * idx;
    double ty = (sy > 0 ? (y + 1 - oy) : (oy - y)) * idy;
    double tz = (sz > 0 ? (z + 1 - oz) : (oz - z)) * idz;
    double t = 0.0; int face = -1;
    for (int it = 0; it < 4 * N + 8; it++) {
      if (t > tm) break;
      uint32_t m = vox[(size_t)x + (size_t)y * N + (size_t)z * N * N];
      if (m != 0u) {
        r.t = (float)(t / 16.0); r.mat = m; r.voxel[0] = x; r.voxel[1] = y; r.voxel[2] = z; r.face = face;
        break;
      }
      if (tx <= ty && tx <= tz) { t = tx; tx += idx; x += sx; face = sx > 0 ? 1 : 0; }
      else if (ty <= tz) { t = ty; ty += idy; y += sy; face = sy > 0 ? 3 : 2; }
      else { t = tz; tz += idz; z += sz; face = sz > 0 ? 5 : 4; }
      if (x < 0 || y < 0 || z < 0 || x >= N || y >= N || z >= N) break;
    }
  }
}

// pathtrace.wgsl:248-330 (plain branch) for rows [row0, row1) stepping row_step.
// rad16: rgba16f bits W*H*4; rad32 (optional): fp32 radiance W*H*4;
// alb8: rgba8 W*H*4; gbuf: rgba32f W*H*4.  Rows not visited are untouched.
void orc_pathtrace_sig(const uint32_t* vox, const uint32_t* bricks, const uint32_t* masks, int N,
                       const void* uniforms, float fclamp, int Wd, int Hd, int row0, int row1, int row_step,
                       uint16_t* rad16, float* rad32, uint8_t* alb8, float* gbuf, OrcStats* stats, uint32_t* sig);

void orc_pathtrace(const uint32_t* vox, const uint32_t* bricks, const uint32_t* masks, int N,
                   const void* uniforms, float fclamp, int Wd, int Hd, int row0, int row1, int row_step,
                   uint16_t* rad16, float* rad32, uint8_t* alb8, float* gbuf, OrcStats* stats) {
  orc_pathtrace_sig(vox, bricks, masks, N, uniforms, fclamp, Wd, Hd, row0, row1, row_step, rad16, rad32, alb8, gbuf,
                    stats, nullptr);
}

// orc_pathtrace plus, when sig is given, the per-pixel path signature (W*H u32).
void orc_pathtrace_sig(const uint32_t* vox, const uint32_t* bricks, const uint32_t* masks, int N,
                       const void* uniforms, float fclamp, int Wd, int Hd, int row0, int row1, int row_step,
                       uint16_t* rad16, float* rad32, uint8_t* alb8, float* gbuf, OrcStats* stats, uint32_t* sig) {
  World W{vox, bricks, masks, N, N / BRICK};
  Uni u; std::memcpy(&u, uniforms, sizeof(Uni));
  if (row_step < 1) row_step = 1;
  std::vector<int> rows;
  for (int y = row0; y < row1 && y < Hd; y += row_step) rows.push_back(y);
  uint64_t rays = 0, outer = 0, inner = 0, vreads = 0, pix = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : rays, outer, inner, vreads, pix)
  for (int ri = 0; ri < (int)rows.size(); ri++) {
    int y = rows[ri];
    PixStats st{0, 0, 0, 0, 0};
    for (int x = 0; x < Wd; x++) {
      float rad[4], gb[4]; uint8_t al[4];
      st.sig = 0u;
      path_pixel(W, u, fclamp, (uint32_t)x, (uint32_t)y, (uint32_t)Wd, (uint32_t)Hd, rad, al, gb, st);
      size_t p = (size_t)y * Wd + x;
      if (sig) sig[p] = st.sig;
      for (int c = 0; c < 4; c++) {
        if (rad16) rad16[4 * p + c] = f32_to_f16(rad[c]);
        if (rad32) rad32[4 * p + c] = rad[c];
        if (alb8) alb8[4 * p + c] = al[c];
        if (gbuf) gbuf[4 * p + c] = gb[c];
      }
    }
    rays += st.rays; outer += st.outer; inner += st.inner; vreads += st.vreads; pix += (uint64_t)Wd;
  }
  if (stats) { stats->rays = rays; stats->outer = outer; stats->inner = inner; stats->vreads = vreads; stats->pixels = pix; }
}

// temporal.wgsl:17-77.  accum_f32 selects rgba32f (1) or rgba16f (0) for the
// history (accumPrev and accumOut), as main.js:148-149 chooses by adapter.
void orc_temporal(const void* uniforms, int Wd, int Hd, const uint16_t* rad16, const float* gbufCur,
                  const void* accumPrev, const float* gbufPrev, void* accumOut, int accum_f32) {
  Uni u; std::memcpy(&u, uniforms, sizeof(Uni));
  const bool temporalOn = (u.params0[2] & 1u) != 0u;
  auto fetchPrev = [&](int x, int y, float out[4]) {
    size_t p = (size_t)y * Wd + x;
    for (int c = 0; c < 4; c++)
      out[c] = accum_f32 ? ((const float*)accumPrev)[4 * p + c] : f16_to_f32(((const uint16_t*)accumPrev)[4 * p + c]);
  };
  auto store = [&](size_t p, const float v[4]) {
    for (int c = 0; c < 4; c++) {
      if (accum_f32) ((float*)accumOut)[4 * p + c] = v[c];
      else ((uint16_t*)accumOut)[4 * p + c] = f32_to_f16(v[c]);
    }
  };
#pragma omp parallel for schedule(dynamic, 4)
  for (int gy = 0; gy < Hd; gy++) {
    for (int gx = 0; gx < Wd; gx++) {
      size_t p = (size_t)gy * Wd + gx;
      float cur[3] = {f16_to_f32(rad16[4 * p]), f16_to_f32(rad16[4 * p + 1]), f16_to_f32(rad16[4 * p + 2])};
      const float* g = gbufCur + 4 * p;
      if (g[3] < 0.0f || !temporalOn) {
        float v[4] = {cur[0], cur[1], cur[2], 1.0f};
        store(p, v);
        continue;
      }
      float uvx = ((float)gx + 0.5f) / (float)Wd;
      float uvy = ((float)gy + 0.5f) / (float)Hd;
      f3 cr = camera_ray(u, uvx, uvy);
      f3 worldPos = add(mk(u.camPos[0], u.camPos[1], u.camPos[2]), muls(cr, g[3]));
      float wp[4] = {worldPos.x, worldPos.y, worldPos.z, 1.0f};
      float pc[4];
      matvec4(u.prevViewProj, wp, pc);
      float color[3] = {cur[0], cur[1], cur[2]};
      float history = 1.0f;
      if (pc[3] > 0.0f) {
        float ndx = pc[0] / pc[3], ndy = pc[1] / pc[3];
        float pux = ndx * 0.5f + 0.5f;
        float puy = (-ndy) * 0.5f + 0.5f;
        if (pux > 0.0f && puy > 0.0f && pux < 1.0f && puy < 1.0f) {
          int ppx = std::min((int)(pux * (float)Wd), Wd - 1), ppy = std::min((int)(puy * (float)Hd), Hd - 1);
          const float* pg = gbufPrev + 4 * ((size_t)ppy * Wd + ppx);
          f3 dv = sub(worldPos, mk(u.prevCamPos[0], u.prevCamPos[1], u.prevCamPos[2]));
          float expectedT = length3(dv);
          bool depthOk = pg[3] > 0.0f && std::fabs(pg[3] - expectedT) < 0.08f * expectedT + 0.02f;
          bool normalOk = ((pg[0] * g[0] + pg[1] * g[1]) + pg[2] * g[2]) > 0.85f;
          if (depthOk && normalOk) {
            float prev[4];
            bilinear(fetchPrev, Wd, Hd, pux, puy, prev);
            history = fminf_(prev[3], u.params4[1]) + 1.0f;
            float alpha = 1.0f / history;
            for (int c = 0; c < 3; c++) color[c] = mixf(prev[c], cur[c], alpha);
          }
        }
      }
      float v[4] = {color[0], color[1], color[2], history};
      store(p, v);
    }
  }
}

// atrous.wgsl:26-83, one iteration at the given step (src/dst rgba16f).
void orc_atrous(const void* uniforms, int Wd, int Hd, const void* src, int src_f32, const float* gbuf,
                uint16_t* dst, int step) {
  (void)uniforms;
  const float K[3] = {0.375f, 0.25f, 0.0625f};
  auto fetch = [&](size_t p, float out[4]) {
    for (int c = 0; c < 4; c++)
      out[c] = src_f32 ? ((const float*)src)[4 * p + c] : f16_to_f32(((const uint16_t*)src)[4 * p + c]);
  };
#pragma omp parallel for schedule(dynamic, 4)
  for (int py = 0; py < Hd; py++) {
    for (int px = 0; px < Wd; px++) {
      size_t p = (size_t)py * Wd + px;
      float center[4]; fetch(p, center);
      const float* g = gbuf + 4 * p;
      if (g[3] < 0.0f) {
        for (int c = 0; c < 4; c++) dst[4 * p + c] = f32_to_f16(center[c]);
        continue;
      }
      float history = fmaxf_(center[3], 1.0f);
      float lumC = luminance(center);
      float relax = 2.0f / std::sqrt(history);
      float sigmaL = fmaxf_(0.08f, relax);
      // wDepth * wLum = exp(-|dt|/(0.05 t + 0.01)) * exp(-|dL|/sigmaL) evaluated
      // as exp(-(|dt| * invD + |dL| * invS)) with the two reciprocals taken once
      // per pixel: within WGSL's accuracy for '/' (2.5 ULP) and exp.
      float invD = 1.0f / (0.05f * g[3] + 0.01f);
      float invS = 1.0f / sigmaL;
      float k00 = K[0] * K[0];
      float sum[3] = {(center[0] * K[0]) * K[0], (center[1] * K[0]) * K[0], (center[2] * K[0]) * K[0]};
      float wSum = k00;
      if (kLiteral) {   // atrous.wgsl:60-79 as written
        for (int dy = -2; dy <= 2; dy++) {
          for (int dx = -2; dx <= 2; dx++) {
            if (dx == 0 && dy == 0) continue;
            int qx = px + dx * step, qy = py + dy * step;
            if (qx < 0 || qy < 0 || qx >= Wd || qy >= Hd) continue;
            size_t q = (size_t)qy * Wd + qx;
            float cq[4]; fetch(q, cq);
            const float* gq = gbuf + 4 * q;
            if (gq[3] < 0.0f) continue;
            float wKernel = K[std::abs(dx)] * K[std::abs(dy)];
            float wNormal = std::pow(fmaxf_((g[0] * gq[0] + g[1] * gq[1]) + g[2] * gq[2], 0.0f), 32.0f);
            float wDepth = std::exp(-std::fabs(g[3] - gq[3]) / (0.05f * g[3] + 0.01f));
            float wLum = std::exp(-std::fabs(lumC - luminance(cq)) / sigmaL);
            float w = ((wKernel * wNormal) * wDepth) * wLum;
            for (int c = 0; c < 3; c++) sum[c] = sum[c] + cq[c] * w;
            wSum = wSum + w;
          }
        }
        float den = fmaxf_(wSum, 1e-6f);
        float v[4] = {sum[0] / den, sum[1] / den, sum[2] / den, center[3]};
        for (int c = 0; c < 4; c++) dst[4 * p + c] = f32_to_f16(v[c]);
        continue;
      }
      for (int dy = -2; dy <= 2; dy++) {
        for (int dx = -2; dx <= 2; dx++) {
          if (dx == 0 && dy == 0) continue;
          int qx = px + dx * step, qy = py + dy * step;
          if (qx < 0 || qy < 0 || qx >= Wd || qy >= Hd) continue;
          size_t q = (size_t)qy * Wd + qx;
          float cq[4]; fetch(q, cq);
          const float* gq = gbuf + 4 * q;
          if (gq[3] < 0.0f) continue;
          float wKernel = K[std::abs(dx)] * K[std::abs(dy)];
          float nd = fmaxf_(std::fmaf(g[2], gq[2], std::fmaf(g[1], gq[1], g[0] * gq[0])), 0.0f);
          float n2 = nd * nd, n4 = n2 * n2, n8 = n4 * n4, n16 = n8 * n8, n32 = n16 * n16;   // pow(., 32)
          if (n32 == 0.0f) continue;   // zero weight: the tap adds nothing
          float e = om_exp(-std::fmaf(std::fabs(g[3] - gq[3]), invD, std::fabs(lumC - luminance(cq)) * invS));
          float w = (wKernel * n32) * e;
          for (int c = 0; c < 3; c++) sum[c] = std::fmaf(cq[c], w, sum[c]);
          wSum = wSum + w;
        }
      }
      float den = fmaxf_(wSum, 1e-6f);
      float v[4] = {sum[0] / den, sum[1] / den, sum[2] / den, center[3]};
      for (int c = 0; c < 4; c++) dst[4 * p + c] = f32_to_f16(v[c]);
    }
  }
}

// present.wgsl:40-55 as a headless pass: texel-centre fetch of the final
// illumination and the sqrt-albedo, remodulate, expose, ACES, gamma 1/2.2.
void orc_present(const void* uniforms, int Wd, int Hd, const void* finalTex, int final_f32,
                 const uint8_t* alb8, uint8_t* out_rgba8) {
  Uni u; std::memcpy(&u, uniforms, sizeof(Uni));
  const float exposure = u.params1[2];
#pragma omp parallel for schedule(static)
  for (int y = 0; y < Hd; y++) {
    for (int x = 0; x < Wd; x++) {
      size_t p = (size_t)y * Wd + x;
      for (int c = 0; c < 3; c++) {
        float il = final_f32 ? ((const float*)finalTex)[4 * p + c] : f16_to_f32(((const uint16_t*)finalTex)[4 * p + c]);
        float as = (float)alb8[4 * p + c] / 255.0f;
        float al = as * as;
        float v = (il * al) * exposure;
        float num = v * (2.51f * v + 0.03f);
        float den = v * (2.43f * v + 0.59f) + 0.14f;
        float t = clampf(num / den, 0.0f, 1.0f);
        float g = om_pow(t, 0.454545468f);   // f32(1/2.2)
        out_rgba8[4 * p + c] = unorm8(g);
      }
      out_rgba8[4 * p + 3] = 255;
    }
  }
}

// main.js:628-659: hdr = illum * (a/255) * (a/255), evaluated in double (JS
// numbers) and stored as f32.
void orc_hdr(int Wd, int Hd, const void* finalTex, int final_f32, const uint8_t* alb8, float* out_rgb) {
  for (size_t p = 0; p < (size_t)Wd * Hd; p++) {
    for (int c = 0; c < 3; c++) {
      double il = final_f32 ? (double)((const float*)finalTex)[4 * p + c]
                            : (double)f16_to_f32(((const uint16_t*)finalTex)[4 * p + c]);
      double a = (double)alb8[4 * p + c] / 255.0;
      out_rgb[3 * p + c] = (float)((il * a) * a);
    }
  }
}

// FP64 accumulation of the per-sample HDR radiance (radiance before
// demodulation = demod * albedo is not recoverable bit-exactly, so the
// accumulator sums the fp32 per-sample value rad*alb8^2/255^2 in double).
// frames [frame0, frame0+spp) with the camera of `uniforms`.
void orc_accumulate_f64(const uint32_t* vox, const uint32_t* bricks, const uint32_t* masks, int N,
                        const void* uniforms, float fclamp, int Wd, int Hd, uint32_t frame0, int spp,
                        double* accum_rgb) {
  World W{vox, bricks, masks, N, N / BRICK};
  Uni u0; std::memcpy(&u0, uniforms, sizeof(Uni));
#pragma omp parallel for schedule(dynamic, 1)
  for (int y = 0; y < Hd; y++) {
    PixStats st{0, 0, 0, 0};
    Uni u = u0;
    for (int s = 0; s < spp; s++) {
      u.params0[0] = frame0 + (uint32_t)s;
      for (int x = 0; x < Wd; x++) {
        float rad[4], gb[4]; uint8_t al[4];
        path_pixel(W, u, fclamp, (uint32_t)x, (uint32_t)y, (uint32_t)Wd, (uint32_t)Hd, rad, al, gb, st);
        size_t p = (size_t)y * Wd + x;
        for (int c = 0; c < 3; c++) {
          double a = (double)al[c] / 255.0;
          accum_rgb[3 * p + c] += ((double)rad[c] * a) * a;
        }
      }
    }
  }
}

// Camera matrices (math.js:3-74, camera.js:47-57), evaluated in double like
// JavaScript and stored as f32.  out: viewProj[16], invViewProj[16].
static void js_mul(const float* a, const float* b, float* out) {
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) {
      double s = 0.0;
      for (int k = 0; k < 4; k++) s += (double)a[k * 4 + r] * (double)b[c * 4 + k];
      out[c * 4 + r] = (float)s;
    }
}

void orc_camera_matrices(const double pos[3], double yaw, double pitch, double fovY, double aspect,
                         double nearZ, double farZ, float* viewProj, float* invViewProj) {
  double f = 1.0 / std::tan(fovY / 2.0);
  float P[16] = {0}, IP[16] = {0};
  P[0] = (float)(f / aspect); P[5] = (float)f; P[10] = (float)(farZ / (nearZ - farZ)); P[11] = -1.0f;
  P[14] = (float)((nearZ * farZ) / (nearZ - farZ));
  IP[0] = (float)(aspect / f); IP[5] = (float)(1.0 / f); IP[11] = (float)((nearZ - farZ) / (nearZ * farZ));
  IP[14] = -1.0f; IP[15] = (float)(1.0 / nearZ);
  double cp = std::cos(pitch), sp = std::sin(pitch), cy = std::cos(yaw), sy = std::sin(yaw);
  double fw[3] = {sy * cp, sp, cy * cp};
  double rt[3] = {-cy, 0.0, sy};
  double up[3] = {rt[1] * fw[2] - rt[2] * fw[1], rt[2] * fw[0] - rt[0] * fw[2], rt[0] * fw[1] - rt[1] * fw[0]};
  float C2W[16] = {(float)rt[0], (float)rt[1], (float)rt[2], 0.0f,
                   (float)up[0], (float)up[1], (float)up[2], 0.0f,
                   (float)-fw[0], (float)-fw[1], (float)-fw[2], 0.0f,
                   (float)pos[0], (float)pos[1], (float)pos[2], 1.0f};
  double z[3] = {-fw[0], -fw[1], -fw[2]};
  auto dt = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  float W2C[16] = {(float)rt[0], (float)up[0], (float)z[0], 0.0f,
                   (float)rt[1], (float)up[1], (float)z[1], 0.0f,
                   (float)rt[2], (float)up[2], (float)z[2], 0.0f,
                   (float)-dt(rt, pos), (float)-dt(up, pos), (float)-dt(z, pos), 1.0f};
  js_mul(P, W2C, viewProj);
  js_mul(C2W, IP, invViewProj);
}

// World generator, restated from scene.js generateScene(N, 'default')
// (scene.js:203-222 noise, 232-264 terrain, 266-301 room, 362-374 light strip
// and boxes, 376-408 trees, lanterns and corner lamp) with the noise seed as a
// parameter (the reference fixes it at 1337), plus the benchmark world of the
// plain-frame workload: the same terrain and room, 40 trees placed by a PCG
// hash chain outside the room and the camera corridor, and red / green / blue
// lanterns of intensity 15.  JavaScript's doubles and int32 wrap-around are
// reproduced with double and 32-bit unsigned arithmetic.  The bench's CPU
// reference arm uses it so that its process loads no product library.
}  // extern "C"

namespace world {
constexpr double kVS = 1.0 / 16.0;
inline uint32_t M(int r, int g, int b, int e = 0) {
  return (uint32_t)r | ((uint32_t)g << 8) | ((uint32_t)b << 16) | ((uint32_t)e << 24);
}
inline int V(double m) { return (int)std::floor(m / kVS + 0.5); }
inline int fl(double x) { return (int)std::floor(x); }
struct Gen {
  int N; uint32_t* vox; int64_t seed;
  std::vector<int> heights;
  int cx, cz, x0, x1, z0, z1, floorY, y1, roomW, roomH;
  void set(int x, int y, int z, uint32_t m) {
    if (x >= 0 && y >= 0 && z >= 0 && x < N && y < N && z < N) vox[(size_t)x + (size_t)y * N + (size_t)z * N * N] = m;
  }
  template <class F> void boxf(int ax, int ay, int az, int bx, int by, int bz, F f) {
    for (int z = az; z <= bz; z++) for (int y = ay; y <= by; y++) for (int x = ax; x <= bx; x++) set(x, y, z, f(x, z));
  }
  void box(int ax, int ay, int az, int bx, int by, int bz, uint32_t m) {
    boxf(ax, ay, az, bx, by, bz, [m](int, int) { return m; });
  }
  double hash(int64_t x, int64_t y) const {        // (x*374761393 + y*668265263 + seed*1442695041) | 0, Math.imul
    uint32_t h = (uint32_t)((uint64_t)x * 374761393ull + (uint64_t)y * 668265263ull + (uint64_t)seed * 1442695041ull);
    h = (h ^ (h >> 13)) * 1274126177u;
    return (double)(h ^ (h >> 16)) / 4294967296.0;
  }
  double noise(double x, double y) const {
    double v = 0.0, amp = 0.5, f = 1.0;
    for (int o = 0; o < 4; o++) {
      const double px = x * f, py = y * f, xi = std::floor(px), yi = std::floor(py);
      auto sm = [](double t) { return t * t * (3 - 2 * t); };
      const double xf = sm(px - xi), yf = sm(py - yi);
      const int64_t X = (int64_t)xi, Y = (int64_t)yi;
      const double a = hash(X, Y), b = hash(X + 1, Y), c = hash(X, Y + 1), d = hash(X + 1, Y + 1);
      v += (a + (b - a) * xf + (c - a) * yf + (a - b - c + d) * xf * yf) * amp;
      amp *= 0.5; f *= 2.0;
    }
    return v;
  }
  int ground(int x, int z) const { return heights[std::max(0, std::min(N - 1, x)) + std::max(0, std::min(N - 1, z)) * N]; }
  void terrain() {
    const int baseH = fl(N * 0.16);
    heights.assign((size_t)N * N, 0);
    for (int z = 0; z < N; z++)
      for (int x = 0; x < N; x++) {
        const int h = baseH + fl(noise(x * 0.02, z * 0.02) * N * 0.10);
        heights[x + z * N] = h;
        for (int y = 0; y <= h && y < N; y++) {
          const int v = (x * 7 + y * 13 + z * 5) % 9;
          vox[(size_t)x + (size_t)y * N + (size_t)z * N * N] =
              y == h ? M(88 + v, 130 + v, 60) : (y > h - 4 ? M(110 + v, 82 + v, 58) : M(120 + v, 120 + v, 125 + v));
        }
      }
  }
  void room() {
    roomW = std::min(V(5), fl(N * 0.45));
    roomH = std::min(V(3.2), fl(N * 0.3));
    cx = fl(N * 0.5); cz = fl(N * 0.55);
    x0 = cx - (roomW >> 1); x1 = cx + (roomW >> 1); z0 = cz - (roomW >> 1); z1 = cz + (roomW >> 1);
    floorY = ground(cx, cz) + 1; y1 = floorY + roomH;
    const int T = 2;
    boxf(x0 - T, floorY, z0 - T, x1 + T, floorY, z1 + T, [](int x, int z) { const int v = (x + z) % 9; return M(110 + v, 82 + v, 58); });
    box(x0 - T, floorY + 1, z0 - T, x1 + T, y1 + T + 4, z1 + T, 0);
    boxf(x0 - T, floorY, z0 - T, x1 + T, floorY, z1 + T,
         [](int x, int z) { return ((x >> 3) + (z >> 3)) % 2 ? M(180, 150, 110) : M(150, 118, 84); });
    const uint32_t white = M(225, 222, 215);
    box(x0 - T, floorY + 1, z1 + 1, x1 + T, y1, z1 + T, white);
    box(x0 - T, floorY + 1, z0 - T, x1 + T, y1, z0 - 1, white);
    box(x0 - T, floorY + 1, z0 - T, x0 - 1, y1, z1 + T, M(200, 45, 40));
    box(x1 + 1, floorY + 1, z0 - T, x1 + T, y1, z1 + T, M(55, 175, 60));
    box(x0 - T, y1 + 1, z0 - T, x1 + T, y1 + T, z1 + T, white);
    const int doorHalf = fl(roomW * 0.28);
    box(cx - doorHalf, floorY + 1, z0 - T, cx + doorHalf, y1 - 2, z0 - 1, 0);
    box(x1 + 1, floorY + fl(roomH * 0.45), cz - fl(roomW * 0.3), x1 + T, floorY + fl(roomH * 0.8), cz + fl(roomW * 0.3), 0);
    const int lHalf = fl(roomW * 0.18);
    box(cx - lHalf, y1, cz - lHalf, cx + lHalf, y1, cz + lHalf, M(255, 240, 220, 210));
    const int tallW = fl(roomW * 0.16), tallH = fl(roomH * 0.55);
    box(cx - fl(roomW * 0.28) - tallW, floorY + 1, cz + fl(roomW * 0.05), cx - fl(roomW * 0.28), floorY + tallH,
        cz + fl(roomW * 0.05) + tallW, M(200, 200, 210));
    const int shortW = fl(roomW * 0.18), shortH = fl(roomH * 0.28);
    box(cx + fl(roomW * 0.10), floorY + 1, cz - fl(roomW * 0.25), cx + fl(roomW * 0.10) + shortW, floorY + shortH,
        cz - fl(roomW * 0.25) + shortW, M(210, 170, 90));
  }
  void tree(int tx, int tz) {
    const int g = ground(tx, tz);
    const int trunkH = V(1.4) + ((tx * 31 + tz * 17) % V(0.8));
    for (int y = g + 1; y <= g + trunkH; y++) { set(tx, y, tz, M(95, 68, 42)); set(tx + 1, y, tz, M(95, 68, 42)); }
    const int cy = g + trunkH + V(0.35), r = V(0.7) + ((tx + tz) % 3);
    for (int dz = -r; dz <= r; dz++)
      for (int dy = -r; dy <= r; dy++)
        for (int dx = -r; dx <= r; dx++) {
          const double d2 = dx * dx + dy * dy * 1.6 + dz * dz;
          if (d2 <= r * r && ((dx * 13 + dy * 7 + dz * 11) % 5 != 0 || d2 < r * r * 0.5)) {
            const int v = (dx * 3 + dy * 5 + dz * 7) % 12 + ((dx + dy + dz) % 2) * 6;
            set(tx + dx, cy + dy, tz + dz, M(50 + v, 120 + v, 45));
          }
        }
  }
  void lantern(int lx, int lz, uint32_t m) {
    const int g = ground(lx, lz), h = V(1.1);
    for (int y = g + 1; y <= g + h; y++) set(lx, y, lz, M(60, 60, 65));
    box(lx - 1, g + h + 1, lz - 1, lx + 1, g + h + 3, lz + 1, m);
  }
};
inline uint32_t pcg_step(uint32_t v) {
  v = v * 747796405u + 2891336453u;
  const uint32_t w = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  return (w >> 22u) ^ w;
}
}  // namespace world

extern "C" {

// kind 0: the reference world (scene.js 'default'); kind 2: the benchmark
// world.  spawn (8 doubles): x, y, z, yaw, pitch, vertical fov, near, far.
int orc_scene_generate(int kind, int N, uint32_t seed, uint32_t* vox, double* spawn) {
  using namespace world;
  if ((kind != 0 && kind != 2) || N < 8 || N % 8 != 0) return 1;
  std::memset(vox, 0, (size_t)N * N * N * sizeof(uint32_t));
  Gen g{N, vox, (int64_t)seed, {}, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  g.terrain();
  g.room();
  const uint32_t lampWarm = M(255, 190, 110, 255);
  if (kind == 0) {
    const double spots[6][2] = {{0.15, 0.2}, {0.82, 0.25}, {0.2, 0.8}, {0.86, 0.78}, {0.12, 0.55}, {0.65, 0.12}};
    for (auto& sp : spots) g.tree(fl(N * sp[0]), fl(N * sp[1]));
    g.lantern(fl(N * 0.35), fl(N * 0.25), lampWarm);
    g.lantern(fl(N * 0.68), fl(N * 0.30), M(90, 220, 255, 255));
    g.lantern(fl(N * 0.25), fl(N * 0.65), M(255, 90, 200, 255));
    g.box(g.x0 + 2, g.floorY + 1, g.z1 - 4, g.x0 + 4, g.floorY + 3, g.z1 - 2, lampWarm);
    if (spawn) {
      const double s[8] = {g.cx * kVS, (g.ground(g.cx, g.z0 - V(3)) + 1) * kVS + 1.65, (g.z0 - V(3.5)) * kVS, 0.0,
                           -0.05, 70.0 * M_PI / 180.0, 0.05, 400.0};
      std::memcpy(spawn, s, sizeof s);
    }
    return 0;
  }
  // benchmark world: seeded trees outside the room and the camera corridor
  const int corX0 = g.cx - 24, corX1 = g.cx + 24;
  uint32_t st = pcg_step(seed * 2654435761u + 17u);
  auto uni = [&]() { st = pcg_step(st); return (double)st / 4294967296.0; };
  int placed = 0;
  for (int attempt = 0; attempt < 4000 && placed < 40; attempt++) {
    const int tx = fl(N * (0.05 + 0.90 * uni()));
    const int tz = fl(N * (0.05 + 0.90 * uni()));
    const int margin = V(0.7) + 3;
    const bool inRoom = tx >= g.x0 - 2 - margin && tx <= g.x1 + 2 + margin && tz >= g.z0 - 2 - margin &&
                        tz <= g.z1 + 2 + margin;
    const bool inCorridor = tx >= corX0 - margin && tx <= corX1 + margin && tz < g.z0;
    if (inRoom || inCorridor) continue;
    g.tree(tx, tz);
    placed++;
  }
  const int E = std::min(255, std::max(1, (int)std::floor(15.0 * 255.0 / 24.0 + 0.5)));
  g.lantern(fl(N * 0.35), fl(N * 0.25), M(255, 40, 40, E));
  g.lantern(fl(N * 0.68), fl(N * 0.30), M(40, 255, 40, E));
  g.lantern(fl(N * 0.25), fl(N * 0.65), M(40, 40, 255, E));
  g.box(g.x0 + 2, g.floorY + 1, g.z1 - 4, g.x0 + 4, g.floorY + 3, g.z1 - 2, lampWarm);
  if (spawn) {
    const int zStart = std::max(2, g.z0 - 60);
    int gmax = g.floorY - 1;
    for (int z = zStart; z <= g.z0; z++)
      for (int x = g.cx - 16; x <= g.cx + 16; x++) gmax = std::max(gmax, g.ground(x, z));
    const double s[8] = {g.cx * kVS, (gmax + 1) * kVS + 1.65, zStart * kVS, -30.0 * M_PI / 180.0, -0.05,
                         60.0 * M_PI / 180.0, 0.05, 400.0};
    std::memcpy(spawn, s, sizeof s);
  }
  return 0;
}

// Scalar checks of the project transcendentals and storage conversions.
void orc_math_eval(int fn, const float* x, float* y, int n) {
  for (int i = 0; i < n; i++) {
    float s, c;
    switch (fn) {
      case 0: om_sincos(x[i], s, c); y[i] = s; break;
      case 1: om_sincos(x[i], s, c); y[i] = c; break;
      case 2: y[i] = om_exp(x[i]); break;
      case 3: y[i] = om_log2(x[i]); break;
      case 4: y[i] = om_pow(x[i], 0.55f); break;
      case 5: y[i] = om_pow(x[i], 0.454545468f); break;
      case 6: y[i] = f16_to_f32(f32_to_f16(x[i])); break;
      default: y[i] = NAN;
    }
  }
}

uint32_t orc_pcg_hash(uint32_t v) { return pcg_hash(v); }

// ---------------------------------------------------------------------------
// Emissive-face light list, power alias table and per-brick light grid
// (scene.js:58-200, 435-461).  JavaScript numbers are doubles and typed-array
// stores round: the restatement computes in double and rounds where the
// reference stores into a Float32Array.
// ---------------------------------------------------------------------------
static double light_weight(uint32_t m) {   // emissiveFaceWeight, scene.js:58-65
  const double e = (double)((m >> 24) & 0xffu) / 255.0;
  if (e <= 0.0) return 0.0;
  const double r = (double)(m & 0xffu) / 255.0;
  const double g = (double)((m >> 8) & 0xffu) / 255.0;
  const double b = (double)((m >> 16) & 0xffu) / 255.0;
  return e * (((0.2126 * r) * r + (0.7152 * g) * g) + (0.0722 * b) * b);
}

// Light list (scene.js:435-456): voxels in z, y, x order, faces +x,-x,+y,-y,+z,-z;
// a face is a light when its neighbour is outside the grid or air.  Writes
// at most `cap` lights (2 words each) and weights; returns the count.
long orc_light_list(const uint32_t* vox, int N, uint32_t* words, double* weights, long cap) {
  static const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  long n = 0;
  for (int z = 0; z < N; z++)
    for (int y = 0; y < N; y++)
      for (int x = 0; x < N; x++) {
        const uint32_t m = vox[(size_t)x + (size_t)y * N + (size_t)z * N * N];
        if (((m >> 24) & 0xffu) == 0u || m == 0u) continue;
        const double w = light_weight(m);
        for (int f = 0; f < 6; f++) {
          const int nx = x + D[f][0], ny = y + D[f][1], nz = z + D[f][2];
          const bool in = nx >= 0 && ny >= 0 && nz >= 0 && nx < N && ny < N && nz < N;
          if (!in || vox[(size_t)nx + (size_t)ny * N + (size_t)nz * N * N] == 0u) {
            if (n < cap) {
              words[2 * n] = (uint32_t)x | ((uint32_t)y << 9) | ((uint32_t)z << 18) | ((uint32_t)f << 27);
              words[2 * n + 1] = m;
              weights[n] = w;
            }
            n++;
          }
        }
      }
  return n;
}

// makeAliasTable (scene.js:67-104): table[4i..4i+3] = (q, alias, prob, 0) as float32.
void orc_light_alias(const double* weights, long n, float* table) {
  if (n == 0) { table[0] = 1.0f; table[1] = 0.0f; table[2] = 1.0f; table[3] = 0.0f; return; }
  double total = 0.0;
  for (long i = 0; i < n; i++) total += weights[i] > 0.0 ? weights[i] : 0.0;
  std::vector<double> prob((size_t)n), scaled((size_t)n);
  for (long i = 0; i < n; i++) {
    prob[(size_t)i] = total > 0.0 ? (weights[i] > 0.0 ? weights[i] : 0.0) / total : 1.0 / (double)n;
    scaled[(size_t)i] = prob[(size_t)i] * (double)n;
  }
  std::vector<uint32_t> alias((size_t)n, 0u);
  std::vector<float> q((size_t)n, 0.0f);
  std::vector<long> small, large;
  for (long i = 0; i < n; i++) (scaled[(size_t)i] < 1.0 ? small : large).push_back(i);
  while (!small.empty() && !large.empty()) {
    const long sidx = small.back(); small.pop_back();
    const long l = large.back(); large.pop_back();
    q[(size_t)sidx] = (float)scaled[(size_t)sidx];
    alias[(size_t)sidx] = (uint32_t)l;
    scaled[(size_t)l] = (scaled[(size_t)l] + scaled[(size_t)sidx]) - 1.0;
    (scaled[(size_t)l] < 1.0 ? small : large).push_back(l);
  }
  for (long i : large) { q[(size_t)i] = 1.0f; alias[(size_t)i] = (uint32_t)i; }
  for (long i : small) { q[(size_t)i] = 1.0f; alias[(size_t)i] = (uint32_t)i; }
  for (long i = 0; i < n; i++) {
    table[4 * i + 0] = q[(size_t)i];
    table[4 * i + 1] = (float)alias[(size_t)i];
    table[4 * i + 2] = (float)(prob[(size_t)i] > 0.0 ? prob[(size_t)i] : 1.0 / (double)n);
    table[4 * i + 3] = 0.0f;
  }
}

// buildLightGrid (scene.js:106-200): per brick cell (BG^3 cells, 34 words
// each) the top-16 lights by power / max(d^2, 16) with a facing test.
void orc_light_grid(int N, const uint32_t* words, const double* weights, long n, uint32_t* grid) {
  const int BG = N / BRICK, K = 16, STRIDE = 2 + 2 * K;
  std::vector<float> fc((size_t)n * 3), fn((size_t)n * 3);
  for (long i = 0; i < n; i++) {
    const uint32_t w0 = words[2 * i];
    const int x = (int)(w0 & 0x1ffu), y = (int)((w0 >> 9) & 0x1ffu), z = (int)((w0 >> 18) & 0x1ffu);
    const int face = (int)((w0 >> 27) & 7u), axis = face >> 1, pos = (face & 1) == 0 ? 1 : 0;
    double c[3] = {x + 0.5, y + 0.5, z + 0.5}, nn[3] = {0, 0, 0};
    const int v[3] = {x, y, z};
    c[axis] = v[axis] + pos;
    nn[axis] = pos ? 1.0 : -1.0;
    for (int k = 0; k < 3; k++) { fc[3 * i + k] = (float)c[k]; fn[3 * i + k] = (float)nn[k]; }
  }
  const double eps = (BRICK / 2.0) * (BRICK / 2.0);
#pragma omp parallel for schedule(dynamic, 16)
  for (int cell = 0; cell < BG * BG * BG; cell++) {
    const int bx = cell % BG, by = (cell / BG) % BG, bz = cell / (BG * BG);
    const double ccx = (bx + 0.5) * BRICK, ccy = (by + 0.5) * BRICK, ccz = (bz + 0.5) * BRICK;
    uint32_t topIdx[16];
    float topW[16];
    int count = 0, minAt = 0;
    double minW = 0.0;
    for (long i = 0; i < n; i++) {
      const double dx = ccx - (double)fc[3 * i], dy = ccy - (double)fc[3 * i + 1], dz = ccz - (double)fc[3 * i + 2];
      if ((dx * (double)fn[3 * i] + dy * (double)fn[3 * i + 1]) + dz * (double)fn[3 * i + 2] <= 0.0) continue;
      const double d2 = (dx * dx + dy * dy) + dz * dz;
      const double w = weights[i] / (d2 > eps ? d2 : eps);
      if (count < K) {
        topIdx[count] = (uint32_t)i;
        topW[count] = (float)w;
        count++;
        if (count == K) {
          minW = topW[0]; minAt = 0;
          for (int k = 1; k < K; k++) if ((double)topW[k] < minW) { minW = topW[k]; minAt = k; }
        }
      } else if (w > minW) {
        topIdx[minAt] = (uint32_t)i;
        topW[minAt] = (float)w;
        minW = topW[0]; minAt = 0;
        for (int k = 1; k < K; k++) if ((double)topW[k] < minW) { minW = topW[k]; minAt = k; }
      }
    }
    uint32_t* g = grid + (size_t)cell * STRIDE;
    double wSum = 0.0;
    for (int k = 0; k < count; k++) wSum += (double)topW[k];
    const float wSumF = (float)wSum;
    g[0] = (uint32_t)count;
    std::memcpy(&g[1], &wSumF, 4);
    for (int k = 0; k < count; k++) {
      g[2 + 2 * k] = topIdx[k];
      std::memcpy(&g[3 + 2 * k], &topW[k], 4);
    }
    for (int k = count; k < K; k++) { g[2 + 2 * k] = 0u; g[3 + 2 * k] = 0u; }
  }
}

// Cache-assisted estimator of every pixel (OrcCachePix per pixel, row-major).
int orc_cache_pix_bytes(void) { return (int)sizeof(OrcCachePix); }

void orc_cache_paths(const uint32_t* vox, const uint32_t* bricks, const uint32_t* masks, int N,
                     const void* uniforms, int Wd, int Hd, uint32_t phase, uint32_t train_bounces,
                     int rec_vertices, OrcCachePix* out) {
  World W{vox, bricks, masks, N, N / BRICK};
  Uni u; std::memcpy(&u, uniforms, sizeof(Uni));
#pragma omp parallel for schedule(dynamic, 1)
  for (int y = 0; y < Hd; y++)
    for (int x = 0; x < Wd; x++)
      cache_pixel(W, u, (uint32_t)x, (uint32_t)y, (uint32_t)Wd, (uint32_t)Hd, phase, train_bounces, rec_vertices,
                  out[(size_t)y * Wd + x]);
}

// Runs the path of rows [row0,row1) step row_step and returns every ray it
// traced as 7 floats (origin xyz and maxT in voxel units, unit direction).
// Writes at most `cap` rays to out7; returns the total number traced.
long orc_collect_rays(const uint32_t* vox, const uint32_t* bricks, const uint32_t* masks, int N,
                      const void* uniforms, float fclamp, int Wd, int Hd, int row0, int row1, int row_step,
                      float* out7, long cap) {
  World W{vox, bricks, masks, N, N / BRICK};
  Uni u; std::memcpy(&u, uniforms, sizeof(Uni));
  if (row_step < 1) row_step = 1;
  std::vector<int> rows;
  for (int y = row0; y < row1 && y < Hd; y += row_step) rows.push_back(y);
  std::vector<std::vector<float>> logs(rows.size());
#pragma omp parallel for schedule(dynamic, 1)
  for (int ri = 0; ri < (int)rows.size(); ri++) {
    tl_ray_log = &logs[ri];
    PixStats st{0, 0, 0, 0};
    for (int x = 0; x < Wd; x++) {
      float rad[4], gb[4]; uint8_t al[4];
      path_pixel(W, u, fclamp, (uint32_t)x, (uint32_t)rows[ri], (uint32_t)Wd, (uint32_t)Hd, rad, al, gb, st);
    }
    tl_ray_log = nullptr;
  }
  long total = 0;
  for (auto& l : logs) {
    long n = (long)(l.size() / 7);
    long room = cap - total;
    if (room > 0) std::memcpy(out7 + 7 * total, l.data(), sizeof(float) * 7 * (size_t)std::min(n, room));
    total += n;
  }
  return total;
}

// ReSTIR passes over whole images (reservoirs: 8 u32 per pixel in the 32-byte
// record of restir.wgsl:14-27).  lights / alias / grid: the scene's light
// data (orc_light_*), read with RF_UNIFIED; dup: the previous frame's
// duplication map (RF_DUPMAP); pairing: the pairing buffer (RF_PAIRED).  stats
// (optional) receives the rays the pass traced.
void orc_restir_initial(const uint32_t* vox, const uint32_t* bricks, const uint32_t* masks, int N,
                        const void* uniforms, float fclamp, int Wd, int Hd, const uint32_t* lights,
                        const float* alias, const uint32_t* grid, uint16_t* rad16, float* rad32, uint8_t* alb8,
                        float* gbuf, uint32_t* resA, uint16_t* direct16, OrcStats* stats) {
  World W{vox, bricks, masks, N, N / BRICK};
  Uni u; std::memcpy(&u, uniforms, sizeof(Uni));
  RestirAux ax{lights, alias, grid, nullptr, nullptr};
  uint64_t rays = 0, outer = 0, inner = 0, vreads = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : rays, outer, inner, vreads)
  for (int y = 0; y < Hd; y++) {
    PixStats st{0, 0, 0, 0};
    for (int x = 0; x < Wd; x++)
      restir_initial_pixel(W, u, ax, fclamp, x, y, Wd, Hd, rad16, rad32, alb8, gbuf, resA, direct16, st);
    rays += st.rays; outer += st.outer; inner += st.inner; vreads += st.vreads;
  }
  if (stats) {
    stats->rays = rays; stats->outer = outer; stats->inner = inner; stats->vreads = vreads;
    stats->pixels = (uint64_t)Wd * Hd;
  }
}

void orc_restir_temporal(const void* uniforms, int Wd, int Hd, const float* gbufCur, const float* gbufPrev,
                         const uint32_t* resB, const float* dup, uint32_t* resA) {
  Uni u; std::memcpy(&u, uniforms, sizeof(Uni));
  if (!(u.params2[0] & 1u) || !(u.params2[0] & RF_TEMPORAL)) return;   // reuse_temporal.wgsl:144
  RestirAux ax{nullptr, nullptr, nullptr, nullptr, dup};
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < Hd; y++)
    for (int x = 0; x < Wd; x++) restir_temporal_pixel(u, ax, x, y, Wd, Hd, gbufCur, gbufPrev, resB, resA);
}

void orc_restir_spatial(const uint32_t* vox, const uint32_t* bricks, const uint32_t* masks, int N,
                        const void* uniforms, int Wd, int Hd, const float* gbufCur, const uint32_t* resA,
                        const uint16_t* direct16, const uint32_t* pairing, uint16_t* rad16, float* rad32,
                        uint32_t* resB, OrcStats* stats) {
  World W{vox, bricks, masks, N, N / BRICK};
  Uni u; std::memcpy(&u, uniforms, sizeof(Uni));
  RestirAux ax{nullptr, nullptr, nullptr, pairing, nullptr};
  uint64_t rays = 0, outer = 0, inner = 0, vreads = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : rays, outer, inner, vreads)
  for (int y = 0; y < Hd; y++) {
    PixStats st{0, 0, 0, 0};
    for (int x = 0; x < Wd; x++)
      restir_spatial_pixel(W, u, ax, x, y, Wd, Hd, gbufCur, resA, direct16, rad16, rad32, resB, st);
    rays += st.rays; outer += st.outer; inner += st.inner; vreads += st.vreads;
  }
  if (stats) {
    stats->rays = rays; stats->outer = outer; stats->inner = inner; stats->vreads = vreads;
    stats->pixels = 0;
  }
}

void orc_restir_dupmap(int Wd, int Hd, const uint32_t* resB, float* dup) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < Hd; y++)
    for (int x = 0; x < Wd; x++) dup[(size_t)y * Wd + x] = dupmap_pixel(x, y, Wd, Hd, resB);
}

// makePairingBuffer (pairing.js:80-89) for sigmas[3].
void orc_pairing_buffer(const double* sigmas, uint32_t* out) {
  const int sizes[3] = {254, 230, 210};
  size_t off = 0;
  for (int i = 0; i < 3; i++) {
    pairing_texture(sizes[i], sigmas[i], 0xc0ffeeu + (uint32_t)i * 7919u, out + off);
    off += (size_t)sizes[i] * sizes[i];
  }
}

}  // extern "C"
